#!/usr/bin/env python
"""bench.py -- throughput of gevolution-2.0's per-step particle-mesh cycle on B200.

Workload (default): box 2560 Mpc/h, grid 512^3, 512^3 particles, mixed
precision (FP32 fields and FFTs; particle positions as cell index + FP64
offset; FP64 background and reductions), GR weak-field gauge, elliptic B, one
full-sky lightcone shell (vertex at the box corner, 0.5-1.0 box lengths) that is
active in every timed cycle.  Seeded Zel'dovich initial conditions at z = 100
(Eisenstein-Hu no-wiggle P(k), A_s = 2.1e-9, n_s = 0.965, h = 0.67,
Omega_m = 0.32).  One "step" is one cycle of main.cu's loop: T00/Tij projection,
Phi, chi, T0i projection, B, lightcone, kick, drift, background, step control.

Metric: Mpart-steps/s = particles x cycles / second (whole job: all ranks).
Multi-GPU (torchrun): every rank evolves its own independent box (replicas;
the single-box cycle is not split across GPUs) -> weak scaling.

--impl reference times the reference's own cycle functions (ref_step in
oracle/_ref: gevolution.hpp's projections, source preparation and Fourier
solvers, update_q / update_pos and background.hpp's integrator, compiled for
the host with a single-rank LATfield2 stand-in, OpenMP over all host cores) on
a 128^3 sample box of the same physics and cell size.
"""
import argparse
import ctypes
import json
import math
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "gevolution-2.0_b200", "python"))

OMEGA_M, OMEGA_L, H_LITTLE = 0.32, 0.68, 0.67
C_LIGHT = 2997.92458
T_START = time.time()


def log(msg):
    print("[bench %7.1fs] %s" % (time.time() - T_START, msg), file=sys.stderr, flush=True)


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--N", type=int, default=512)
    p.add_argument("--boxsize", type=float, default=None, help="Mpc/h (default: 5 Mpc/h per cell)")
    p.add_argument("--z-in", type=float, default=100.0)
    p.add_argument("--seed", type=int, default=42)
    p.add_argument("--tensor", action="store_true", help="keep the h_ij / h_ij' state (full metric solve)")
    p.add_argument("--no-fp64", action="store_true", help="skip the FP64 comparison run")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--e2e-steps", type=int, default=5)
    p.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    p.add_argument("--no-adjoint", action="store_true", help="skip the differentiable-run measurement")
    p.add_argument("--no-late", action="store_true", help="skip the run on to z = 0")
    p.add_argument("--adj-N", type=int, default=128)
    p.add_argument("--adj-steps", type=int, default=32)
    p.add_argument("--adj-modes", type=int, default=64)
    p.add_argument("--cpu-sample-N", type=int, default=128)
    p.add_argument("--cpu-sample-steps", type=int, default=4)
    return p.parse_args()


# ---------------------------------------------------------------------------
# clocks sampled during the timed region (nvidia-smi, 200 ms)
# ---------------------------------------------------------------------------
class Clocks:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    # started before the warm-up so that the sampler is running when the timed
    # region begins; samples are kept by their arrival time within the region
    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.proc = None
        self.lines = []
        self.t0 = self.t1 = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.idx), "--query-gpu=" + self.Q, "--format=csv,noheader,nounits",
                                          "-lms", "50"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, ValueError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.time(), line.strip()))

    def begin(self):
        self.t0 = time.time()

    def end(self):
        self.t1 = time.time()

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.1)   # let the sample taken at the end of the region arrive
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        t0 = self.t0 if self.t0 is not None else 0.0
        t1 = (self.t1 if self.t1 is not None else time.time()) + 0.06
        sm, mx, reasons = [], None, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ts, ln in list(self.lines):
            if ts < t0 or ts > t1:
                continue
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return d["hbm_gbs"], "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
def lightcone_args(gev, d):
    """Full-sky shell, vertex at the box corner, comoving radius 0.5-1.0 box lengths."""
    return gev.LightconeArgs((0.0, 0.0, 0.0), (1.0 / math.sqrt(3),) * 3, -1.0, (1.0, 0.5), d, 1, 0)


SINGLE_KERNEL_STAGES = ("deposit_T00_Tij_T0i",)

# DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum) from one
# ncu --set full capture of each deposit kernel at 256^3 in mixed precision
# (python bench.py --N 256 --steps 2 --warmup 3 --no-fp64 --no-e2e --no-cpu
# --no-adjoint --no-late under ncu -k regex:"k_deposit<float, \(int\)4" for the
# cycle's deposit, its tile launch, plus its dense-tile launch (0.07 MB) from
# the capture of the two-launch form; the separate T00+Tij and T0i kernels
# from the earlier capture of the single-launch form), scaled by the particle
# count; the profiles/ summaries record the captures.  The cycle's deposit was
# captured with one vertex per thread; the two-vertex tile launch reads and
# writes the same global arrays (it changes only how often a record is read
# from shared memory).
NCU_TRAFFIC_256 = {"deposit_T00_Tij_T0i": 0.7499e9 + 0.6387e9 + 0.0001e9, "deposit_T00_Tij": 0.7451e9 + 0.4423e9,
                   "deposit_T0i": 0.7434e9 + 0.1865e9}


def ncu_traffic(stage, N):
    t = NCU_TRAFFIC_256.get(stage)
    return None if t is None else t * (N / 256.0) ** 3


def workload_config(N, box, world, tensor=False):
    return {"workload": "PM cycle, box %g Mpc/h, grid %d^3, %d^3 particles, mixed precision, GR, elliptic B%s, "
                        "full-sky lightcone shell 0.5-1.0 box lengths" % (box, N, N, ", h_ij evolved" if tensor else ""),
            "N": N, "particles": N ** 3, "boxsize_mpc_h": box, "tensor": bool(tensor),
            "parallelism": "replicas" if world > 1 else "single GPU",
            "l2": "inputs larger than L2 (particles %.1f GB, fields %.1f GB)" % (N ** 3 * 48 / 1e9, N ** 3 * 12 * 4 / 1e9)}


def max_over_ranks(ms, world, device):
    """The slowest rank's duration: every rank takes part in the same all-reduce."""
    import torch
    t = torch.tensor([float(ms)], device=device, dtype=torch.float64)
    if world > 1:
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def job_rate(world, particles_per_rank, cycles, ms_max):
    """Whole-job Mpart-steps/s: every replica advances its own particles."""
    return world * particles_per_rank * cycles / (ms_max * 1e-3) / 1e6


def run_gpu(args, rank, world, local_rank):
    import numpy as np
    import torch

    import gevb200 as gev
    from gevb200 import roofline
    from gevb200.ics import linear_pk, sc1_template

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    N = args.N
    box = args.boxsize or 5.0 * N
    np_ = N ** 3
    log("initial conditions %d^3" % N)
    # the reference's initial conditions (generateIC_basic's tabulated-spectrum
    # branch, gev_ics_basic) in FP64: the linear EH no-wiggle P(k) at z_in, the
    # sc1 template tiled N/4 times, k-sphere, corrected displacement; every
    # replica has its own seed
    a0 = 1.0 / (1.0 + args.z_in)
    fourpiG = 1.5 * box * box / C_LIGHT ** 2
    mass = OMEGA_M / np_
    kt = np.logspace(-5, 3, 4096)
    pt = linear_pk(kt, a0, H_LITTLE, OMEGA_M)
    with gev.Context(N, precision=gev.FP64, capacity=np_, boxsize=box, device=local_rank) as gen:
        gen.ics_basic(box, a0, fourpiG, OMEGA_M, OMEGA_L, kt, pt, sc1_template(), N // 4,
                      seed=args.seed + 1000 * rank, ksphere=True, correct_displacement=True, gr=True)
        p_, q_, i_ = gen.get_particles()
        phi_h = gen.get_field(gev.FIELD_PHI).ravel()
        chi_h = gen.get_field(gev.FIELD_CHI).ravel()
    log("initial conditions done")
    # host copies in pinned memory: the C ABI takes host buffers
    pos_h = torch.from_numpy(p_).pin_memory().numpy()
    q_h = torch.from_numpy(q_).pin_memory().numpy()
    ids_h = torch.from_numpy(i_).pin_memory().numpy()
    del p_, q_, i_

    z_relax = args.z_in
    cosmo = gev.Cosmo(OMEGA_M, OMEGA_L, 0.0, fourpiG, 48.0, 0.04, z_relax, box)
    H = gev.hconf(a0, fourpiG, ctypes.byref(cosmo))
    dtau0 = min(48.0 / N, 0.04 / H)
    tau0 = gev.particle_horizon(a0, fourpiG, ctypes.byref(cosmo))
    # the crossing surface d - tau starts just inside the shell's outer limit (1.0
    # box lengths) and moves inward by the conformal time of each cycle: over the
    # warm-up and timed cycles from z = 100 (tau grows by about 2 % per cycle) it
    # stays inside [0.5, 1.0], so every cycle writes a populated shell
    d_lc = tau0 + 0.98
    lc = lightcone_args(gev, d_lc)
    lc_cap = int(0.2 * np_)

    def make(precision):
        c = gev.Context(N, precision=precision, capacity=np_, boxsize=box, vector_method=gev.VECTOR_ELLIPTIC,
                        tensor=args.tensor, device=local_rank)
        c.set_particles(pos_h, q_h, ids_h, mass)
        c.set_field(gev.FIELD_PHI, phi_h)
        c.set_field(gev.FIELD_CHI, chi_h)
        return c

    def cycle(c, st):
        """One cycle of main.cu's loop with the lightcone between the solves and
        the kick; returns the number of particles the shell selected."""
        return c.step_lightcone(cosmo, st, lc, lc_cap)

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    mem_used = {}

    def timed_run(precision, steps, warmup):
        log("context (%s)" % ("fp64" if precision == gev.FP64 else "mixed"))
        c = make(precision)
        st = gev.State(a0, tau0, dtau0, 0.0, 0, 0.0, 0.0, 0.0)
        stream = torch.cuda.ExternalStream(c.stream())
        clocks = Clocks(local_rank)
        clocks.start()
        log("warm-up")
        for _ in range(warmup):
            cycle(c, st)
        c.synchronize()
        free_b, total_b = torch.cuda.mem_get_info(local_rank)
        mem_used[precision] = (total_b - free_b) / 1e9
        log("timed cycles (device memory in use %.1f GB)" % mem_used[precision])
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        barrier()
        torch.cuda.synchronize()
        clocks.begin()
        l0 = c.kernel_launches()
        counts = []
        taus = [st.tau]
        e0.record(stream)
        for _ in range(steps):
            counts.append(cycle(c, st))
        e1.record(stream)
        e1.synchronize()
        clocks.end()
        launches = c.kernel_launches() - l0
        clk = clocks.stop()
        torch.cuda.synchronize()
        barrier()
        ms = e0.elapsed_time(e1)
        taus.append(st.tau)
        return c, st, ms, launches, clk, stream, (counts, taus)

    # ---- mixed precision: the headline ----
    c, st, ms, launches, clk, stream, (lc_counts, lc_taus) = timed_run(gev.MIXED, args.steps, args.warmup)
    ms_max = max_over_ranks(ms, world, dev)
    value = job_rate(world, np_, args.steps, ms_max)

    # ---- per-stage breakdown on the final state (CUDA events on the context stream) ----
    log("mixed: %.3f ms/cycle; stage breakdown" % (ms_max / args.steps))
    stages = {}

    def stage(name, fn, reps=5):
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        fn()
        c.synchronize()
        ev0.record(stream)
        for _ in range(reps):
            fn()
        ev1.record(stream)
        ev1.synchronize()
        stages[name] = ev0.elapsed_time(ev1) / reps

    a = st.a
    dx = 1.0 / N
    Hc = gev.hconf(a, fourpiG, ctypes.byref(cosmo))
    deposit = lambda: c.project(gev.PROJ_T00 | gev.PROJ_TIJ | gev.PROJ_T0I_SUMS, a, 1.0, True)
    stage("deposit_T00_Tij_T0i", deposit)
    stage("solve_phi", lambda: c.solve_phi(True, OMEGA_M, 3 * Hc * dx * dx / st.dtau_old, fourpiG * dx * dx / a,
                                           3 * Hc * Hc * dx * dx, 1 / (dx * dx), 3 * Hc / st.dtau_old))
    stage("solve_chi", lambda: c.solve_chi(2 * fourpiG * dx * dx / a, False, Hc, st.dtau, st.dtau_old))
    # the B solve as the cycle runs it, completing the deposit's T0i sums: timed
    # after a deposit each time, less the deposit's own time
    stage("deposit_and_solve_B", lambda: (deposit(), c.solve_B(fourpiG * dx * dx)))
    stages["solve_B"] = stages.pop("deposit_and_solve_B") - stages["deposit_T00_Tij_T0i"]
    stage("kick_drift", lambda: c.kick_drift(0.0, a, a * a * N, 3, 0.0, a, a * a * N, 3))
    stage("lightcone", lambda: c.lightcone(lc, st.tau, st.dtau, st.dtau_old, a, a * Hc, lc_cap, fetch=False))

    # ---- late times: the same initial conditions run on to z = 0 with gev_step
    # (most of a run's cycles are at low redshift, where the particles cluster):
    # the whole run's rate, then cycles and the particle stages at z ~ 0 ----
    late = None
    if not args.no_late:
        log("late times")
        cl = make(gev.MIXED)
        sl = gev.State(a0, tau0, dtau0, 0.0, 0, 0.0, 0.0, 0.0)
        sl_stream = torch.cuda.ExternalStream(cl.stream())
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        cl.synchronize()
        ev0.record(sl_stream)
        n_run = 0
        while 1.0 / sl.a - 1.0 > 0.0:
            cl.step(cosmo, sl)
            n_run += 1
        ev1.record(sl_stream)
        ev1.synchronize()
        run_ms = ev0.elapsed_time(ev1)
        z0_steps = 5
        ev0.record(sl_stream)
        for _ in range(z0_steps):
            cl.step(cosmo, sl)
        ev1.record(sl_stream)
        ev1.synchronize()
        z0_ms = ev0.elapsed_time(ev1) / z0_steps
        al = sl.a
        late_stages = {}
        for name, fn in (("deposit_T00_Tij_T0i", lambda: cl.project(gev.PROJ_T00 | gev.PROJ_TIJ | gev.PROJ_T0I_SUMS, al, 1.0, True)),
                         ("kick_drift", lambda: cl.kick_drift(0.0, al, al * al * N, 3, 0.0, al, al * al * N, 3))):
            fn()
            cl.synchronize()
            ev0.record(sl_stream)
            for _ in range(3):
                fn()
            ev1.record(sl_stream)
            ev1.synchronize()
            late_stages[name] = ev0.elapsed_time(ev1) / 3
        late = {"workload": "the same box from z = %g to z = 0 with gev_step (no lightcone shell), then %d cycles at z ~ 0"
                            % (args.z_in, z0_steps),
                "cycles_to_z0": n_run, "run_ms_per_step": run_ms / n_run,
                "run_value": np_ * n_run / (run_ms * 1e-3) / 1e6, "unit": "Mpart-steps/s",
                "z_end": 1.0 / sl.a - 1.0, "ms_per_step_at_z0": z0_ms, "stage_ms_at_z0": late_stages}
        cl.close()
        del cl

    peak, peak_kind = measured_peaks()
    # per-stage HBM fractions: algorithmic bytes of the stage / its event time / peak
    stage_alg = {"deposit_T00_Tij_T0i": "deposit_T00_Tij_T0i", "solve_phi": "solve_phi",
                 "solve_chi": "solve_chi_tensor" if args.tensor else "solve_chi", "solve_B": "solve_B_sums",
                 "kick_drift": "kick_drift"}
    stage_frac = {k: roofline.stage_bytes(v, N, "mixed") / (stages[k] * 1e-3) / 1e9 / peak for k, v in stage_alg.items()}
    # the dominant kernel: the deposit (its tile launch; the dense-tile launch is
    # empty at z = 100); the other stages are several launches (FFT passes;
    # kick/drift + scan + re-bin), each shorter than the deposit in the ncu
    # launch list (profiles/)
    dom = max(SINGLE_KERNEL_STAGES, key=lambda s: stages[s])
    dom_bytes = roofline.stage_bytes(dom, N, "mixed")
    achieved = dom_bytes / (stages[dom] * 1e-3) / 1e9
    step_alg = roofline.step_bytes(N, "mixed")
    if args.tensor:
        step_alg += roofline.stage_bytes("solve_chi_tensor", N) - roofline.stage_bytes("solve_chi", N)
    step_gbs = step_alg / (ms_max / args.steps * 1e-3) / 1e9

    # ---- validation: P(k) and particle displacements of the mixed run vs an
    # FP64 run from the same ICs (the stage timings above leave the particle
    # state as the timed cycles left it: their kick and drift use dtau = 0) ----
    log("stages %s" % json.dumps(stages))
    pk_mixed = c.power_spectrum(1024)

    def by_id(ctx):
        """final positions in ID order (IDs are the 0..N^3-1 cell indexes of the ICs)"""
        p_, _, i_ = ctx.get_particles()
        out = np.empty_like(p_)
        out[i_] = p_
        return out

    pos0 = np.empty_like(pos_h)
    pos0[ids_h] = pos_h
    pos_mixed = None if args.no_fp64 else by_id(c)
    c.close()
    del c
    fp64 = None
    if not args.no_fp64:
        c64, st64, ms64, _, _, _, _ = timed_run(gev.FP64, args.steps, args.warmup)
        pk64 = c64.power_spectrum(1024)
        pos64 = by_id(c64)

        def disp(p):
            d = p - pos0
            d -= np.round(d)
            return d

        d64 = disp(pos64)
        dmx = disp(pos_mixed)
        rms64 = float(np.sqrt((d64 ** 2).sum(axis=1).mean()))
        rmsmx = float(np.sqrt((dmx ** 2).sum(axis=1).mean()))
        dd = dmx - d64
        dd -= np.round(dd)
        rms_diff = float(np.sqrt((dd ** 2).sum(axis=1).mean()))
        del pos64, d64, dmx, dd
        occ = pk64[4] > 0
        kb = pk64[0][occ]
        kny = math.pi * N
        sel = kb < 0.5 * kny
        rel = np.abs(pk_mixed[1][occ][sel] / pk64[1][occ][sel] - 1)
        fp64 = {"value": np_ * args.steps / (ms64 * 1e-3) / 1e6, "ms_per_step": ms64 / args.steps,
                "mixed_speedup": (np_ * args.steps / (ms_max * 1e-3)) / (np_ * args.steps / (ms64 * 1e-3)),
                "pk_max_rel_err_vs_fp64": float(rel.max()), "pk_k_range_h_per_mpc": [float(kb[sel].min() / box), float(kb[sel].max() / box)],
                "rms_displacement_cells_fp64": rms64 * N, "rms_disp_rel_err_vs_fp64": abs(rmsmx / rms64 - 1.0),
                "per_particle_disp_rel_err_vs_fp64": rms_diff / rms64,
                "cycles_compared": args.warmup + args.steps}
        c64.close()
        del c64

    # ---- e2e: the same cycles through the C ABI with host buffers ----
    e2e = None
    if not args.no_e2e:
        log("e2e")
        c = make(gev.MIXED)
        st = gev.State(a0, tau0, dtau0, 0.0, 0, 0.0, 0.0, 0.0)
        cycle(c, st)                          # warm-up
        pos_o = torch.empty(pos_h.shape, dtype=torch.float64).pin_memory().numpy()
        q_o = torch.empty(q_h.shape, dtype=torch.float64).pin_memory().numpy()
        ids_o = torch.empty(ids_h.shape, dtype=torch.int64).pin_memory().numpy()
        pos_i, q_i, ids_i = pos_h, q_h, ids_h
        pin = torch.empty((lc_cap, 3), dtype=torch.float32).pin_memory().numpy()
        pinv = torch.empty((lc_cap, 3), dtype=torch.float32).pin_memory().numpy()
        pini = torch.empty(lc_cap, dtype=torch.int64).pin_memory().numpy()
        lib = gev._lib
        stream = torch.cuda.ExternalStream(c.stream())
        barrier()
        torch.cuda.synchronize()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        n = ctypes.c_int64()
        lc_bytes = 0
        c.set_particles(pos_i, q_i, ids_i, mass)               # H2D of the first cycle's particle state
        for k in range(args.e2e_steps):
            cycle(c, st)
            lib.gev_lightcone_fetch(c.handle, lc_cap, pin.ctypes.data_as(ctypes.c_void_p), pinv.ctypes.data_as(ctypes.c_void_p),
                                    pini.ctypes.data_as(ctypes.c_void_p), ctypes.byref(n))
            lc_bytes += n.value * 32
            if k + 1 < args.e2e_steps:
                # D2H of the cycle's state and H2D of the next cycle's input (that
                # state, read back) in one call, both directions of the link at once
                c.exchange_particles(pos_o, q_o, ids_o, pos_o, q_o, ids_o, mass)
            else:
                lib.gev_particles_get(c.handle, pos_o.ctypes.data_as(ctypes.c_void_p), q_o.ctypes.data_as(ctypes.c_void_p),
                                      ids_o.ctypes.data_as(ctypes.c_void_p), np_, ctypes.byref(n))
        ev1.record(stream)
        ev1.synchronize()
        ms_e2e = ev0.elapsed_time(ev1)
        ms_e2e = max_over_ranks(ms_e2e, world, dev)
        e2e = {"value": job_rate(world, np_, args.e2e_steps, ms_e2e), "unit": "Mpart-steps/s",
               "h2d_bytes_per_step": int(np_ * 56), "d2h_bytes_per_step": int(np_ * 56 + lc_bytes // max(args.e2e_steps, 1)),
               "steps": args.e2e_steps}
        c.close()

    # ---- differentiable run: adjoint cost and gradient checks, rank 0 only ----
    adj = None
    if rank == 0 and not args.no_adjoint:
        log("adjoint")
        adj = adjoint_block(args, dev)

    # ---- CPU baseline: the oracle on a bounded sample, rank 0 only ----
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        log("cpu baseline")
        cpu = cpu_sample(args)

    if rank == 0:
        line = {
            "metric": "Mpart-steps/s at 512^3 (mixed vs FP64 GPU, P(k) err<1e-4); grad/fwd ratio",
            "value": value, "unit": "Mpart-steps/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 fields/FFT + f64 particle offsets, background and reductions",
            "data": "synthetic: the reference's Zel'dovich ICs at z=%g (generateIC_basic's tabulated-spectrum branch, "
                    "reproduced on the GPU by gev_ics_basic: sitmo stream seed %d, sc1 template tiled N/4, k-sphere, "
                    "corrected displacement, linear EH no-wiggle P(k))" % (args.z_in, args.seed),
            "config": workload_config(N, box, world, args.tensor),
            "gpu_launches": launches,
            "stage_ms": stages,
            "stage_hbm_frac": stage_frac,
            "device_memory_gb": mem_used.get(gev.MIXED),
            "lightcone_counts": lc_counts,
            "lightcone_distance_box": [d_lc - lc_taus[0], d_lc - lc_taus[1]],
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_kind": peak_kind, "traffic": ncu_traffic(dom, N),
                         "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch of the same "
                                           "kernel at 256^3, mixed precision, scaled by the particle count",
                         "algorithmic_bytes_per_launch": dom_bytes,
                         "step_algorithmic_bytes": step_alg, "step_achieved_gbs": step_gbs, "step_frac": step_gbs / peak},
            "clocks": clk,
            "fp64": fp64,
            "e2e": e2e,
            "cpu_baseline": cpu,
            "adjoint": adj,
            "late_time": late,
        }
        print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# CPU: the reference's own cycle (oracle/_ref) on the host cores
# ---------------------------------------------------------------------------
def _load_ics_module():
    """gevb200/ics.py by file path: the reference arm uses its numpy/torch IC
    synthesis without importing the package (which loads the CUDA library)."""
    import importlib.util
    path = os.path.join(ROOT, "gevolution-2.0_b200", "python", "gevb200", "ics.py")
    spec = importlib.util.spec_from_file_location("gev_ics_host", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def reference_cycle_rate(Ns, steps, warmup, seed, z_in=100.0):
    """Time ref_step -- one cycle of main.cu:608-1317 composed from the
    reference's own functors, Fourier solvers and background integrator,
    compiled for the host by oracle/Makefile with the single-rank LATfield2
    stand-in (OpenMP) -- on an Ns^3 box with 5 Mpc/h cells from the initial
    conditions of the reference's own generator (ref_ics_basic:
    generateIC_basic's tabulated-spectrum branch at z_in, sc1 template,
    k-sphere, corrected displacement).  LATfield2's FFT is stood in for by
    pocketfft (scipy.fft, all host threads).  Returns
    (Mpart-steps/s, seconds of the timed cycles, threads) or None when the
    reference build is absent."""
    import numpy as np
    import scipy.fft
    import torch

    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from _libs import ptr, ref

    r = ref()
    if r is None:
        return None

    class Sim(ctypes.Structure):   # orc_sim
        _fields_ = [("N", ctypes.c_int), ("boxsize", ctypes.c_double), ("fourpiG", ctypes.c_double),
                    ("mass", ctypes.c_double), ("Om", ctypes.c_double), ("OL", ctypes.c_double),
                    ("Orad", ctypes.c_double), ("z_relax", ctypes.c_double), ("Cf", ctypes.c_double),
                    ("steplimit", ctypes.c_double), ("with_B", ctypes.c_int)]

    class State(ctypes.Structure):   # orc_state
        _fields_ = [("a", ctypes.c_double), ("tau", ctypes.c_double), ("dtau", ctypes.c_double),
                    ("dtau_old", ctypes.c_double), ("cycle", ctypes.c_int), ("T00hom", ctypes.c_double),
                    ("phi_hom", ctypes.c_double), ("maxvel", ctypes.c_double)]

    fft_t = ctypes.CFUNCTYPE(None, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p)
    dptr = ctypes.POINTER(ctypes.c_double)

    def r2c(N, pin, pout):
        f = np.ctypeslib.as_array(ctypes.cast(pin, dptr), shape=(N, N, N))
        o = np.ctypeslib.as_array(ctypes.cast(pout, dptr), shape=(N, N, N + 2)).view(np.complex128)
        o[...] = scipy.fft.rfftn(f, workers=-1)

    def c2r(N, pin, pout):
        F = np.ctypeslib.as_array(ctypes.cast(pin, dptr), shape=(N, N, N + 2)).view(np.complex128)
        o = np.ctypeslib.as_array(ctypes.cast(pout, dptr), shape=(N, N, N))
        o[...] = scipy.fft.irfftn(F, s=(N, N, N), norm="forward", workers=-1)

    cb = (fft_t(r2c), fft_t(c2r))
    r.lib.ref_set_fft.argtypes = [fft_t, fft_t]
    r.lib.ref_set_fft.restype = None
    r.lib.ref_step.argtypes = [ctypes.POINTER(Sim), ctypes.POINTER(State), ctypes.c_int64] + [ctypes.c_void_p] * 5
    r.lib.ref_step.restype = None
    r.lib.ref_set_fft(*cb)

    box = 5.0 * Ns
    ics = _load_ics_module()
    a0 = 1.0 / (1.0 + z_in)
    fourpiG = 1.5 * box * box / C_LIGHT ** 2
    mass = OMEGA_M / Ns ** 3
    kt = np.logspace(-5, 3, 4096)
    pt = ics.linear_pk(kt, a0, H_LITTLE, OMEGA_M)
    tmpl = ics.sc1_template()
    n3 = Ns ** 3
    pos, q, ids = np.zeros((n3, 3)), np.zeros((n3, 3)), np.zeros(n3, dtype=np.int64)
    phi, chi, Bi, mv = np.zeros(n3), np.zeros(n3), np.zeros(3 * n3), np.zeros(1)
    if r.ics_basic(Ns, box, a0, fourpiG, OMEGA_M, OMEGA_L, 0.0, ptr(kt), ptr(pt), len(kt), seed, 1, 1, 1, Ns // 4,
                   ptr(tmpl), len(tmpl), ptr(pos), ptr(q), ptr(ids), ptr(phi), ptr(chi), ptr(Bi), ptr(mv)) != 0:
        return None
    del torch
    sim = Sim(Ns, box, fourpiG, mass, OMEGA_M, OMEGA_L, 0.0, z_in, 48.0, 0.04, 1)
    H = math.sqrt((2 * fourpiG / 3) * (OMEGA_M / a0 + OMEGA_L * a0 * a0))
    st = State(a0, 0.0, min(48.0 / Ns, 0.04 / H), 0.0, 0, 0, 0, 0)

    def cycle():
        r.lib.ref_step(ctypes.byref(sim), ctypes.byref(st), len(pos), ptr(pos), ptr(q), ptr(phi), ptr(chi), ptr(Bi))

    for _ in range(max(1, warmup)):
        cycle()
    t0 = time.perf_counter()
    for _ in range(steps):
        cycle()
    dt = time.perf_counter() - t0
    r.lib.ref_set_fft(fft_t(0), fft_t(0))
    threads = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    return Ns ** 3 * steps / dt / 1e6, dt, threads


def reference_sample_config(Ns, N):
    box = 5.0 * Ns
    return {"workload": "PM cycle of the reference's own functions on the host cores (FP64): box %g Mpc/h, grid %d^3, "
                        "%d^3 particles, GR, elliptic B; a bounded sample of the %d^3 workload with the same physics and "
                        "5 Mpc/h cells" % (box, Ns, Ns, N),
            "N": Ns, "particles": Ns ** 3, "boxsize_mpc_h": box, "sample_of": "grid %d^3, %d^3 particles" % (N, N),
            "parallelism": "host cores (OpenMP)"}


def adjoint_block(args, dev):
    """Differentiable Newtonian run (box 640 Mpc/h at 128^3, 32 steps from z = 50
    to 0, checkpoints every 8 steps): forward and adjoint device times, their
    ratio, and the gradient checks (central differences on random white-noise
    modes, FP64 adjoint against the mixed-precision one)."""
    import numpy as np
    import torch

    import gevb200 as gev
    from gevb200 import pm as gpm

    N, nsteps = args.adj_N, args.adj_steps
    box = 5.0 * N
    fourpiG = 1.5 * box * box / C_LIGHT ** 2
    a_in = 1.0 / 51.0
    coef, _ = gpm.schedule(N, fourpiG, OMEGA_M, OMEGA_L, a_in, 1.0, nsteps)
    g = torch.Generator(device="cpu").manual_seed(args.seed + 77)
    noise = torch.randn(N ** 3, generator=g, dtype=torch.float64).to(dev)
    target = 0.5 * torch.randn(N ** 3, generator=g, dtype=torch.float64).to(dev)
    mass = OMEGA_M / N ** 3

    def run(precision, w, reps=3):
        """min device times (ms) of forward and adjoint over reps passes on one
        PM object; a first, untimed pass allocates the checkpoints"""
        p = gpm.PM(N, N ** 3, mass, precision, checkpoint_every=8)
        x0, q0 = gpm.zeldovich_map(w, N, box, a_in, fourpiG, OMEGA_M, OMEGA_L, H_LITTLE)
        x0, q0 = x0.detach().contiguous(), q0.detach().contiguous()
        delta = torch.empty(N ** 3, dtype=torch.float64, device=dev)
        gx = torch.empty_like(x0)
        gq = torch.empty_like(q0)
        st = torch.cuda.ExternalStream(p.stream())
        fwd, adj = [], []
        for r in range(reps + 1):
            e = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
            torch.cuda.synchronize()
            e[0].record(st)
            p.forward(coef, x0, q0, delta)
            e[1].record(st)
            torch.cuda.synchronize()
            gd = (2.0 * (delta - target)).contiguous()
            torch.cuda.synchronize()
            e[2].record(st)
            p.adjoint(gd, gx, gq)
            e[3].record(st)
            torch.cuda.synchronize()
            if r > 0:
                fwd.append(e[0].elapsed_time(e[1]))
                adj.append(e[2].elapsed_time(e[3]))
        p.close()
        return min(fwd), min(adj)

    def grad_modes(precision, w):
        wv = w.clone().requires_grad_(True)
        x0, q0 = gpm.zeldovich_map(wv, N, box, a_in, fourpiG, OMEGA_M, OMEGA_L, H_LITTLE)
        p = gpm.PM(N, N ** 3, mass, precision, checkpoint_every=8)
        delta = gpm.run_function().apply(x0, q0, p, coef)
        ((delta - target) ** 2).sum().backward()
        return wv.grad.detach()

    def loss_of(w):
        p = gpm.PM(N, N ** 3, mass, gev.FP64, checkpoint_every=8)
        x0, q0 = gpm.zeldovich_map(w, N, box, a_in, fourpiG, OMEGA_M, OMEGA_L, H_LITTLE)
        delta = torch.empty(N ** 3, dtype=torch.float64, device=dev)
        p.forward(coef, x0.contiguous(), q0.contiguous(), delta)
        return float(((delta - target) ** 2).sum())

    out = {"config": {"workload": "differentiable Newtonian PM run (main.cu gr_flag = 0): box %g Mpc/h, grid %d^3, "
                                  "%d^3 particles, %d steps z = 50 -> 0, loss sum (delta_CIC - target)^2, checkpoints "
                                  "every 8 steps" % (box, N, N, nsteps), "N": N, "steps": nsteps}}
    for name, prec in (("mixed", gev.MIXED), ("fp64", gev.FP64)):
        fwd, adjm = run(prec, noise)
        out[name] = {"fwd_ms": fwd, "adjoint_ms": adjm, "grad_fwd_ratio": adjm / fwd,
                     "fwd_mpart_steps_s": N ** 3 * nsteps / (fwd * 1e-3) / 1e6}
    g64 = grad_modes(gev.FP64, noise)
    g32 = grad_modes(gev.MIXED, noise)
    rng = np.random.default_rng(args.seed)
    modes = rng.choice(N ** 3, size=args.adj_modes, replace=False)
    eps = 1e-4
    fd = []
    for m in modes:
        d = torch.zeros_like(noise)
        d[int(m)] = eps
        fd.append((loss_of(noise + d) - loss_of(noise - d)) / (2 * eps))
    fd = np.array(fd)
    ad = g64.cpu().numpy()[modes]
    out["checks"] = {"fd_modes": int(args.adj_modes), "fd_eps": eps,
                     "fd_vs_fp64_adjoint_rel_err": float(np.linalg.norm(fd - ad) / np.linalg.norm(ad)),
                     "mixed_vs_fp64_adjoint_rel_err": float(torch.linalg.norm(g32 - g64) / torch.linalg.norm(g64))}
    out["grad_fwd_ratio"] = out["mixed"]["grad_fwd_ratio"]
    return out


def cpu_sample(args):
    cores = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(cores))
    res = reference_cycle_rate(args.cpu_sample_N, args.cpu_sample_steps, 1, args.seed)
    if res is None:
        return None
    rate, dt, threads = res
    return {"value": rate, "unit": "Mpart-steps/s", "cores": threads, "kind": "reference",
            "sample": "%d cycles of the reference's own cycle functions (ref_step, oracle/_ref) on a %d^3 box with %d^3 "
                      "particles from the reference's IC generator at z = 100, %.1f s, FFT by pocketfft" % (args.cpu_sample_steps, args.cpu_sample_N,
                                                                                     args.cpu_sample_N, dt)}


def run_reference(args, rank):
    if rank != 0:
        return
    cores = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(cores))
    Ns = args.cpu_sample_N
    res = reference_cycle_rate(Ns, args.steps, args.warmup, args.seed)
    if res is None:
        print(json.dumps({"impl": "reference", "unavailable": "the reference's cycle functions were not built here "
                                                              "(oracle/_ref/libgevref.so is missing)"}), flush=True)
        return
    rate, dt, threads = res
    line = {"impl": "reference", "metric": "Mpart-steps/s at 512^3 (mixed vs FP64 GPU, P(k) err<1e-4); grad/fwd ratio",
            "value": rate, "unit": "Mpart-steps/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": max(1, args.warmup), "ms_per_step": dt / args.steps * 1e3, "ms_per_step_grid": "%d^3" % Ns,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic: the reference's Zel'dovich ICs at z=100 (ref_ics_basic: generateIC_basic's tabulated-"
                    "spectrum branch, EH no-wiggle P(k), sc1 template), on the host, seed %d" % args.seed,
            "config": reference_sample_config(Ns, args.N),
            "cpu_baseline": {"value": rate, "unit": "Mpart-steps/s", "cores": threads, "kind": "reference",
                             "sample": "the reference's own cycle functions (ref_step: gevolution.hpp projections, "
                                       "prepareFTsource, Fourier solvers, update_q/update_pos, background.hpp) on a %d^3 "
                                       "box, %d cycles after %d warm-up, %.1f s; FFT by pocketfft" % (Ns, args.steps,
                                                                                                     max(1, args.warmup), dt)},
            "e2e": {"value": rate, "unit": "Mpart-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return
    if world > 1:
        import datetime

        import torch
        torch.cuda.set_device(local_rank)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                             device_id=torch.device("cuda", local_rank))
    try:
        run_gpu(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch
            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
