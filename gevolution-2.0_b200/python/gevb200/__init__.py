"""gevb200 -- Python binding of the C ABI in include/gev.h.

The product is the CUDA library libgevb200.so (sm_100a kernels + C ABI); this
module only marshals numpy arrays through ctypes.  It has no CPU fallback: if
the library is missing, importing the module raises.

The method names mirror the reference's interface for the per-step cycle
(gevolution.hpp / main.cu of gevolution-2.0):

    Context.project(...)        projection_T00/Tij/T0i_project + *_comm
    Context.solve_phi(...)      prepareFTsource + FFT + solveModifiedPoissonFT + FFT^-1
    Context.solve_chi(...)      prepareFTsource(Tij) + FFT + projectFTscalar (+ tensor) + FFT^-1
    Context.solve_B(...)        FFT + projectFTvector + FFT^-1
    Context.kick / drift        perfParticles::updateVel(update_q) / moveParticles(update_pos)
    Context.power_spectrum      scalarProjectionCIC_project + FFT + extractPowerSpectrum
    Context.lightcone           writeLightcones, particle branch
    Context.step                one cycle of main.cu's main loop
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.normpath(os.path.join(_HERE, "..", "..", "libgevb200.so"))

if not os.path.exists(LIB_PATH):
    raise ImportError("gevb200: %s is missing; build it with `make -C gevolution-2.0_b200`" % LIB_PATH)

_lib = ctypes.CDLL(LIB_PATH)

GEV_OK = 0
GEV_ERR_ARG, GEV_ERR_CUDA, GEV_ERR_STATE, GEV_ERR_DEVICE, GEV_ERR_NOMEM, GEV_ERR_CAPACITY = 1, 2, 3, 4, 5, 6
GEV_ERR_SIZE = 7
FP64, MIXED = 0, 1
VECTOR_PARABOLIC, VECTOR_ELLIPTIC = 0, 1
FIELD_PHI, FIELD_CHI, FIELD_SOURCE, FIELD_SIJ, FIELD_BI, FIELD_HIJ_FT, FIELD_HIJP_FT, FIELD_BI_FT = range(8)
PROJ_T00, PROJ_TIJ, PROJ_T0I, PROJ_CIC, PROJ_T0I_SUMS = 1, 2, 4, 8, 16

_d, _i, _u, _l, _p = ctypes.c_double, ctypes.c_int32, ctypes.c_uint32, ctypes.c_int64, ctypes.c_void_p


class Config(ctypes.Structure):
    _fields_ = [("N", _i), ("precision", _i), ("capacity", _l), ("boxsize", _d),
                ("vector_method", _i), ("tensor", _i), ("device", _i), ("reserved", _i)]


class Cosmo(ctypes.Structure):
    _fields_ = [("Omega_m", _d), ("Omega_Lambda", _d), ("Omega_rad", _d), ("fourpiG", _d),
                ("Cf", _d), ("steplimit", _d), ("z_relax", _d), ("boxsize", _d)]


class State(ctypes.Structure):
    _fields_ = [("a", _d), ("tau", _d), ("dtau", _d), ("dtau_old", _d), ("cycle", _l),
                ("T00hom", _d), ("phi_hom", _d), ("maxvel", _d)]


class IcsParams(ctypes.Structure):
    _fields_ = [("boxsize", _d), ("a", _d), ("fourpiG", _d), ("Omega_m", _d), ("Omega_Lambda", _d),
                ("Omega_rad", _d), ("seed", ctypes.c_uint64), ("pk_k", _p), ("pk_p", _p), ("n_pk", _i),
                ("ksphere", _i), ("gr", _i), ("reserved", _i), ("noise", _p), ("noise_out", _p)]


class IcsBasicParams(ctypes.Structure):
    _fields_ = [("boxsize", _d), ("a", _d), ("fourpiG", _d), ("Omega_m", _d), ("Omega_Lambda", _d),
                ("Omega_rad", _d), ("pk_k", _p), ("pk_p", _p), ("n_pk", _i), ("seed", ctypes.c_uint32),
                ("ksphere", _i), ("correct_displacement", _i), ("gr", _i), ("numtile", _i), ("template_pos", _p),
                ("template_n", _l)]


class LightconeArgs(ctypes.Structure):
    _fields_ = [("vertex", _d * 3), ("direction", _d * 3), ("opening", _d), ("distance", _d * 2),
                ("d", _d), ("tracer_factor", _i), ("shell", _i)]


def _sig(name, args, res=ctypes.c_int):
    fn = getattr(_lib, name)
    fn.argtypes = args
    fn.restype = res
    return fn


_create = _sig("gev_ctx_create", [ctypes.POINTER(Config), ctypes.POINTER(_p)])
_destroy = _sig("gev_ctx_destroy", [_p])
_last_error = _sig("gev_last_error", [_p], ctypes.c_char_p)
_version = _sig("gev_version", [], ctypes.c_char_p)
_pset = _sig("gev_particles_set", [_p, _p, _p, _p, _l, _d])
_pget = _sig("gev_particles_get", [_p, _p, _p, _p, _l, ctypes.POINTER(_l)])
_pxch = _sig("gev_particles_exchange", [_p, _p, _p, _p, _l, ctypes.POINTER(_l), _p, _p, _p, _l, _d])
_pcount = _sig("gev_particles_count", [_p, ctypes.POINTER(_l)])
_fget = _sig("gev_field_get", [_p, _i, _p])
_fset = _sig("gev_field_set", [_p, _i, _p])
_fcomp = _sig("gev_field_components", [_i])
_project = _sig("gev_project", [_p, _u, _d, _d, _i, _i])
_solve_phi = _sig("gev_solve_phi", [_p, _i, _d, _d, _d, _d, _d, _d, ctypes.POINTER(_d), ctypes.POINTER(_d)])
_solve_chi = _sig("gev_solve_chi", [_p, _d, _i, _d, _d, _d, _d])
_prep_t00 = _sig("gev_prepare_T00", [_p, _d, _d, _d, _d, ctypes.POINTER(_d)])
_prep_tij = _sig("gev_prepare_Tij", [_p, _d])
_solve_B = _sig("gev_solve_B", [_p, _d, _d])
_kick = _sig("gev_kick", [_p, _d, _d, _d, _i, ctypes.POINTER(_d)])
_drift = _sig("gev_drift", [_p, _d, _d, _d, _i])
_kick_drift = _sig("gev_kick_drift", [_p, _d, _d, _d, _i, _d, _d, _d, _i, ctypes.POINTER(_d)])
_pk = _sig("gev_power_spectrum", [_p, _i, _d, _p, _p, _p, _p, _p])
_lc = _sig("gev_lightcone", [_p, ctypes.POINTER(LightconeArgs), _d, _d, _d, _d, _d, _l, _p, _p, _p, ctypes.POINTER(_l)])
_lcf = _sig("gev_lightcone_fetch", [_p, _l, _p, _p, _p, ctypes.POINTER(_l)])
_step = _sig("gev_step", [_p, ctypes.POINTER(Cosmo), ctypes.POINTER(State)])
_step_lc = _sig("gev_step_lightcone", [_p, ctypes.POINTER(Cosmo), ctypes.POINTER(State), ctypes.POINTER(LightconeArgs),
                                      _l, ctypes.POINTER(_l)])
_sync = _sig("gev_synchronize", [_p])
_stream = _sig("gev_stream", [_p], _p)
_launches = _sig("gev_kernel_launches", [_p], _l)
hconf = _sig("gev_hconf", [_d, _d, ctypes.POINTER(Cosmo)], _d)
particle_horizon = _sig("gev_particle_horizon", [_d, _d, ctypes.POINTER(Cosmo)], _d)
_rk4 = _sig("gev_rungekutta4bg", [ctypes.POINTER(_d), _d, ctypes.POINTER(Cosmo), _d], None)


def rungekutta4bg(a, fourpiG, cosmo, dtau):
    x = _d(a)
    _rk4(ctypes.byref(x), fourpiG, ctypes.byref(cosmo), dtau)
    return x.value


def version():
    return _version().decode()


_poisson_noalloc = _sig("gev_poisson_noalloc", [_i, _i, _p, _p, _d, _d, _p])
_ics = _sig("gev_ics_zeldovich", [_p, ctypes.POINTER(IcsParams)])
_ics_basic = _sig("gev_ics_basic", [_p, ctypes.POINTER(IcsBasicParams)])
_sitmo = _sig("gev_sitmo_words", [ctypes.c_uint32, ctypes.c_uint64, _l, _p])


def sitmo_words(seed, start, n):
    """Words [start, start + n) of the reference IC generator's random stream
    (sitmo::prng_engine of `seed`), as uint32."""
    out = np.zeros(max(int(n), 1), dtype=np.uint32)
    rc = _sitmo(int(seed), int(start), int(n), out.ctypes.data_as(_p))
    if rc != GEV_OK:
        raise GevError(rc, "gev_sitmo_words failed")
    return out[:int(n)]
_ckw = _sig("gev_checkpoint_write", [_p, ctypes.c_char_p, ctypes.POINTER(State)])
_ckr = _sig("gev_checkpoint_read", [_p, ctypes.c_char_p, ctypes.POINTER(State)])


def poisson_noalloc(N, precision, source_ptr, phi_ptr, poisson_coeff, modif, stream=None):
    """gev_poisson_noalloc on device pointers (ints); returns the status code.
    Queues the work on `stream` (a raw cudaStream_t handle, None = default
    stream) without synchronising."""
    return _poisson_noalloc(int(N), int(precision), _p(source_ptr), _p(phi_ptr), float(poisson_coeff),
                            float(modif), _p(stream) if stream else None)


class GevError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("gev error %d: %s" % (code, msg))
        self.code = code


def _ptr(a):
    if a is None:
        return None
    if not a.flags["C_CONTIGUOUS"]:
        raise ValueError("arrays must be C-contiguous")
    return a.ctypes.data_as(_p)


class Context:
    """One simulation box on one GPU (gev_ctx)."""

    def __init__(self, N, precision=MIXED, capacity=None, boxsize=1.0, vector_method=VECTOR_ELLIPTIC,
                 tensor=False, device=0):
        self.N = int(N)
        cfg = Config(self.N, int(precision), int(capacity if capacity is not None else self.N ** 3), float(boxsize),
                     int(vector_method), int(bool(tensor)), int(device), 0)
        h = _p()
        rc = _create(ctypes.byref(cfg), ctypes.byref(h))
        if rc != GEV_OK:
            raise GevError(rc, _last_error(None).decode())
        self._h = h
        self.cfg = cfg
        self._destroy = _destroy   # held by the object: module globals may be gone when it is collected at exit

    def close(self):
        if getattr(self, "_h", None):
            self._destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _ck(self, rc):
        if rc != GEV_OK:
            raise GevError(rc, _last_error(self._h).decode())

    @property
    def handle(self):
        return self._h

    def stream(self):
        return _stream(self._h)

    def synchronize(self):
        self._ck(_sync(self._h))

    def kernel_launches(self):
        """Number of kernels this context has launched (the library's own kernels)."""
        return int(_launches(self._h))

    # ---- particles ----
    def set_particles(self, pos, q, ids=None, mass=1.0):
        pos = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1, 3)
        q = np.ascontiguousarray(q, dtype=np.float64).reshape(-1, 3)
        ids = None if ids is None else np.ascontiguousarray(ids, dtype=np.int64)
        self._ck(_pset(self._h, _ptr(pos), _ptr(q), _ptr(ids), pos.shape[0], float(mass)))

    def get_particles(self):
        n = _l()
        self._ck(_pcount(self._h, ctypes.byref(n)))
        pos = np.empty((n.value, 3)); q = np.empty((n.value, 3)); ids = np.empty(n.value, dtype=np.int64)
        self._ck(_pget(self._h, _ptr(pos), _ptr(q), _ptr(ids), n.value, ctypes.byref(n)))
        return pos, q, ids

    def exchange_particles(self, pos_out, q_out, ids_out, pos_in, q_in, ids_in, mass=1.0):
        """Copy the current particles into the output arrays and load the input
        arrays in one call, both directions of the host link at once
        (gev_particles_exchange).  The output arrays are written in place:
        float64 (n, 3), float64 (n, 3) and int64 (n,), C-contiguous; the
        input arrays may be the same arrays.  Returns the number of particles
        written."""
        for arr, dt in ((pos_out, np.float64), (q_out, np.float64), (ids_out, np.int64)):
            if not (isinstance(arr, np.ndarray) and arr.dtype == dt and arr.flags.c_contiguous):
                raise TypeError("output arrays must be C-contiguous numpy arrays of float64/float64/int64")
        pos_in = np.ascontiguousarray(pos_in, dtype=np.float64).reshape(-1, 3)
        q_in = np.ascontiguousarray(q_in, dtype=np.float64).reshape(-1, 3)
        ids_in = np.ascontiguousarray(ids_in, dtype=np.int64)
        n = _l()
        self._ck(_pxch(self._h, _ptr(pos_out), _ptr(q_out), _ptr(ids_out), ids_out.shape[0], ctypes.byref(n),
                       _ptr(pos_in), _ptr(q_in), _ptr(ids_in), pos_in.shape[0], float(mass)))
        return n.value

    # ---- fields ----
    def get_field(self, field):
        nc = _fcomp(field)
        N = self.N
        if field in (FIELD_HIJ_FT, FIELD_HIJP_FT, FIELD_BI_FT):
            out = np.empty((nc, N, N, N // 2 + 1), dtype=np.complex128)
        else:
            out = np.empty((nc, N, N, N), dtype=np.float64)
        self._ck(_fget(self._h, field, _ptr(out)))
        return out[0] if nc == 1 else out

    def set_field(self, field, values):
        nc = _fcomp(field)
        N = self.N
        dt = np.complex128 if field in (FIELD_HIJ_FT, FIELD_HIJP_FT, FIELD_BI_FT) else np.float64
        v = np.ascontiguousarray(values, dtype=dt)
        if v.size != nc * (N * N * (N // 2 + 1) if dt == np.complex128 else N ** 3):
            raise ValueError("field has the wrong size")
        self._ck(_fset(self._h, field, _ptr(v)))

    # ---- the cycle ----
    def project(self, which, a=1.0, coeff=1.0, use_phi=True, accumulate=False):
        self._ck(_project(self._h, int(which), float(a), float(coeff), int(bool(use_phi)), int(bool(accumulate))))

    def solve_phi(self, prepare, bgmodel, coeff, coeff2, coeff3, poisson_coeff, modif):
        s, h = _d(), _d()
        self._ck(_solve_phi(self._h, int(bool(prepare)), bgmodel, coeff, coeff2, coeff3, poisson_coeff, modif,
                            ctypes.byref(s), ctypes.byref(h)))
        return s.value, h.value

    def prepare_T00(self, bgmodel, coeff, coeff2, coeff3):
        """prepareFTsource (T00 form) in place on the source field; returns the sum of T00."""
        s = _d()
        self._ck(_prep_t00(self._h, bgmodel, coeff, coeff2, coeff3, ctypes.byref(s)))
        return s.value

    def prepare_Tij(self, coeff):
        """prepareFTsource (Tij form) in place on the Sij field."""
        self._ck(_prep_tij(self._h, coeff))

    def solve_chi(self, coeff, cycle0=False, hubble=0.0, dtau=0.0, dtau_old=0.0, a2dtau=0.0):
        self._ck(_solve_chi(self._h, coeff, int(bool(cycle0)), hubble, dtau, dtau_old, a2dtau))

    def solve_B(self, coeff, modif=0.0):
        self._ck(_solve_B(self._h, coeff, modif))

    def kick(self, dtau, a, bcoeff, nfield):
        v = _d()
        self._ck(_kick(self._h, dtau, a, bcoeff, int(nfield), ctypes.byref(v)))
        return v.value

    def drift(self, dtau, a, bcoeff, nfield):
        self._ck(_drift(self._h, dtau, a, bcoeff, int(nfield)))

    def kick_drift(self, dtau_k, a_k, b_k, nf_k, dtau_d, a_d, b_d, nf_d):
        v = _d()
        self._ck(_kick_drift(self._h, dtau_k, a_k, b_k, int(nf_k), dtau_d, a_d, b_d, int(nf_d), ctypes.byref(v)))
        return v.value

    def power_spectrum(self, numbins, kmax=0.0):
        kb, pw, ks, ps = (np.zeros(numbins) for _ in range(4))
        oc = np.zeros(numbins, dtype=np.int32)
        self._ck(_pk(self._h, int(numbins), float(kmax), _ptr(kb), _ptr(pw), _ptr(ks), _ptr(ps), _ptr(oc)))
        return kb, pw, ks, ps, oc

    def lightcone(self, args, tau, dtau, dtau_old, a, dadtau, capacity, fetch=True):
        """Selects the shell's crossing particles; returns (pos, vel, ids) host
        arrays, or the count alone when fetch is False (data stays on the device)."""
        n = _l()
        if not fetch:
            self._ck(_lc(self._h, ctypes.byref(args), tau, dtau, dtau_old, a, dadtau, int(capacity), None, None, None,
                         ctypes.byref(n)))
            return n.value
        pos = np.empty((max(capacity, 1), 3), dtype=np.float32)
        vel = np.empty((max(capacity, 1), 3), dtype=np.float32)
        ids = np.empty(max(capacity, 1), dtype=np.int64)
        self._ck(_lc(self._h, ctypes.byref(args), tau, dtau, dtau_old, a, dadtau, int(capacity), _ptr(pos), _ptr(vel),
                     _ptr(ids), ctypes.byref(n)))
        return pos[:n.value], vel[:n.value], ids[:n.value]

    def lightcone_fetch(self, capacity):
        pos = np.empty((max(capacity, 1), 3), dtype=np.float32)
        vel = np.empty((max(capacity, 1), 3), dtype=np.float32)
        ids = np.empty(max(capacity, 1), dtype=np.int64)
        n = _l()
        self._ck(_lcf(self._h, int(capacity), _ptr(pos), _ptr(vel), _ptr(ids), ctypes.byref(n)))
        return pos[:n.value], vel[:n.value], ids[:n.value]

    def step(self, cosmo, state):
        self._ck(_step(self._h, ctypes.byref(cosmo), ctypes.byref(state)))
        return state

    def step_lightcone(self, cosmo, state, args, capacity):
        """gev_step with the lightcone shell between the solves and the kick;
        returns the number of selected particles (left on the device)."""
        n = _l()
        self._ck(_step_lc(self._h, ctypes.byref(cosmo), ctypes.byref(state), ctypes.byref(args), int(capacity),
                          ctypes.byref(n)))
        return n.value

    def ics_zeldovich(self, boxsize, a, fourpiG, omega_m, omega_l, pk_k, pk_p, seed=0, omega_rad=0.0,
                      ksphere=False, gr=True, noise=None, return_noise=False):
        """Zel'dovich initial conditions (gev_ics_zeldovich): replaces the
        particles and phi.  pk_k [h/Mpc], pk_p [(Mpc/h)^3] tabulate P(k) at a."""
        k = np.ascontiguousarray(pk_k, dtype=np.float64)
        pk = np.ascontiguousarray(pk_p, dtype=np.float64)
        w = None if noise is None else np.ascontiguousarray(noise, dtype=np.float64).ravel()
        out = np.empty(self.N ** 3) if return_noise else None
        prm = IcsParams(float(boxsize), float(a), float(fourpiG), float(omega_m), float(omega_l), float(omega_rad),
                        int(seed), k.ctypes.data_as(_p), pk.ctypes.data_as(_p), len(k), int(bool(ksphere)),
                        int(bool(gr)), 0, _ptr(w), _ptr(out))
        self._ck(_ics(self._h, ctypes.byref(prm)))
        return out

    def ics_basic(self, boxsize, a, fourpiG, omega_m, omega_l, pk_k, pk_p, template_pos, numtile, seed=0,
                  omega_rad=0.0, ksphere=False, correct_displacement=True, gr=True):
        """The reference's own initial conditions (gev_ics_basic): the tabulated
        spectrum pk_k [h/Mpc], pk_p [(Mpc/h)^3] as read from an mPk file, the
        particle template (n x 3 positions in [0, 1]) tiled numtile times per
        axis.  Replaces the particles, phi, chi and B_i."""
        k = np.ascontiguousarray(pk_k, dtype=np.float64)
        pk = np.ascontiguousarray(pk_p, dtype=np.float64)
        t = np.ascontiguousarray(template_pos, dtype=np.float32).reshape(-1, 3)
        prm = IcsBasicParams(float(boxsize), float(a), float(fourpiG), float(omega_m), float(omega_l), float(omega_rad),
                             k.ctypes.data_as(_p), pk.ctypes.data_as(_p), len(k), int(seed) & 0xFFFFFFFF,
                             int(bool(ksphere)), int(bool(correct_displacement)), int(bool(gr)), int(numtile),
                             t.ctypes.data_as(_p), len(t))
        self._ck(_ics_basic(self._h, ctypes.byref(prm)))

    def checkpoint_write(self, path, state):
        self._ck(_ckw(self._h, str(path).encode(), ctypes.byref(state)))

    def checkpoint_read(self, path):
        st = State()
        self._ck(_ckr(self._h, str(path).encode(), ctypes.byref(st)))
        return st
