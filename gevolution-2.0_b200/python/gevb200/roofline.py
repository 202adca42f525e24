"""Algorithmic bytes of the PM cycle (the minimum HBM traffic: one read or write
of each array per data-dependent stage; stage boundaries are forced by the
FFTs; particle re-bucketing is overhead and not counted).

Per particle (Np = N^3):  mixed  cell u32 4 B + FP64 offsets 24 B + q FP32 12 B = 40 B
                          FP64   cell u32 4 B + FP64 offsets 24 B + q FP64 24 B = 52 B
Per cell, F = 4 B (mixed) or 8 B (FP64) per real component; the half spectrum
counts F per component per cell.
"""

PARTICLE_BYTES = {"mixed": 40, "fp64": 52}
FIELD_BYTES = {"mixed": 4, "fp64": 8}


def stage_bytes(stage, N, precision="mixed", np_=None):
    """Algorithmic bytes moved by one launch of a stage of the cycle."""
    n3 = N ** 3
    np_ = n3 if np_ is None else np_
    P = PARTICLE_BYTES[precision]
    F = FIELD_BYTES[precision]
    table = {
        # read particles, read phi, write T00 + 6 Tij
        "deposit_T00_Tij": np_ * P + n3 * F * (1 + 7),
        # read particles, read phi, write 3 T0i
        "deposit_T0i": np_ * P + n3 * F * (1 + 3),
        # one deposit for the cycle (GEV_PROJ_T0I_SUMS): read particles, read phi,
        # write T00 + 6 Tij + 3 potential-free T0i sums
        "deposit_T00_Tij_T0i": np_ * P + n3 * F * (1 + 7 + 3),
        # read T00, phi, chi; write spectrum; read spectrum; write phi
        "solve_phi": n3 * F * (3 + 1 + 1 + 1),
        # read 6 Tij + phi, write 6 spectra; read 6 spectra (as the fused solve needs them), write chi
        "solve_chi": n3 * F * (7 + 6 + 6 + 1),
        # the same with the tensor state (evolveFTtensor): read and write h_ij and h_ij' (12 spectra each)
        "solve_chi_tensor": n3 * F * (7 + 6 + 6 + 1 + 12 + 12),
        # read 3 T0i, write 3 spectra; read 3, write 3 B
        "solve_B": n3 * F * (3 + 3 + 3 + 3),
        # the same from the T0i sums, which the x pass completes with phi (one more read)
        "solve_B_sums": n3 * F * (3 + 1 + 3 + 3 + 3),
        # read + write particles, read phi, chi, 3 B
        "kick_drift": 2 * np_ * P + n3 * F * 5,
    }
    return table[stage]


# the cycle's stages: in mixed precision one deposit completes T0i through the
# B solve (GEV_PROJ_T0I_SUMS); FP64 keeps the separate T0i deposit
STAGES = {"mixed": ("deposit_T00_Tij_T0i", "solve_phi", "solve_chi", "solve_B_sums", "kick_drift"),
          "fp64": ("deposit_T00_Tij", "solve_phi", "solve_chi", "deposit_T0i", "solve_B", "kick_drift")}


def step_bytes(N, precision="mixed", np_=None):
    return sum(stage_bytes(s, N, precision, np_) for s in STAGES[precision])
