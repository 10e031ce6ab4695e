"""ctypes binding of ``libfirestep.so`` (the C ABI in ``include/firestep.h``).

The library is built in-tree by ``firewebapp_b200/csrc/Makefile``.  There is
no fallback: if the shared object is missing or a symbol is absent, importing
anything that needs it raises ``RuntimeError``.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

_HERE = Path(__file__).resolve().parent
LIB_PATH = Path(os.environ.get("FIRESTEP_LIB", _HERE / "libfirestep.so"))

P = C.c_void_p
D = C.c_double
I = C.c_int
I64 = C.c_int64
PP = C.POINTER(C.c_void_p)


class FsGrid(C.Structure):
    _fields_ = [("nx", I), ("ny", I), ("nz", I), ("dx", D), ("dy", D),
                ("dz", P), ("d_above", P), ("d_below", P)]


class FsBedParticles(C.Structure):
    _fields_ = [(n, P) for n in ("x", "y", "z", "alive", "m_solid", "m_water", "m_char",
                                 "T_s", "m_water_0", "sav", "m_char_max")]


class FsBedSegments(C.Structure):
    _fields_ = [("nseg", I), ("seg_start", P), ("seg_cell", P), ("perm", P)]


class FsBedSources(C.Structure):
    _fields_ = [(n, P) for n in ("S_pyro", "S_drying", "Q_pyro", "Q_drying", "Y_F_source",
                                 "Q_char", "Q_smold", "Q_g_conv")]


class FsBedParams(C.Structure):
    _fields_ = [("dt", D), ("h_conv", D), ("rho_true", D), ("cp_solid", D), ("eps_solid", D),
                ("T_amb", D), ("view", D), ("h_bed", D), ("kappa_bed", D), ("char_cap", D),
                ("ash_exp", D), ("do_dry", I), ("do_pyro", I), ("do_char", I),
                ("do_smold", I), ("mode", I), ("geometric", I), ("n_split", I),
                ("Qsx", P), ("q_rad", P), ("drip_on", I), ("n_z_bed", I), ("i_src0", I),
                ("i_src1", I)]


class FsColumnDiag(C.Structure):
    _fields_ = [("n_ign", I64), ("lead_i", I), ("S_pyro_max", D), ("hrr_max", D)]


class FsCaseDesc(C.Structure):
    _fields_ = ([("nx", I), ("ny", I), ("nz", I), ("n_z_bed", I), ("dx", D), ("dy", D),
                 ("dz", P), ("d_above", P), ("d_below", P)]
                + [(n, D) for n in ("T_amb", "h_bed", "sav", "cfl", "dz_min", "U_mf", "min_dt_s",
                                    "dt0", "ignition_duration_s", "ignition_q_mult",
                                    "canopy_C_d", "canopy_beta_p", "canopy_beta_d", "h_conv",
                                    "rho_solid_true", "cp_solid", "eps_solid", "view_factor",
                                    "kappa_bed_eff", "char_ox_flux_cap", "char_ox_ash_exp",
                                    "chi_rad", "T_ign", "proj_div_tol", "x_front0",
                                    "bed_x_end")]
                + [(n, I) for n in ("drying_mode", "view_factor_geometric", "n_per_cell",
                                    "i_src_start", "i_src_end", "proj_max_iter",
                                    "dom_subcycle_every", "edc_extinction_enable")]
                + [("M", I), ("ox", P), ("oy", P), ("oz", P), ("w", P), ("n_soil", I),
                   ("soil_dz", P), ("soil_d_above", P), ("soil_d_below", P), ("form", I),
                   ("projection_rtol", D), ("proj_maxiter", I), ("overlap_dom", I)])


class FsInitState(C.Structure):
    _fields_ = ([(n, P) for n in ("rho", "u", "v", "w", "T_g", "Y_fuel", "Y_O2", "Y_H2O", "T_s",
                                  "alpha_s", "k_turb", "eps_turb", "nu_t", "phi", "u_inlet",
                                  "sigma_x", "T_soil")]
                + [("n_particles", I64)]
                + [(n, P) for n in ("px", "py", "pz", "m_solid", "m_water", "m_char", "pT_s",
                                    "m_water_0", "psav", "m_char_max", "alive")])


class FsStepOut(C.Structure):
    _fields_ = [("steps", I), ("finished", I), ("step_count", I64), ("t", D), ("dt", D),
                ("cg_iters", I), ("proj_iters", I), ("dom_iters", I), ("div_max", D)]


_G = C.POINTER(FsGrid)

# name -> (restype, argtypes)
SIGNATURES = {
    "fs_last_error": (C.c_char_p, []),
    "fs_version": (I, []),
    "fs_launch_count": (C.c_ulonglong, []),
    "fs_species_transport": (I, [_G, I, PP, PP, PP, C.POINTER(D), P, P, P, P, D, D, P]),
    "fs_species_sources": (I, [I64, P, P, P, P, P, P, P, P, P]),
    "fs_species_step": (I, [_G, PP, PP, P, P, C.POINTER(D), P, P, P, P, D, D, D, P]),
    "fs_advect_scalar_muscl": (I, [_G, P, P, P, P, P, D, P]),
    "fs_gas_energy_adv": (I, [_G, P, P, P, P, P, D, D, D, P]),
    "fs_turb_diffusion_nsub": (I, [_G, P, D, D, C.POINTER(I), C.POINTER(D), P]),
    "fs_turb_diffusion_substep": (I, [_G, I, PP, PP, P, D, D, I, C.POINTER(D),
                                      C.POINTER(D), P]),
    "fs_drag_force": (I, [I64, P, P, P, P, P, D, D, P, P, P, P]),
    "fs_tentative_velocity": (I, [_G, P, P, P, P, P, P, P, P, P, D, D, P, P, P, P, P, P,
                                  D, D, P]),
    "fs_outflow_sponge": (I, [_G, P, P, P, P, D, D, P]),
    "fs_k_epsilon": (I, [_G, P, P, P, P, P, P, P, P, P, P, P, P, P, P, P, D, D, D, D, D, P]),
    "fs_edc_scratch_bytes": (I64, [I64]),
    "fs_edc": (I, [I64, P, P, P, P, P, P, P, P, D, D, D, I, D, D, I, P, P]),
    "fs_edc_noalloc": (I, [I64, P, P, P, P, P, P, P, P, D, D, D, I, D, D, I, P]),
    "fs_gas_energy_update": (I, [_G, P, P, P, P, P, P, P, P, P, D, D, D, I, I, I, I, P]),
    "fs_gas_energy_solid_update": (I, [_G, P, P, P, P, P, P, P, P, P, D, D, D, I, I, I, I,
                                       P, P, D, D, D, D, D, P]),
    "fs_eos": (I, [_G, P, P, P, P, D, P]),
    "fs_clip": (I, [I64, P, D, D, P]),
    "fs_div_target": (I, [I64, P, P, P, P, D, P, P]),
    "fs_ctx_create": (I, [C.POINTER(FsCaseDesc), C.POINTER(FsInitState), C.POINTER(P)]),
    "fs_ctx_destroy": (None, [P]),
    "fs_ctx_last_error": (C.c_char_p, [P]),
    "fs_step": (I, [P, I, C.POINTER(FsStepOut)]),
    "fs_batch_run": (I, [C.POINTER(P), I, I, C.POINTER(FsStepOut)]),
    "fs_ctx_field_size": (I64, [P, I]),
    "fs_ctx_field": (P, [P, I]),
    "fs_ctx_read": (I, [P, I, P]),
    "fs_ctx_write": (I, [P, I, P]),
    "fs_ctx_stream": (P, [P]),
    "fs_convert": (I, [I64, I, PP, PP, I, P]),
    "fs_edc_f32_scratch_bytes": (I64, [I64]),
    "fs_edc_f32": (I, [I64, P, P, P, P, P, P, P, P, D, D, D, I, D, D, I, P, P]),
    "fs_species_step_f32": (I, [_G, PP, PP, P, P, C.POINTER(D), P, P, P, P, D, D, D, P]),
    "fs_turb_diffusion_substep_f32": (I, [_G, I, PP, PP, P, D, D, I, C.POINTER(D),
                                          C.POINTER(D), P]),
    "fs_gas_energy_update_f32": (I, [_G, P, P, P, P, P, P, P, P, P, D, D, D, I, I, I, I, P]),
    "fs_clip_f32": (I, [I64, P, D, D, P]),
    "fs_stencil_status": (I, [I]),
    "fs_set_tma": (I, [I]),
    "fs_column_diag_scratch_bytes": (I64, [_G]),
    "fs_column_diag": (I, [_G, P, P, P, P, D, D, D, P, P, C.POINTER(FsColumnDiag), P]),
    "fs_ignition_pulse": (I, [_G, P, I, I, I, D, P]),
    "fs_solid_conduction": (I, [_G, P, P, P, D, D, D, D, P]),
    "fs_solid_conduction_capped": (I, [_G, P, P, P, D, D, D, D, D, D, P]),
    "fs_soil_step": (I, [I, I, I, P, P, D, P, P, P, D, D, D, D, D, P]),
    "fs_proj_create": (I, [_G, PP]),
    "fs_proj_destroy": (None, [P]),
    "fs_proj_rebuild": (I, [P, P, P]),
    "fs_proj_project": (I, [P, P, P, P, P, P, D, D, I, C.POINTER(I), P]),
    "fs_proj_pressure": (P, [P]),
    "fs_proj_apply": (I, [P, P, P, P]),
    "fs_proj_configure": (I, [P, I, D]),
    "fs_proj_set_fine_sweeps": (I, [P, I]),
    "fs_proj_set_coarse_tail": (I, [P, I]),
    "fs_proj_set_precision": (I, [P, I]),
    "fs_proj_stats": (I, [P, C.POINTER(D)]),
    "fs_proj_set_learned": (I, [P, P, I, D]),
    "fs_proj_set_log": (I, [P, P, P]),
    "fs_proj_fcg_stats": (I, [P, C.POINTER(D)]),
    "fs_proj_smooth_pair": (I, [P, P, P, P, P, P]),
    "fs_unet_set_output_scale": (I, [P, C.c_float]),
    "fs_unet_nparams": (I64, []),
    "fs_unet_create": (I, [I, I, I, PP]),
    "fs_unet_destroy": (None, [P]),
    "fs_unet_set_params": (I, [P, P, I64, P]),
    "fs_unet_get_params": (I, [P, P, I64, P]),
    "fs_unet_get_grads": (I, [P, P, I64, P]),
    "fs_unet_apply": (I, [P, P, P, P]),
    "fs_unet_forward": (I, [P, P, P, P]),
    "fs_unet_grad": (I, [P, P, P, C.POINTER(D), P]),
    "fs_unet_train_step": (I, [P, P, P, C.c_float, C.POINTER(D), P]),
    "fs_divergence_max": (I, [_G, P, P, P, P, P, P, C.POINTER(D), P]),
    "fs_dom_create": (I, [_G, I, C.POINTER(D), C.POINTER(D), C.POINTER(D), C.POINTER(D), D,
                          PP]),
    "fs_dom_destroy": (None, [P]),
    "fs_dom_solve": (I, [P, P, P, P, P, D, D, P, P, P, P, P, P, P, P]),
    "fs_dom_begin": (I, [P, P, P, P, P, D, D, P, P, P, P, P]),
    "fs_dom_end": (I, [P, P, P, P, P]),
    "fs_dom_intensity": (P, [P]),
    "fs_dom_iterations": (I, [P]),
    "fs_dom_set_sweep_mode": (I, [P, I, I]),
    "fs_dom_sweep_mode": (I, [P]),
    "fs_dom_set_sweep_kernel": (I, [P, I]),
    "fs_dom_sweep_kernel": (I, [P]),
    "fs_dom_launch_shape": (I, [P, P]),
    "fs_dom_set_wait_test": (I, [P, I]),
    "fs_index_divide": (I, [C.c_uint32, C.c_int64, P, P]),
    "fs_dom_set_octant_groups": (I, [P, I]),
    "fs_dom_set_precision": (I, [P, I]),
    "fs_dom_load_intensity": (I, [P, P, P]),
    "fs_dom_wrap_size": (I64, [P]),
    "fs_dom_get_wrap": (I, [P, P, P]),
    "fs_dom_set_wrap": (I, [P, P, P]),
    "fs_dom_sweep_timing": (I, [P, I, C.POINTER(D), C.POINTER(C.c_longlong)]),
    "fs_bed_step": (I, [_G, C.POINTER(FsBedParticles), C.POINTER(FsBedSegments),
                        C.POINTER(FsBedSources), C.POINTER(FsBedParams), P, P, P]),
    "fs_bed_aggregate": (I, [C.POINTER(FsBedParticles), C.POINTER(FsBedSegments), P, I, P]),
    "fs_bed_hcond": (I, [_G, P, P, P, I, D, D, D, D, C.POINTER(FsBedParticles),
                         C.POINTER(FsBedSegments), P, P]),
    "fs_levelset": (I, [_G, P, P, P, D, I, P]),
    "fs_active_count": (I, [I64, P, P, P, P, P, P]),
    "fs_copy_to_host": (I, [P, P, I64, P]),
    "fs_field_max": (I, [_G, P, I, C.POINTER(D), P]),
    "fs_field_max_multi": (I, [_G, I, PP, C.POINTER(I), C.POINTER(D), P, P]),
}

STATUS = {0: "ok", 1: "bad argument", 2: "non-finite value", 3: "solver did not converge",
          4: "device wait timed out", 5: "CUDA error"}


class FireStepError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"firestep status {status} ({STATUS.get(status, '?')}): {msg}")
        self.status = status


_lib = None


def lib():
    """Load the shared library (once) and bind every declared entry point."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(
            f"libfirestep.so not found at {LIB_PATH}; build it with "
            f"`make -C firewebapp_b200/csrc` (no CPU fallback exists)")
    L = C.CDLL(str(LIB_PATH))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(L, name)  # AttributeError -> missing symbol: fail loudly
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def check(status: int, where: str = ""):
    if status != 0:
        msg = lib().fs_last_error().decode(errors="replace")
        raise FireStepError(status, f"{where}: {msg}" if where else msg)


def ptr(t) -> int:
    """Device pointer of a torch tensor (None -> NULL)."""
    if t is None:
        return None
    return t.data_ptr()


def ptr_array(ts):
    arr = (C.c_void_p * len(ts))()
    for k, t in enumerate(ts):
        arr[k] = ptr(t)
    return arr


def dbl_array(xs):
    arr = (C.c_double * len(xs))()
    for k, x in enumerate(xs):
        arr[k] = float(x)
    return arr


def stream_ptr(stream=None):
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream
