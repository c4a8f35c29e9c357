"""ctypes binding of libghost_b200.so (the C ABI of include/ghost_b200.h).

The library is the only compute path: if it is missing or cannot load, this
module raises, and nothing falls back to another implementation.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libghost_b200.so")

GHOST_OK = 0
TIMER_NAMES = ["z_inv", "y_inv", "x_nl", "y_fwd", "z_fwd", "z_c2c", "x_c2r", "x_r2c", "pointwise", "reduce"]
ERRORS = {
    1: "GHOST_ERR_ARG", 2: "GHOST_ERR_SIZE", 3: "GHOST_ERR_ALLOC", 4: "GHOST_ERR_CUDA",
    5: "GHOST_ERR_TIMEOUT", 6: "GHOST_ERR_NAN", 7: "GHOST_ERR_STATE", 8: "GHOST_ERR_NODEV", 9: "GHOST_ERR_IO",
}
GHOST_SINGLE = 4
GHOST_DOUBLE = 8
GHOST_REAL_TO_COMPLEX = -1
GHOST_COMPLEX_TO_REAL = 1


class GhostError(RuntimeError):
    def __init__(self, code: int, where: str, msg: str):
        super().__init__(f"{where}: {ERRORS.get(code, code)}: {msg}")
        self.code = code


class GhostInfo(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
        ("precision", ctypes.c_int), ("anis", ctypes.c_int),
        ("nmax", ctypes.c_int), ("nmaxperp", ctypes.c_int),
        ("kmax", ctypes.c_double), ("tiny", ctypes.c_double),
        ("Lx", ctypes.c_double), ("Ly", ctypes.c_double), ("Lz", ctypes.c_double),
        ("Dkx", ctypes.c_double), ("Dky", ctypes.c_double), ("Dkz", ctypes.c_double),
        ("Dkk", ctypes.c_double),
        ("spectral_elems", ctypes.c_size_t), ("real_elems", ctypes.c_size_t),
    ]


P = ctypes.c_void_p
I = ctypes.c_int
D = ctypes.c_double
PD = ctypes.POINTER(ctypes.c_double)
PP = ctypes.POINTER(ctypes.c_void_p)  # an array of device pointers

# name -> argument types (all return int status)
SIGNATURES = {
    "ghost_ctx_create": [I, I, I, D, D, D, I, I, ctypes.POINTER(P)],
    "ghost_ctx_destroy": [P],
    "ghost_ctx_get_info": [P, ctypes.POINTER(GhostInfo)],
    "ghost_ctx_set_stream": [P, P],
    "ghost_ctx_set_kmax": [P, D],
    "ghost_ctx_synchronize": [P],
    "ghost_ctx_set_wait_cap": [P, ctypes.c_uint],
    "ghost_ctx_inject_stall": [P, I],
    "ghost_ctx_launch_count": [P, ctypes.POINTER(ctypes.c_longlong)],
    "ghost_ctx_enable_timers": [P, I],
    "ghost_ctx_read_timers": [P, PD, ctypes.POINTER(ctypes.c_longlong)],
    "ghost_fftp3d_create_plan": [P, ctypes.POINTER(ctypes.c_int), I, I, ctypes.POINTER(P)],
    "ghost_fftp3d_destroy_plan": [P],
    "ghost_fftp3d_real_to_complex": [P, P, P],
    "ghost_fftp3d_complex_to_real": [P, P, P],
    "ghost_derivk3": [P, P, P, I],
    "ghost_laplak3": [P, P, P],
    "ghost_rotor3": [P, P, P, P, I],
    "ghost_prodre3": [P, P, P, P, P, P, P],
    "ghost_nonlhd3": [P, P, P, P, P, I],
    "ghost_energy": [P, P, P, P, PD, I],
    "ghost_helicity": [P, P, P, P, PD],
    "ghost_cross": [P, P, P, P, P, P, P, PD, I],
    "ghost_divergence": [P, P, P, P, PD],
    "ghost_maxabs": [P, P, P, P, PD, I],
    "ghost_spectrumc": [P, P, P, P, I, I, PD, PD],
    "ghost_spectrumc_noalloc": [P, P, P, P, I, I, PD, PD],
    "ghost_hdcheck": [P, P, P, P, P, P, P, I, I, PD],
    "ghost_normalize": [P, P, P, P, D, I],
    "ghost_sharp": [P, P, P, D],
    "ghost_hd_rkstep1": [P, P, P, P, P, P, P],
    "ghost_hd_rkstep2": [P, I, D, D, P, P, P, P, P, P, P, P, P],
    "ghost_hd_run": [P, I, I, D, D, P, P, P, P, P, P, P, P, P],
    "ghost_advect3": [P, P, P, P, P, P],
    "ghost_bouss_rkstep2": [P, I, D, D, D, D, D, D] + [P] * 12,
    "ghost_bouss_run": [P, I, I, D, D, D, D, D, D] + [P] * 8,
    "ghost_init_random_solenoidal": [P, ctypes.POINTER(ctypes.c_int32), D, D, I, D, P, P, P],
    "ghost_ctx_create_batch": [I, I, I, I, I, ctypes.POINTER(P)],
    "ghost_batch_set_nu": [P, PD],
    "ghost_batch_energy": [P, P, P, P, I, PD],
    "ghost_batch_init_random_solenoidal": [P, ctypes.POINTER(ctypes.c_int32), D, D, I, D, P, P, P],
    "ghost_ensemble_create": [I, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int), I, ctypes.POINTER(P)],
    "ghost_ensemble_destroy": [P],
    "ghost_ensemble_fields": [P, I, ctypes.POINTER(P), ctypes.POINTER(P), ctypes.POINTER(P)],
    "ghost_ensemble_class": [P, I, ctypes.POINTER(P)],
    "ghost_ensemble_init": [P, ctypes.POINTER(ctypes.c_int32), D, D, I, D, PD],
    "ghost_ensemble_autotune": [P, I, D, ctypes.POINTER(ctypes.c_int)],
    "ghost_ensemble_run": [P, I, I, D],
    "ghost_ensemble_set_mode": [P, I],
    "ghost_ensemble_get_mode": [P, ctypes.POINTER(ctypes.c_int)],
    "ghost_ensemble_energy": [P, I, PD],
    "ghost_slab_range": [I, I, I, I, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)],
    "ghost_slab_create": [I, I, I, D, D, D, I, I, I, I, ctypes.POINTER(ctypes.c_void_p)],
    "ghost_slab_destroy": [P],
    "ghost_slab_layout": [P] + [ctypes.POINTER(ctypes.c_int)] * 4,
    "ghost_slab_rows": [P, ctypes.POINTER(ctypes.c_int)],
    "ghost_slab_launch_count": [P, ctypes.POINTER(ctypes.c_longlong)],
    "ghost_slab_set_stream": [P, P],
    "ghost_slab_synchronize": [P],
    "ghost_slab_hd_front": [P, PP, PP, I, I, PP],
    "ghost_slab_hd_xpass": [P, I, PP, PP],
    "ghost_slab_hd_back": [P, I, D, D, I, PP, PP, PP, PP],
    "ghost_slab_pack": [P, I, I, I, PP, P],
    "ghost_slab_unpack": [P, I, I, I, P, PP],
    "ghost_slab_set_self_direct": [P, I],
    "ghost_slab_exchange_self": [P, I, I, I, PP, PP],
    "ghost_slab_hd_front_z": [P, PP, PP, I, I, PP],
    "ghost_slab_ypass": [P, I, I, I, PP],
    "ghost_slab_hd_back_z": [P, I, D, D, I, PP, PP, PP, PP],
    "ghost_ctx_set_tile_cfg": [P, I],
    "ghost_ctx_get_tile_cfg": [P, ctypes.POINTER(ctypes.c_int)],
    "ghost_hd_autotune": [P, I, D, D, P, P, P, P, P, P, ctypes.POINTER(ctypes.c_int)],
    "ghost_mlp_create": [I, ctypes.POINTER(P)],
    "ghost_mlp_destroy": [P],
    "ghost_mlp_set_stream": [P, P],
    "ghost_mlp_get_params": [P, P],
    "ghost_mlp_set_params": [P, P],
    "ghost_mlp_forward": [P, P, P, I],
    "ghost_mlp_gradients": [P, P, P, I, P, PD],
    "ghost_mlp_train_step": [P, P, P, I, ctypes.c_float, PD],
    "ghost_les_create": [P, I, ctypes.POINTER(P)],
    "ghost_les_destroy": [P],
    "ghost_les_truncate": [P, P, P, P],
    "ghost_les_samples": [P, P, P, P, P, ctypes.c_float, P, P],
    "ghost_les_features": [P, P, P, P, ctypes.c_float, ctypes.c_float, P],
    "ghost_les_spectral_features": [P, P, P],
    "ghost_les_tau_force": [P, P, ctypes.c_float, P, P, P, P, P, P],
    "ghost_les_set_model": [P, I, P, D, D, D, D],
    "ghost_les_set_fallback": [P, I, D],
    "ghost_les_status": [P, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_longlong)],
    "ghost_les_set_time": [P, D],
    "ghost_les_closure_force": [P, D, P, P, P, P, P, P, P, P, P],
    "ghost_les_run": [P, I, I, D, D, P, P, P, P, P, P],
    "ghost_les_edqnm_last": [P, PD, PD, PD],
    "ghost_evedqnm": [I, I, D, D, PD, D, D, PD, PD, PD],
    "ghost_evedqnm_hel": [I, I, D, D, PD, PD, D, D, I, PD, PD, PD, PD, PD, PD],
    "ghost_les_set_helicity": [P, I],
    "ghost_les_edqnm_last_hel": [P, PD, PD, PD],
    "ghost_phd_run": [P, I, I, D, D, D, P, P, P, P, P, P, P, P],
    "ghost_phaseshift": [P, P, D, D],
    "ghost_forcing_slow": [P, I, I, P, P, P, P, P, P, P, P, P],
    "ghost_vector3": [P, P, P, P, P, P, P, P, P, P],
    "ghost_nonlin3": [P, P, P, P, P, P, P, P, I],
    "ghost_gauge3": [P, P, P, P, P, I],
    "ghost_mhd_run": [P, I, I, D, D, D] + [P] * 12,
    "ghost_variance": [P, P, I, PD],
    "ghost_spectrscc": [P, P, D, PD],
    "ghost_sctrans": [P, P, P, I, PD],
    "ghost_havgcomp": [P, P, P, P, P, D, D, I, PD],
    "ghost_tbouss": [P, P, P, P, P, D, D, PD, PD, PD],
    "ghost_specpara": [P, P, P, P, I, I, PD, PD],
    "ghost_specperp": [P, P, P, P, I, I, PD, PD],
    "ghost_entpara": [P, P, P, P, P, P, P, I, PD],
    "ghost_entperp": [P, P, P, P, P, P, P, I, PD],
    "ghost_heltpara": [P, P, P, P, P, P, P, I, PD],
    "ghost_heltperp": [P, P, P, P, P, P, P, I, PD],
    "ghost_entrans": [P, P, P, P, P, P, P, I, PD],
    "ghost_heltrans": [P, P, P, P, P, P, P, I, PD],
    "ghost_io_filename": [ctypes.c_char_p, ctypes.c_char_p, I, I, ctypes.c_char_p, ctypes.c_size_t],
    "ghost_io_write": [P, P, ctypes.c_char_p, I],
    "ghost_io_read": [P, ctypes.c_char_p, I, P],
    "ghost_io_output": [P, P, ctypes.c_char_p, I],
    "ghost_io_restart": [P, ctypes.c_char_p, I, P],
}

_lib = None


def load() -> ctypes.CDLL:
    """Load the in-tree library (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m ghost_b200.build`")
    lib = ctypes.CDLL(LIB_PATH)
    for name, args in SIGNATURES.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = ctypes.c_int
    lib.ghost_last_error_string.argtypes = []
    lib.ghost_last_error_string.restype = ctypes.c_char_p
    _lib = lib
    return lib


def check(status: int, where: str) -> None:
    if status != GHOST_OK:
        msg = load().ghost_last_error_string().decode(errors="replace")
        raise GhostError(status, where, msg)
