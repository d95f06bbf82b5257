"""ctypes binding of libsod2d_b200.so (the C ABI declared in include/sod2d_b200.h).

The library is the only compute path: there is no CPU fallback.  Importing this module
without the built library, or calling into it without a CUDA device, raises.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsod2d_b200.so")

SOD_OK = 0
SOD_FP64 = 0
SOD_MIXED = 1
ERRORS = {-1: "SOD_ERR_ARG", -2: "SOD_ERR_CUDA", -3: "SOD_ERR_NONFINITE", -4: "SOD_ERR_NOT_CONVERGED",
          -5: "SOD_ERR_TIMEOUT", -6: "SOD_ERR_NOMEM", -7: "SOD_ERR_UNSUPPORTED"}

_p = C.c_void_p
_d = C.c_double
_i = C.c_int


class SodError(RuntimeError):
    def __init__(self, rc: int, msg: str):
        super().__init__(f"{ERRORS.get(rc, rc)}: {msg}")
        self.rc = rc


class SodParams(C.Structure):
    _fields_ = [("gamma_gas", _d), ("Rgas", _d), ("Cp", _d), ("Prt", _d), ("ce", _d), ("cmax", _d), ("cglob", _d),
                ("c_rho", _d), ("c_ener", _d), ("flag_normalise_entropy", C.c_int32), ("cfl_conv", _d),
                ("cfl_diff", _d), ("flag_les", C.c_int32), ("c_sgs", _d), ("flag_total_enthalpy", C.c_int32)]


class SodBcParams(C.Structure):
    _fields_ = [(n, _d) for n in ("rho_inf", "u_inf", "p_inf", "c_inf", "gamma_inf", "Rgas_inf", "T_H", "T_C")]


class SodBufferParams(C.Structure):
    _fields_ = [("on_" + s, C.c_int32) for s in ("east", "west", "north", "south", "top", "bottom")] + \
        [(n, _d) for s in "ewnstb" for n in (s + "_min", s + "_size")] + \
        [(n, _d) for n in ("rho_inf", "u_inf", "p_inf", "gamma_inf")]


class SodMeshDesc(C.Structure):
    _fields_ = [("nelem", C.c_int32), ("npoin", C.c_int32), ("npoin_orig", C.c_int32), ("porder", C.c_int32),
                ("index_base", C.c_int32), ("connec", _p), ("connec_orig", _p), ("coord_orig", _p),
                ("dlxigp_ip", _p), ("wgp", _p), ("invAtoIJK", _p), ("gmshAtoI", _p), ("gmshAtoJ", _p),
                ("gmshAtoK", _p), ("He", _p), ("gpvol", _p), ("Ml", _p), ("helem", _p), ("helem_l", _p),
                ("npoin_w", C.c_int32), ("lpoin_w", _p)]


class SodState(C.Structure):
    _fields_ = [(n, _p) for n in ("rho", "q", "E", "u", "pr", "Tem", "e_int", "eta", "csound", "machno",
                                  "mu_fluid", "mu_factor", "mu_e", "Reta", "mu_sgs")]


_SIGS = {
    "sod_params_default": (None, [_p]),
    "sod_mesh_create": (_i, [_p, _p, _p]),
    "sod_mesh_destroy": (None, [_p]),
    "sod_mesh_get_geometry": (_i, [_p, _p, _p, _p, _p, _p]),
    "sod_mesh_set_params": (_i, [_p, _p]),
    "sod_rk4_main": (_i, [_p, _p, _p, _p, _i, _p]),
    "sod_rk4_steps": (_i, [_p, _p, _p, _i, _i, _p]),
    "sod_rk4_main_host": (_i, [_p, _p, _d, _p, _i, _p]),
    "sod_step_profile": (_i, [_p, _p, _p, _i, _i, _p, _p]),
    "sod_rhs": (_i, [_p, _p, _p, _p, _p, _p, _p, _p, _p, _p, _i, _p]),
    "sod_smart_visc_spectral": (_i, [_p, _p, _p, _p, _p, _p, _p, _p, _p]),
    "sod_adapt_dt_cfl": (_i, [_p, _p, _p, _p, _p, _p, _p, _p]),
    "sod_full_convec_ijk": (_i, [_p, _p, _p, _p, _p, _p, _p, _p, _p, _p]),
    "sod_full_convec_ijk_H": (_i, [_p, _p, _p, _p, _p, _p, _p, _p, _p, _p]),
    "sod_full_convec_ijk_noalloc": (_i, [C.c_int32, C.c_int32, C.c_int32] + [_p] * 16),
    "sod_generic_scalar_convec_ijk": (_i, [_p, _p, _p, _p, _p, _p]),
    "sod_full_convec_ijk_ref": (_i, [C.c_int32] * 3 + [_p] * 20),
    "sod_full_convec_ijk_H_ref": (_i, [C.c_int32] * 3 + [_p] * 20),
    "sod_generic_scalar_convec_ijk_ref": (_i, [C.c_int32] * 3 + [_p] * 16),
    "sod_full_diffusion_ijk_ref": (_i, [C.c_int32] * 3 + [_p] * 9 + [_d, _d] + [_p] * 12),
    "sod_smart_visc_spectral_ref": (_i, [C.c_int32] * 4 + [_p] * 8 + [_d] + [_p] * 16),
    "sod_full_diffusion_ijk": (_i, [_p, _d, _d, _p, _p, _p, _p, _p, _p, _p, _p, _p, _p, _p]),
    "sod_lumped_solver": (_i, [_p, _p, _i, _p]),
    "sod_sutherland_viscosity": (_i, [C.c_int32, _p, _p, _p, _p]),
    "sod_poisson_create": (_i, [_p, _p]),
    "sod_poisson_destroy": (None, [_p]),
    "sod_poisson_apply": (_i, [_p, _p, _p, _p]),
    "sod_poisson_diag": (_i, [_p, _p, _p]),
    "sod_conjgrad_pressure": (_i, [_p, _p, _p, _i, _d, _i, _p, _p, _p]),
    "sod_csr_spmv_scal": (_i, [C.c_int32, C.c_int32, _p, _p, _p, _p, _p, _p]),
    "sod_rhs_vjp": (_i, [_p, _p, _p, _p, _p, _p, _p, _p, _p, _p, _p, _p, _p]),
    "sod_rk4_step_vjp": (_i, [_p] * 16),
    "sod_tgv_diagnostics": (_i, [_p, _p, _p, _p, _p, _d, _d, _p, _p]),
    "sod_mesh_set_boundaries": (_i, [_p] * 6),
    "sod_mesh_set_buffer": (_i, [_p] * 4),
    "sod_set_rhs_config": (_i, [_p, _i, _i]),
    "sod_compute_field_derivs": (_i, [_p] * 9),
    "sod_bc_dirichlet_prim_vjp": (_i, [_p] * 8),
    "sod_mesh_set_wall_model": (_i, [_p, _i, _i, _i, _p, _p, _p, _i, _p, _p, _p, _p, _p, _p]),
    "sod_wall_model": (_i, [_p] * 7),
    "sod_wall_model_tauw": (_i, [_p] * 3),
    "sod_mesh_set_source_term": (_i, [_p] * 2),
    "sod_update_buffer": (_i, [_p] * 5),
    "sod_bc_dirichlet_prim": (_i, [_p] * 7),
    "sod_bc_fix_dirichlet_residual": (_i, [_p] * 5),
    "sod_bc_fix_dirichlet_residual_entropy": (_i, [_p] * 3),
    "sod_legacy_mass_convec": (_i, [_i] * 5 + [_p] * 7),
    "sod_legacy_generic_scalar_convec": (_i, [_i] * 5 + [_p] * 7),
    "sod_legacy_mom_convec": (_i, [_i] * 5 + [_p] * 9),
    "sod_legacy_ener_convec": (_i, [_i] * 5 + [_p] * 9),
    "sod_legacy_mom_diffusion": (_i, [_i] * 5 + [_p] * 8),
    "sod_rk4_main_record": (_i, [_p, _p, _p, _p, _p, _i, _p]),
    "sod_batch_create": (_i, [_p, _i, _p]),
    "sod_batch_destroy": (None, [_p]),
    "sod_batch_set_member": (_i, [_p, _i, _p]),
    "sod_batch_get_member": (_i, [_p, _i, _p]),
    "sod_batch_set_dt": (_i, [_p, _p]),
    "sod_batch_get_dt": (_i, [_p, _p]),
    "sod_batch_adapt_dt": (_i, [_p, _p]),
    "sod_batch_mesh": (_i, [_p, _p]),
    "sod_batch_autotune": (_i, [_p, _i, _p, _p, _p]),
    "sod_batch_rk4_steps": (_i, [_p, _i, _i, _p]),
    "sod_autotune": (_i, [_p, _p, _i, _p, _p, _p]),
    "sod_autotune_table": (_i, [_p, _i, _i, _p, _p, _p]),
    "sod_set_stage_launch": (_i, [_p, _i, _i]),
    "sod_last_error": (C.c_char_p, []),
    "sod_version": (C.c_char_p, []),
    "sod_launch_count": (C.c_int64, []),
    "sod_check_finite": (_i, [_p, _p]),
    "sod_set_wait_timeout": (None, [_d]),
}

_lib = None


def load(required: bool = True):
    """Load the library.  Raises (never falls back) when it is missing."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is not built; run `python -m sod2d_refmap_b200.build`")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(L, name, None)
            if fn is None:
                continue
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def exported_symbols():
    L = load()
    return [n for n in _SIGS if hasattr(L, n)]


def check(rc: int):
    if rc != SOD_OK:
        msg = load().sod_last_error()
        raise SodError(rc, msg.decode() if msg else "")
    return rc


def launch_count() -> int:
    return int(load().sod_launch_count())
