"""ctypes wrapper of the CPU oracle (test infrastructure; see sod2d_oracle.hpp).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs import this module.
It never backs the product path: the library in sod2d_refmap_b200 has no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle_sod2d.so")

_p = C.c_void_p
_i32p = C.POINTER(C.c_int32)


class ElemCtx(C.Structure):
    _fields_ = [("nelem", C.c_int), ("npoin", C.c_int), ("connec", _p), ("He", _p), ("gpvol", _p),
                ("dlxigp_ip", _p), ("invAtoIJK", _p), ("gmshAtoI", _p), ("gmshAtoJ", _p),
                ("gmshAtoK", _p), ("ncolors", C.c_int), ("color_ptr", _p), ("color_elems", _p),
                ("npoin_w", C.c_int), ("lpoin_w", _p)]


class Params(C.Structure):
    _fields_ = [("gamma_gas", C.c_double), ("Rgas", C.c_double), ("Cp", C.c_double), ("Prt", C.c_double),
                ("ce", C.c_double), ("cmax", C.c_double), ("cglob", C.c_double), ("c_rho", C.c_double),
                ("c_ener", C.c_double), ("flag_normalise_entropy", C.c_int), ("cfl_conv", C.c_double),
                ("cfl_diff", C.c_double), ("flag_les", C.c_int), ("c_sgs", C.c_double),
                ("flag_total_enthalpy", C.c_int)]


class State(C.Structure):
    _fields_ = [(n, _p) for n in ("rho", "u", "q", "pr", "E", "Tem", "e_int", "eta", "csound", "machno",
                                  "mu_fluid", "mu_e", "mu_sgs", "mue_l")]


class StageCapture(C.Structure):
    _fields_ = [("Rmass", _p), ("Rmom", _p), ("Rener", _p), ("Reta", _p), ("stage", C.c_int)]


class BcData(C.Structure):
    _fields_ = [("bou_codes_nodes", _p), ("lnbn_nodes", _p), ("normals", _p), ("u_buffer", _p)] + \
        [(n, C.c_double) for n in ("rho_inf", "u_inf", "p_inf", "c_inf", "gamma_inf", "Rgas_inf", "T_H", "T_C")]


class WallModelData(C.Structure):
    _fields_ = [("type", C.c_int), ("nboun", C.c_int), ("npbou", C.c_int), ("numBoundsWM", C.c_int)] + \
        [(n, _p) for n in ("bound", "bounorm", "wgp_b", "listBoundsWM", "point2elem", "coord", "normals", "zo",
                           "walave", "tauw")]


class WallModel:
    """Wall-model data for the oracle (0-based ids; arrays kept alive here); tauw receives the
    wall shear of the last evaluation."""

    def __init__(self, wtype, bound, bounorm, wgp_b, list_wm, point2elem, coord, normals, zo=None, walave=None):
        self.bound = np.asfortranarray(bound, dtype=np.int32)
        self.bounorm = np.asfortranarray(bounorm, dtype=np.float64)
        self.wgp_b = np.ascontiguousarray(wgp_b, dtype=np.float64)
        self.list_wm = np.ascontiguousarray(list_wm, dtype=np.int32)
        self.point2elem = np.ascontiguousarray(point2elem, dtype=np.int32)
        self.coord = np.asfortranarray(coord, dtype=np.float64)
        self.normals = np.asfortranarray(normals, dtype=np.float64)
        self.zo = None if zo is None else np.ascontiguousarray(zo, dtype=np.float64)
        self.walave = None if walave is None else np.asfortranarray(walave, dtype=np.float64)
        self.tauw = np.zeros((len(self.point2elem), 3), order="F")
        pz = lambda a: ptr(a).value if a is not None else None
        self.c = WallModelData(int(wtype), self.bound.shape[0], self.bound.shape[1], len(self.list_wm),
                               pz(self.bound), pz(self.bounorm), pz(self.wgp_b), pz(self.list_wm), pz(self.point2elem),
                               pz(self.coord), pz(self.normals), pz(self.zo), pz(self.walave), pz(self.tauw))


class BufferData(C.Structure):
    _fields_ = [("coord", _p), ("u_buffer", _p), ("on", C.c_int32 * 6), ("mn", C.c_double * 6),
                ("sz", C.c_double * 6)] + [(n, C.c_double) for n in ("rho_inf", "u_inf", "p_inf", "gamma_inf")]


BUFFER_SIDES = ("east", "west", "north", "south", "top", "bottom")


class BufferZone:
    """Buffer-zone data (flag_buffer_on) for the oracle: prm is the flat dict of
    sod2d_refmap_b200.mesh.buffer_params (on_*, *_min, *_size per side, nscbc_* values)."""

    def __init__(self, coord, u_buffer, prm: dict):
        self.coord = np.asfortranarray(coord, dtype=np.float64)
        self.u_buffer = np.asfortranarray(u_buffer, dtype=np.float64)
        on = (C.c_int32 * 6)(*(int(prm["on_" + s]) for s in BUFFER_SIDES))
        mn = (C.c_double * 6)(*(float(prm[s[0] + "_min"]) for s in BUFFER_SIDES))
        sz = (C.c_double * 6)(*(float(prm[s[0] + "_size"]) for s in BUFFER_SIDES))
        self.c = BufferData(ptr(self.coord).value, ptr(self.u_buffer).value, on, mn, sz,
                            *(float(prm[k]) for k in ("rho_inf", "u_inf", "p_inf", "gamma_inf")))


class Boundaries:
    """Boundary data of a non-periodic mesh for the oracle (arrays kept alive here)."""

    def __init__(self, codes, lnbn, normals, u_buffer, bc: dict):
        self.codes = np.ascontiguousarray(codes, dtype=np.int32)
        self.lnbn = np.ascontiguousarray(lnbn, dtype=np.int32)
        self.normals = np.asfortranarray(normals, dtype=np.float64)
        self.u_buffer = np.asfortranarray(u_buffer, dtype=np.float64)
        self.c = BcData(ptr(self.codes).value, ptr(self.lnbn).value, ptr(self.normals).value,
                        ptr(self.u_buffer).value,
                        *(float(bc[k]) for k in ("rho_inf", "u_inf", "p_inf", "c_inf", "gamma_inf", "Rgas_inf",
                                                 "T_H", "T_C")))


def build() -> str:
    """Compile the oracle with its Makefile (idempotent)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        L.oracle_adapt_dt_cfl.restype = C.c_double
        L.oracle_set_threads.restype = C.c_int
        L.oracle_conjgrad_pressure.restype = C.c_int
        L.oracle_rk_4_main.argtypes = [C.POINTER(ElemCtx), C.POINTER(Params), _p, _p, _p, _p, _p, _p,
                                       C.c_double, C.c_int, C.POINTER(State), C.POINTER(StageCapture),
                                       C.POINTER(BcData), C.POINTER(BufferData), _p, C.POINTER(WallModelData)]
        L.oracle_wall_model.argtypes = [C.POINTER(ElemCtx), C.POINTER(WallModelData), _p, _p, _p, _p]
        L.oracle_compute_field_derivs.argtypes = [C.POINTER(ElemCtx), _p, _p, _p, _p, _p, _p, _p]
        L.oracle_update_buffer.argtypes = [C.c_int, C.POINTER(BufferData), _p, _p, _p]
        L.oracle_bc_dirichlet_prim.argtypes = [C.c_int, C.POINTER(BcData), _p, _p, _p, _p, _p]
        L.oracle_bc_jvp.argtypes = [C.c_int, C.POINTER(BcData)] + [_p] * 14
        L.oracle_bc_fix_dirichlet_residual.argtypes = [C.c_int, C.POINTER(BcData), _p, _p, _p]
        L.oracle_bc_fix_dirichlet_residual_entropy.argtypes = [C.c_int, C.POINTER(BcData), _p]
        L.oracle_adapt_dt_cfl.argtypes = [C.POINTER(ElemCtx), _p, _p, _p, C.c_double, C.c_double, _p, _p, _p]
        L.oracle_conjgrad_pressure.argtypes = [C.POINTER(ElemCtx), _p, _p, _p, C.c_int, C.c_double,
                                               C.POINTER(C.c_double)]
        _lib = L
    return _lib


def ptr(a: np.ndarray):
    """A pointer to a's data that keeps a alive (safe for temporaries in an argument list)."""
    return a.ctypes.data_as(C.c_void_p)


def set_threads(n: int) -> int:
    return lib().oracle_set_threads(int(n))


def box_colouring(n: int):
    """Colour classes of an n^3 periodic box such that elements of one class share no node."""
    e = np.arange(n ** 3, dtype=np.int64)
    ex, ey, ez = e % n, (e // n) % n, e // (n * n)

    def cl(v):
        c = v % 2
        if n % 2 == 1:
            c = np.where(v == n - 1, 2, c)
        return c

    col = cl(ex) + 3 * (cl(ey) + 3 * cl(ez))
    order = np.argsort(col, kind="stable").astype(np.int32)
    counts = np.bincount(col, minlength=27)
    ptrs = np.concatenate([[0], np.cumsum(counts)]).astype(np.int32)
    return ptrs, order


class OracleMesh:
    """Holds a BoxMesh's arrays and the oracle's geometry (He, gpvol, Ml, helem, helem_l)."""

    def __init__(self, mesh, colour: bool = True):
        L = lib()
        T = mesh.tables
        self.mesh = mesh
        self.nelem, self.npoin = mesh.nelem, mesh.npoin
        # shape tables restated by the oracle itself (checked against the product's in tests)
        self.xgp = np.zeros((64, 3), order="F"); self.wgp = np.zeros(64)
        self.Ngp = np.zeros((64, 64), order="F"); self.dNgp = np.zeros((3, 64, 64), order="F")
        self.dlxigp_ip = np.zeros((64, 3, 4), order="F")
        self.invAtoIJK = np.zeros((4, 4, 4), np.int32, order="F")
        self.gI = np.zeros(64, np.int32); self.gJ = np.zeros(64, np.int32); self.gK = np.zeros(64, np.int32)
        atoIJK = np.ascontiguousarray(T.atoIJK, dtype=np.int32)
        L.oracle_shape_tables(ptr(atoIJK), ptr(self.xgp), ptr(self.wgp), ptr(self.Ngp), ptr(self.dNgp),
                              ptr(self.dlxigp_ip), ptr(self.invAtoIJK), ptr(self.gI), ptr(self.gJ), ptr(self.gK))
        self.connec = np.asfortranarray(mesh.connec, dtype=np.int32)
        self.connec_orig = np.asfortranarray(mesh.connec_orig, dtype=np.int32)
        self.He = np.zeros((3, 3, 64, self.nelem), order="F")
        self.gpvol = np.zeros((1, 64, self.nelem), order="F")
        L.oracle_elem_jacobian(self.nelem, mesh.npoin_orig, ptr(self.connec_orig), ptr(mesh.coord_orig),
                               ptr(self.dNgp), ptr(self.wgp), ptr(self.gpvol), ptr(self.He))
        self.Ml = np.zeros(self.npoin)
        L.oracle_lumped_mass(self.nelem, self.npoin, ptr(self.connec), ptr(self.gpvol), ptr(self.Ml))
        self.helem = np.zeros(self.nelem)
        L.oracle_char_length(self.nelem, mesh.npoin_orig, ptr(self.connec_orig), ptr(mesh.coord_orig), ptr(self.helem))
        self.helem_l = np.zeros((self.nelem, 64), order="F")
        L.oracle_char_length_spectral(self.nelem, mesh.npoin_orig, ptr(self.connec_orig), ptr(mesh.coord_orig),
                                      ptr(self.helem_l))
        if colour:
            self.cptr, self.celems = box_colouring(mesh.n)
            ncol = len(self.cptr) - 1
        else:
            self.cptr, self.celems = np.zeros(1, np.int32), np.zeros(1, np.int32)
            ncol = 0
        lw = mesh.extra.get("lpoin_w") if getattr(mesh, "extra", None) else None
        self.lpoin_w = None if lw is None else np.ascontiguousarray(lw, dtype=np.int32)
        self.ctx = ElemCtx(self.nelem, self.npoin, ptr(self.connec).value, ptr(self.He).value,
                           ptr(self.gpvol).value, ptr(self.dlxigp_ip).value, ptr(self.invAtoIJK).value,
                           ptr(self.gI).value, ptr(self.gJ).value, ptr(self.gK).value, ncol,
                           ptr(self.cptr).value, ptr(self.celems).value,
                           0 if lw is None else len(self.lpoin_w), 0 if lw is None else ptr(self.lpoin_w).value)


def params_of(prm) -> Params:
    return Params(prm.gamma_gas, prm.Rgas, prm.Cp, prm.Prt, prm.ce, prm.cmax, prm.cglob, prm.c_rho,
                  prm.c_ener, int(prm.flag_normalise_entropy), prm.cfl_conv, prm.cfl_diff,
                  int(getattr(prm, "flag_les", 0)), float(getattr(prm, "c_sgs", 0.025)),
                  int(getattr(prm, "flag_total_enthalpy", 0)))


def adapt_dt(om: OracleMesh, st, prm) -> float:
    return lib().oracle_adapt_dt_cfl(C.byref(om.ctx), ptr(om.helem), ptr(st.u), ptr(st.csound), prm.cfl_conv,
                                     prm.cfl_diff, ptr(st.mu_fluid), ptr(st.mu_sgs), ptr(st.rho))


def rk4(om: OracleMesh, prm, st, dt: float, nsteps: int = 1, capture_stage: int = 0,
        bnd: "Boundaries | None" = None, buf: "BufferZone | None" = None, source=None,
        wall: "WallModel | None" = None):
    """Runs nsteps rk_4_main steps in place on st (a FlowState).  Returns the stage residuals of
    capture_stage (1..4) of the first step when requested.  bnd selects the non-periodic path,
    buf the buffer zone (flag_buffer_on), source (npoin,3) the constant momentum source term."""
    src = None if source is None else np.asfortranarray(source, dtype=np.float64)
    P = params_of(prm)
    mue_l = np.zeros((om.nelem, 64), order="F")
    S = State(*(ptr(a).value for a in (st.rho, st.u, st.q, st.pr, st.E, st.Tem, st.e_int, st.eta, st.csound,
                                       st.machno, st.mu_fluid, st.mu_e, st.mu_sgs, mue_l)))
    cap = None
    out = None
    if capture_stage:
        out = dict(Rmass=np.zeros(om.npoin), Rmom=np.zeros((om.npoin, 3), order="F"), Rener=np.zeros(om.npoin),
                   Reta=np.zeros(om.npoin))
        cap = StageCapture(ptr(out["Rmass"]).value, ptr(out["Rmom"]).value, ptr(out["Rener"]).value,
                           ptr(out["Reta"]).value, int(capture_stage))
    lib().oracle_rk_4_main(C.byref(om.ctx), C.byref(P), ptr(om.Ml), ptr(st.mu_factor), ptr(om.gpvol), ptr(om.wgp),
                           ptr(om.helem), ptr(om.helem_l), float(dt), int(nsteps), C.byref(S),
                           C.byref(cap) if cap is not None else None, C.byref(bnd.c) if bnd is not None else None,
                           C.byref(buf.c) if buf is not None else None, ptr(src) if src is not None else None,
                           C.byref(wall.c) if wall is not None else None)
    return out


def wall_model(om: OracleMesh, wall: WallModel, rho, ui, mu_fluid, Rdiff):
    """evalWallModel* in place on Rdiff (npoin,3) Fortran order; wall.tauw receives tauw."""
    lib().oracle_wall_model(C.byref(om.ctx), C.byref(wall.c), ptr(rho), ptr(ui), ptr(mu_fluid), ptr(Rdiff))


def levi_civita() -> np.ndarray:
    """The (3,3,3) symbol CFDSolverBase sets (CFDSolverBase.f90:1248-1253)."""
    e = np.zeros((3, 3, 3), order="F")
    e[1, 2, 0] = 1.0; e[2, 1, 0] = -1.0; e[0, 2, 1] = -1.0; e[2, 0, 1] = 1.0; e[0, 1, 2] = 1.0; e[1, 0, 2] = -1.0
    return e


def compute_field_derivs(om: OracleMesh, rho, u, levi=None):
    """compute_fieldDerivs: (gradRho (npoin,3), curlU (npoin,3), divU, Qcrit)."""
    N = om.npoin
    lv = np.asfortranarray(levi_civita() if levi is None else levi, dtype=np.float64)
    r = np.ascontiguousarray(rho, dtype=np.float64)
    uu = np.asfortranarray(u, dtype=np.float64)
    g = np.zeros((N, 3), order="F"); c = np.zeros((N, 3), order="F"); dv = np.zeros(N); qc = np.zeros(N)
    lib().oracle_compute_field_derivs(C.byref(om.ctx), ptr(lv), ptr(r), ptr(uu), ptr(g), ptr(c), ptr(dv), ptr(qc))
    return g, c, dv, qc


def update_buffer(buf: BufferZone, rho, q, E):
    """updateBuffer in place on FP64 arrays rho (npoin), q (npoin,3) Fortran order, E."""
    lib().oracle_update_buffer(len(rho), C.byref(buf.c), ptr(rho), ptr(q), ptr(E))


def bc_dirichlet_prim(bnd: Boundaries, rho, q, u, pr, E):
    """temporary_bc_routine_dirichlet_prim in place on the given FP64 arrays."""
    lib().oracle_bc_dirichlet_prim(len(rho), C.byref(bnd.c), ptr(rho), ptr(q), ptr(u), ptr(pr), ptr(E))


def bc_jvp(bnd: Boundaries, rho, q, E, drho, dq, dE, u=None, du=None):
    """The routine's new (rho, q, E) and its tangent along (drho, dq, dE, du) (dual numbers);
    u: the aux_u the slip branch reads (zeros when None), du its tangent (zeros when None)."""
    N = len(rho)
    z = np.zeros((N, 3), order="F")
    ins = [np.ascontiguousarray(rho, dtype=np.float64), np.asfortranarray(q, dtype=np.float64),
           z if u is None else np.asfortranarray(u, dtype=np.float64),
           np.ascontiguousarray(E, dtype=np.float64), np.ascontiguousarray(drho, dtype=np.float64),
           np.asfortranarray(dq, dtype=np.float64), np.ascontiguousarray(dE, dtype=np.float64),
           z if du is None else np.asfortranarray(du, dtype=np.float64)]
    outs = [np.zeros(N), np.zeros((N, 3), order="F"), np.zeros(N), np.zeros(N), np.zeros((N, 3), order="F"),
            np.zeros(N)]
    lib().oracle_bc_jvp(N, C.byref(bnd.c), *(ptr(a) for a in ins), *(ptr(a) for a in outs))
    return (outs[0], outs[1], outs[2]), (outs[3], outs[4], outs[5])


def bc_fix_residual(bnd: Boundaries, Rmass, Rmom, Rener):
    lib().oracle_bc_fix_dirichlet_residual(len(Rmass), C.byref(bnd.c), ptr(Rmass), ptr(Rmom), ptr(Rener))


def bc_fix_residual_entropy(bnd: Boundaries, R):
    lib().oracle_bc_fix_dirichlet_residual_entropy(len(R), C.byref(bnd.c), ptr(R))


def convec(om: OracleMesh, u, q, rho, pr, E):
    Rm = np.zeros(om.npoin); Rmo = np.zeros((om.npoin, 3), order="F"); Re = np.zeros(om.npoin)
    lib().oracle_full_convec_ijk(C.byref(om.ctx), ptr(u), ptr(q), ptr(rho), ptr(pr), ptr(E), ptr(Rm), ptr(Rmo), ptr(Re))
    return Rm, Rmo, Re


def convec_H(om: OracleMesh, u, q, rho, pr, E):
    """full_convec_ijk_H (E: total energy rho E)."""
    Rm = np.zeros(om.npoin); Rmo = np.zeros((om.npoin, 3), order="F"); Re = np.zeros(om.npoin)
    lib().oracle_full_convec_ijk_H(C.byref(om.ctx), ptr(u), ptr(q), ptr(rho), ptr(pr), ptr(E), ptr(Rm), ptr(Rmo),
                                   ptr(Re))
    return Rm, Rmo, Re


def scalar_convec(om: OracleMesh, f, eta, u):
    R = np.zeros(om.npoin)
    lib().oracle_generic_scalar_convec_ijk(C.byref(om.ctx), ptr(f), ptr(eta), ptr(u), ptr(R))
    return R


def diffusion(om: OracleMesh, prm, rho_n, rho, u, Tem, mu_fluid, mu_e, mu_sgs):
    P = params_of(prm)
    Rm = np.zeros(om.npoin); Rmo = np.zeros((om.npoin, 3), order="F"); Re = np.zeros(om.npoin)
    lib().oracle_full_diffusion_ijk(C.byref(om.ctx), C.byref(P), ptr(rho_n), ptr(rho), ptr(u), ptr(Tem),
                                    ptr(mu_fluid), ptr(mu_e), ptr(mu_sgs), ptr(Rm), ptr(Rmo), ptr(Re))
    return Rm, Rmo, Re


def smart_visc(om: OracleMesh, prm, Reta, rho, u, csound, Tem, eta, mu_e_in):
    P = params_of(prm)
    mu_e = np.array(mu_e_in, order="F", copy=True)
    mue_l = np.zeros((om.nelem, 64), order="F")
    lib().oracle_smart_visc_spectral(C.byref(om.ctx), C.byref(P), ptr(Reta), ptr(om.gpvol), ptr(om.wgp), ptr(rho),
                                     ptr(u), ptr(csound), ptr(Tem), ptr(eta), ptr(om.helem_l), ptr(om.helem),
                                     ptr(mu_e), ptr(mue_l))
    return mu_e


def laplacian_mult(om: OracleMesh, p):
    out = np.zeros(om.npoin)
    lib().oracle_eval_laplacian_mult(C.byref(om.ctx), ptr(np.ascontiguousarray(p)), ptr(out))
    return out


def laplacian_diag(om: OracleMesh):
    d = np.zeros(om.npoin)
    lib().oracle_eval_laplacian_diag(C.byref(om.ctx), ptr(om.dNgp), ptr(d))
    return d


def conjgrad_pressure(om: OracleMesh, rhs, x0=None, max_iter: int = 10000, tol: float = 1e-10):
    R = np.array(rhs, dtype=np.float64, copy=True)
    Rp0 = np.zeros(om.npoin) if x0 is None else np.ascontiguousarray(x0, dtype=np.float64)
    rel = C.c_double(0.0)
    it = lib().oracle_conjgrad_pressure(C.byref(om.ctx), ptr(om.dNgp), ptr(Rp0), ptr(R), int(max_iter),
                                        float(tol), C.byref(rel))
    return R, it, rel.value


def csr_spmv_scal(rdom, cdom, Mc, v):
    rdom = np.ascontiguousarray(rdom, np.int32); cdom = np.ascontiguousarray(cdom, np.int32)
    Mc = np.ascontiguousarray(Mc, np.float64); v = np.ascontiguousarray(v, np.float64)
    u = np.zeros(len(rdom) - 1)
    lib().oracle_csr_spmv_scal(len(u), len(Mc), ptr(rdom), ptr(cdom), ptr(Mc), ptr(v), ptr(u))
    return u


def rhs_stage(om: OracleMesh, prm, st, mu_e=None):
    """Stage RHS (mass, mom x3, energy; /Ml) without the entropy residual: (5, npoin) array."""
    P = params_of(prm)
    R = np.zeros(5 * om.npoin)
    mue = np.asfortranarray(st.mu_e if mu_e is None else mu_e)
    lib().oracle_rhs_stage(C.byref(om.ctx), C.byref(P), ptr(om.Ml), ptr(st.mu_factor), ptr(mue), None, ptr(st.rho),
                           ptr(np.asfortranarray(st.q)), ptr(st.E), ptr(R))
    return R.reshape(5, om.npoin)


def rhs_stage_ld(om: OracleMesh, prm, st, mu_e=None):
    """rhs_stage evaluated in x87 extended precision (64-bit significand), rounded to FP64:
    the reference value against which FP64 rounding is measured."""
    P = params_of(prm)
    R = np.zeros(5 * om.npoin)
    mue = np.asfortranarray(st.mu_e if mu_e is None else mu_e)
    lib().oracle_rhs_stage_ld(C.byref(om.ctx), C.byref(P), ptr(om.Ml), ptr(st.mu_factor), ptr(mue), None,
                              ptr(st.rho), ptr(np.asfortranarray(st.q)), ptr(st.E), ptr(R))
    return R.reshape(5, om.npoin)


def rhs_opcount(om: OracleMesh, prm, st, mu_e=None) -> float:
    """Arithmetic operations of one stage RHS evaluation (reference formulation, whole mesh)."""
    P = params_of(prm)
    mue = np.asfortranarray(st.mu_e if mu_e is None else mu_e)
    f = lib().oracle_rhs_opcount
    f.restype = C.c_double
    return float(f(C.byref(om.ctx), C.byref(P), ptr(om.Ml), ptr(st.mu_factor), ptr(mue), ptr(st.rho),
                   ptr(np.asfortranarray(st.q)), ptr(st.E)))


def rhs_jvp(om: OracleMesh, prm, st, drho, dq, dE, mu_e=None, mu_sgs=None, wall: "WallModel | None" = None):
    """Exact JVP of rhs_stage along (drho, dq(npoin,3), dE): returns (R, dR) as (5, npoin).
    mu_sgs (nelem,64): a frozen SGS viscosity in the diffusion (LES), None for none; wall: the
    wall model's term in the momentum residual."""
    P = params_of(prm)
    R = np.zeros(5 * om.npoin); dR = np.zeros(5 * om.npoin)
    mue = np.asfortranarray(st.mu_e if mu_e is None else mu_e)
    sgs = None if mu_sgs is None else np.asfortranarray(mu_sgs)
    lib().oracle_rhs_jvp(C.byref(om.ctx), C.byref(P), ptr(om.Ml), ptr(st.mu_factor), ptr(mue),
                         ptr(sgs) if sgs is not None else None, ptr(st.rho),
                         ptr(np.asfortranarray(st.q)), ptr(st.E), ptr(np.ascontiguousarray(drho)),
                         ptr(np.asfortranarray(dq)), ptr(np.ascontiguousarray(dE)), ptr(R), ptr(dR),
                         C.byref(wall.c) if wall is not None else None)
    return R.reshape(5, om.npoin), dR.reshape(5, om.npoin)


# ---- legacy unit-test API (generic gpcar-based element loops; 1-based connec) -------------------
def _legacy_args(connec, Ngp, gpcar, gpvol):
    connec = np.asfortranarray(connec, dtype=np.int32)
    nelem, nnode = connec.shape
    Ngp = np.asfortranarray(Ngp, dtype=np.float64)
    gpcar = np.asfortranarray(gpcar, dtype=np.float64)
    gpvol = np.asfortranarray(gpvol, dtype=np.float64)
    ndime, _, ngaus, _ = gpcar.shape
    return nelem, ngaus, nnode, ndime, connec, Ngp, gpcar, gpvol


def legacy_mass_convec(connec, Ngp, gpcar, gpvol, q):
    """mass_convec / generic_scalar_convec: R_a = sum_g gpvol N_a div q (q: (npoin, ndime))."""
    nelem, ngaus, nnode, ndime, connec, Ngp, gpcar, gpvol = _legacy_args(connec, Ngp, gpcar, gpvol)
    q = np.asfortranarray(q, dtype=np.float64)
    R = np.zeros(q.shape[0])
    lib().oracle_legacy_mass_convec(nelem, ngaus, q.shape[0], nnode, ndime, ptr(connec), ptr(Ngp), ptr(gpcar),
                                    ptr(gpvol), ptr(q), ptr(R))
    return R


def legacy_mom_convec(connec, Ngp, gpcar, gpvol, u, q, pr):
    nelem, ngaus, nnode, ndime, connec, Ngp, gpcar, gpvol = _legacy_args(connec, Ngp, gpcar, gpvol)
    u = np.asfortranarray(u, dtype=np.float64); q = np.asfortranarray(q, dtype=np.float64)
    pr = np.ascontiguousarray(pr, dtype=np.float64)
    R = np.zeros(u.shape, order="F")
    lib().oracle_legacy_mom_convec(nelem, ngaus, u.shape[0], nnode, ndime, ptr(connec), ptr(Ngp), ptr(gpcar),
                                   ptr(gpvol), ptr(u), ptr(q), ptr(pr), ptr(R))
    return R


def legacy_ener_convec(connec, Ngp, gpcar, gpvol, u, pr, E):
    nelem, ngaus, nnode, ndime, connec, Ngp, gpcar, gpvol = _legacy_args(connec, Ngp, gpcar, gpvol)
    u = np.asfortranarray(u, dtype=np.float64)
    pr = np.ascontiguousarray(pr, dtype=np.float64); E = np.ascontiguousarray(E, dtype=np.float64)
    R = np.zeros(u.shape[0])
    lib().oracle_legacy_ener_convec(nelem, ngaus, u.shape[0], nnode, ndime, ptr(connec), ptr(Ngp), ptr(gpcar),
                                    ptr(gpvol), ptr(u), ptr(pr), ptr(E), ptr(R))
    return R


def legacy_mom_diffusion(connec, Ngp, gpcar, gpvol, u, mu_e):
    nelem, ngaus, nnode, ndime, connec, Ngp, gpcar, gpvol = _legacy_args(connec, Ngp, gpcar, gpvol)
    u = np.asfortranarray(u, dtype=np.float64); mu_e = np.ascontiguousarray(mu_e, dtype=np.float64)
    R = np.zeros(u.shape, order="F")
    lib().oracle_legacy_mom_diffusion(nelem, ngaus, u.shape[0], nnode, ndime, ptr(connec), ptr(Ngp), ptr(gpcar),
                                      ptr(gpvol), ptr(u), ptr(mu_e), ptr(R))
    return R


def tgv_diagnostics(om: OracleMesh, tables, rho0: float, st, volT: float, mu_e=None):
    """(EK, eps_S, eps_D, eps_T) of volAvg_EK and visc_dissipationRate (mod_analysis.f90:10-144)."""
    L = lib()
    L.oracle_volavg_ek.restype = C.c_double
    Ngp = np.asfortranarray(tables.Ngp)
    dNgp = np.asfortranarray(tables.dNgp)
    u = np.asfortranarray(st.u)
    ek = L.oracle_volavg_ek(C.byref(om.ctx), ptr(Ngp), C.c_double(rho0), ptr(st.rho), ptr(u))
    eps = np.zeros(3)
    mue = np.asfortranarray(st.mu_e if mu_e is None else mu_e)
    L.oracle_visc_dissipation_rate(C.byref(om.ctx), ptr(dNgp), C.c_double(rho0), ptr(st.mu_fluid), ptr(mue), ptr(u),
                                   C.c_double(volT), ptr(eps))
    return float(ek), float(eps[0]), float(eps[1]), float(eps[2])
