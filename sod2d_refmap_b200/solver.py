"""Host-side mirror of the reference solver interface over the C ABI.

``Sod2dMesh`` plays the role of the reference's mesh/setup phase (CFDSolverBase_run's
evalShapeFunctions / evalJacobians / evalMass / evalCharLength, CFDSolverBase.f90:1143-1389),
``Sod2dState`` the device-resident level-2 arrays of ``rk_4_main`` (time_integ.f90:137-193),
and ``Sod2dMesh.rk_4_main`` / ``rk4_steps`` the time-loop call of CFDSolverPeriodic.f90:50-52.
Device memory comes from torch (CUDA tensors are plain device buffers here); every numeric
operation runs in libsod2d_b200.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .mesh import BoxMesh, FlowState, TGVParams, bc_params


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("sod2d_refmap_b200 needs a CUDA device (no CPU fallback)")
    return torch


def _ptr(t) -> int:
    return 0 if t is None else int(t.data_ptr())


def _contig(t):
    """t itself, after checking that it is a contiguous float64 CUDA tensor."""
    torch = _torch()
    if t.device.type != "cuda" or t.dtype != torch.float64 or not t.is_contiguous():
        raise ValueError("expected a contiguous float64 CUDA tensor")
    return t


def _np_ptr(a) -> C.c_void_p:
    # data_as keeps a reference to the array for as long as the pointer object lives
    return a.ctypes.data_as(C.c_void_p) if a is not None else C.c_void_p(0)


def _stream(stream=None) -> C.c_void_p:
    torch = _torch()
    s = stream if stream is not None else torch.cuda.current_stream()
    return C.c_void_p(int(s.cuda_stream))


def params_struct(prm: TGVParams) -> _lib.SodParams:
    return _lib.SodParams(prm.gamma_gas, prm.Rgas, prm.Cp, prm.Prt, prm.ce, prm.cmax, prm.cglob, prm.c_rho, prm.c_ener,
                          int(prm.flag_normalise_entropy), prm.cfl_conv, prm.cfl_diff, int(prm.flag_les), prm.c_sgs,
                          int(getattr(prm, "flag_total_enthalpy", 0)))


def set_wait_timeout(seconds: float):
    """Limit on the library's host waits (0 = none); past it calls raise SOD_ERR_TIMEOUT."""
    _lib.load().sod_set_wait_timeout(C.c_double(float(seconds)))


FP64 = _lib.SOD_FP64
MIXED = _lib.SOD_MIXED


class Sod2dState:
    """Device arrays of one solver state in the reference layouts (level pos=2)."""

    FIELDS = ("rho", "q", "E", "u", "pr", "Tem", "e_int", "eta", "csound", "machno", "mu_fluid", "mu_factor",
              "mu_e", "Reta", "mu_sgs")

    def __init__(self, npoin: int, nelem: int, device="cuda"):
        torch = _torch()
        f64 = dict(dtype=torch.float64, device=device)
        self.npoin, self.nelem = npoin, nelem
        # (npoin,3) Fortran arrays are stored as (3,npoin) torch tensors (same memory order)
        self.rho = torch.zeros(npoin, **f64)
        self.q = torch.zeros(3, npoin, **f64)
        self.E = torch.zeros(npoin, **f64)
        self.u = torch.zeros(3, npoin, **f64)
        self.pr = torch.zeros(npoin, **f64)
        self.Tem = torch.zeros(npoin, **f64)
        self.e_int = torch.zeros(npoin, **f64)
        self.eta = torch.zeros(npoin, **f64)
        self.csound = torch.zeros(npoin, **f64)
        self.machno = torch.zeros(npoin, **f64)
        self.mu_fluid = torch.zeros(npoin, **f64)
        self.mu_factor = torch.zeros(npoin, **f64)
        self.mu_e = torch.zeros(64, nelem, **f64)   # (nelem,64) Fortran
        self.Reta = torch.zeros(npoin, **f64)
        self.mu_sgs = torch.zeros(64, nelem, **f64)  # (nelem,64) Fortran; used when flag_les = 1
        self.dt = torch.zeros(1, **f64)

    @classmethod
    def from_host(cls, st: FlowState, nelem: int) -> "Sod2dState":
        torch = _torch()
        s = cls(len(st.rho), nelem)
        for name in ("rho", "E", "pr", "Tem", "e_int", "eta", "csound", "machno", "mu_fluid", "mu_factor"):
            getattr(s, name).copy_(torch.from_numpy(np.ascontiguousarray(getattr(st, name))))
        s.q.copy_(torch.from_numpy(np.ascontiguousarray(st.q.T)))
        s.u.copy_(torch.from_numpy(np.ascontiguousarray(st.u.T)))
        s.mu_e.copy_(torch.from_numpy(np.ascontiguousarray(st.mu_e.T)))
        s.mu_sgs.copy_(torch.from_numpy(np.ascontiguousarray(st.mu_sgs.T)))
        return s

    def struct(self) -> _lib.SodState:
        return _lib.SodState(*(_ptr(getattr(self, f)) for f in self.FIELDS))

    def to_host(self) -> dict:
        out = {}
        for f in self.FIELDS:
            t = getattr(self, f)
            a = t.detach().cpu().numpy()
            out[f] = np.asfortranarray(a.T) if t.dim() == 2 else a.copy()
        return out


class Sod2dMesh:
    """A SodMesh handle built from a BoxMesh (or any reference-layout mesh arrays)."""

    def __init__(self, mesh: BoxMesh, prm: TGVParams | None = None, geometry: dict | None = None):
        _torch()
        L = _lib.load()
        self.box = mesh
        self.prm = prm or TGVParams()
        T = mesh.tables
        self._keep = []
        def keep(a):
            self._keep.append(a)
            return _np_ptr(a)
        desc = _lib.SodMeshDesc()
        desc.nelem, desc.npoin, desc.npoin_orig, desc.porder, desc.index_base = (
            mesh.nelem, mesh.npoin, mesh.npoin_orig, 3, 0)
        desc.connec = keep(np.asfortranarray(mesh.connec, dtype=np.int32))
        desc.connec_orig = keep(np.asfortranarray(mesh.connec_orig, dtype=np.int32))
        desc.coord_orig = keep(np.asfortranarray(mesh.coord_orig, dtype=np.float64))
        desc.dlxigp_ip = keep(np.asfortranarray(T.dlxigp_ip))
        desc.wgp = keep(np.ascontiguousarray(T.wgp))
        desc.invAtoIJK = keep(np.asfortranarray(T.invAtoIJK, dtype=np.int32))
        desc.gmshAtoI = keep(np.ascontiguousarray(T.gmshAtoI, dtype=np.int32))
        desc.gmshAtoJ = keep(np.ascontiguousarray(T.gmshAtoJ, dtype=np.int32))
        desc.gmshAtoK = keep(np.ascontiguousarray(T.gmshAtoK, dtype=np.int32))
        lw = mesh.extra.get("lpoin_w") if getattr(mesh, "extra", None) else None
        if lw is not None:  # SOD2D's array form: rows outside lpoin_w are periodic slaves
            desc.npoin_w = len(lw)
            desc.lpoin_w = keep(np.ascontiguousarray(lw, dtype=np.int32))
        if geometry:
            for k in ("He", "gpvol", "Ml", "helem", "helem_l"):
                if geometry.get(k) is not None:
                    setattr(desc, k, keep(np.asfortranarray(geometry[k], dtype=np.float64)))
        p = params_struct(self.prm)
        h = C.c_void_p(0)
        _lib.check(L.sod_mesh_create(C.byref(desc), C.byref(p), C.byref(h)))
        self.handle = h
        self.nelem, self.npoin = mesh.nelem, mesh.npoin
        self._keep = []  # the library copied everything it needs

    def close(self):
        if getattr(self, "handle", None) and self.handle.value:
            _lib.load().sod_mesh_destroy(self.handle)
            self.handle = C.c_void_p(0)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def geometry(self) -> dict:
        E, N = self.nelem, self.npoin
        out = dict(He=np.zeros((3, 3, 64, E), order="F"), gpvol=np.zeros((1, 64, E), order="F"), Ml=np.zeros(N),
                   helem=np.zeros(E), helem_l=np.zeros((E, 64), order="F"))
        _lib.check(_lib.load().sod_mesh_get_geometry(self.handle, *(_np_ptr(out[k]) for k in
                                                                    ("He", "gpvol", "Ml", "helem", "helem_l"))))
        return out

    def set_params(self, prm: TGVParams):
        self.prm = prm
        p = params_struct(prm)
        _lib.check(_lib.load().sod_mesh_set_params(self.handle, C.byref(p)))

    def check_finite(self, stream=None):
        """Raises SodError(SOD_ERR_NONFINITE) when a step since the last check produced a NaN/Inf
        in rho, q or E (waits for the stream's work; clears the flag)."""
        _lib.check(_lib.load().sod_check_finite(self.handle, _stream(stream)))

    # ---- boundary conditions (non-periodic meshes) -------------------------------------
    def set_boundaries(self, bou_codes_nodes, lnbn_nodes, normals, u_buffer=None, bc: dict | None = None):
        """Registers rk_4_main's boundary data (host numpy arrays, 0-based node ids): the step
        then applies the boundary routines (noBoundaries = .false.).  bou_codes_nodes=None
        removes them.  bc: the nscbc_* values (mesh.bc_params)."""
        L = _lib.load()
        if bou_codes_nodes is None:
            _lib.check(L.sod_mesh_set_boundaries(self.handle, None, None, None, None, None))
            self._bnd = None
            return
        if bc is None:
            bc = bc_params(self.prm)
        arrs = (np.ascontiguousarray(bou_codes_nodes, dtype=np.int32), np.ascontiguousarray(lnbn_nodes, dtype=np.int32),
                np.asfortranarray(normals, dtype=np.float64),
                None if u_buffer is None else np.asfortranarray(u_buffer, dtype=np.float64))
        p = _lib.SodBcParams(*(float(bc[k]) for k in ("rho_inf", "u_inf", "p_inf", "c_inf", "gamma_inf", "Rgas_inf",
                                                      "T_H", "T_C")))
        _lib.check(L.sod_mesh_set_boundaries(self.handle, *(_np_ptr(a) if a is not None else None for a in arrs),
                                             C.byref(p)))
        self._bnd = arrs

    def set_buffer(self, prm: dict | None, coord=None, u_buffer=None):
        """Registers the buffer zone of rk_4_main (flag_buffer_on = .true.): prm is the flat dict
        of mesh.buffer_params, coord (npoin,3) and u_buffer (npoin,3) host arrays (u_buffer None:
        zeros).  prm=None removes it."""
        L = _lib.load()
        if prm is None:
            _lib.check(L.sod_mesh_set_buffer(self.handle, None, None, None))
            return
        sides = ("east", "west", "north", "south", "top", "bottom")
        p = _lib.SodBufferParams(*(int(prm["on_" + s]) for s in sides),
                                 *(float(prm[s + k]) for s in "ewnstb" for k in ("_min", "_size")),
                                 *(float(prm[k]) for k in ("rho_inf", "u_inf", "p_inf", "gamma_inf")))
        c = np.asfortranarray(coord, dtype=np.float64)
        ub = None if u_buffer is None else np.asfortranarray(u_buffer, dtype=np.float64)
        _lib.check(L.sod_mesh_set_buffer(self.handle, C.byref(p), _np_ptr(c), _np_ptr(ub) if ub is not None else None))

    def set_source_term(self, source):
        """The source_term of rk_4_main (mom_source_const_vect): a device tensor (3, npoin) =
        Fortran (npoin,3) that the mesh keeps (and this object references) until replaced;
        None removes it."""
        if source is None:
            _lib.check(_lib.load().sod_mesh_set_source_term(self.handle, None))
            self._source = None
            return
        src = _contig(source)
        _lib.check(_lib.load().sod_mesh_set_source_term(self.handle, C.c_void_p(_ptr(src))))
        self._source = src

    def set_wall_model(self, wtype: int, bound, bounorm, wgp_b, list_wm, point2elem, coord, normals, zo=None,
                       walave_u=None):
        """Registers the wall model (isWallModelOn): wtype 1 Reichardt, 2 ABL; host arrays with
        0-based ids (mesh.wall_faces); list_wm the wall-model faces; walave_u a device tensor
        (3, npoin) kept by the mesh, or None.  list_wm empty/None removes it."""
        L = _lib.load()
        if list_wm is None or len(list_wm) == 0:
            _lib.check(L.sod_mesh_set_wall_model(self.handle, 1, 0, 0, *([None] * 3), 0, *([None] * 6)))
            self._walave = None
            return
        b = np.asfortranarray(bound, dtype=np.int32)
        bn = np.asfortranarray(bounorm, dtype=np.float64)
        wg = np.ascontiguousarray(wgp_b, dtype=np.float64)
        lw = np.ascontiguousarray(list_wm, dtype=np.int32)
        pe = np.ascontiguousarray(point2elem, dtype=np.int32)
        co = np.asfortranarray(coord, dtype=np.float64)
        nr = np.asfortranarray(normals, dtype=np.float64)
        z = None if zo is None else np.ascontiguousarray(zo, dtype=np.float64)
        wa = None if walave_u is None else _contig(walave_u)
        _lib.check(L.sod_mesh_set_wall_model(
            self.handle, int(wtype), b.shape[0], b.shape[1], _np_ptr(b), _np_ptr(bn), _np_ptr(wg), len(lw),
            _np_ptr(lw), _np_ptr(pe), _np_ptr(co), _np_ptr(nr), _np_ptr(z) if z is not None else None,
            C.c_void_p(_ptr(wa)) if wa is not None else None))
        self._walave = wa

    def wall_model(self, rho, u, mu_fluid, Rdiff, tauw=None, stream=None):
        """The registered wall model as the reference routine: Rdiff (3, npoin) += the wall terms."""
        _lib.check(_lib.load().sod_wall_model(self.handle, *(C.c_void_p(_ptr(_contig(t))) for t in (
            rho, u, mu_fluid, Rdiff)), C.c_void_p(_ptr(tauw)) if tauw is not None else None, _stream(stream)))

    def wall_model_tauw(self, stream=None):
        torch = _torch()
        t = torch.empty(3, self.npoin, dtype=torch.float64, device="cuda")
        _lib.check(_lib.load().sod_wall_model_tauw(self.handle, C.c_void_p(_ptr(t)), _stream(stream)))
        return t

    def update_buffer(self, rho, q, E, stream=None):
        """updateBuffer in place on device tensors rho (npoin), q (3,npoin) storage = Fortran
        (npoin,3), E (npoin)."""
        _lib.check(_lib.load().sod_update_buffer(self.handle, *(C.c_void_p(_ptr(_contig(t))) for t in (rho, q, E)),
                                                 _stream(stream)))

    def bc_dirichlet_prim(self, rho, q, u, pr, E, stream=None):
        """temporary_bc_routine_dirichlet_prim in place on device tensors ((npoin), q/u (3,npoin)
        storage = Fortran (npoin,3))."""
        _lib.check(_lib.load().sod_bc_dirichlet_prim(self.handle, *(C.c_void_p(_ptr(_contig(t))) for t in (
            rho, q, u, pr, E)), _stream(stream)))

    def bc_dirichlet_prim_vjp(self, rho, q, E, bar_rho, bar_q, bar_E, stream=None):
        """Adjoint of temporary_bc_routine_dirichlet_prim in place on (bar_rho, bar_q (3,npoin),
        bar_E); (rho, q, E) the state the routine read."""
        _lib.check(_lib.load().sod_bc_dirichlet_prim_vjp(self.handle, *(C.c_void_p(_ptr(_contig(t))) for t in (
            rho, q, E, bar_rho, bar_q, bar_E)), _stream(stream)))

    def bc_fix_residual(self, Rmass, Rmom, Rener, stream=None):
        _lib.check(_lib.load().sod_bc_fix_dirichlet_residual(self.handle, *(C.c_void_p(_ptr(_contig(t))) for t in (
            Rmass, Rmom, Rener)), _stream(stream)))

    def bc_fix_residual_entropy(self, R, stream=None):
        _lib.check(_lib.load().sod_bc_fix_dirichlet_residual_entropy(self.handle, C.c_void_p(_ptr(_contig(R))),
                                                                      _stream(stream)))

    # ---- time integration --------------------------------------------------------------
    def rk_4_main(self, state: Sod2dState, precision: int = FP64, update_dt: bool = True, stream=None):
        st = state.struct()
        _lib.check(_lib.load().sod_rk4_main(self.handle, C.byref(st), C.c_void_p(_ptr(state.dt)),
                                           C.c_void_p(_ptr(state.dt) if update_dt else 0), int(precision),
                                           _stream(stream)))

    def rk4_steps(self, state: Sod2dState, nsteps: int, precision: int = FP64, stream=None):
        st = state.struct()
        _lib.check(_lib.load().sod_rk4_steps(self.handle, C.byref(st), C.c_void_p(_ptr(state.dt)), int(nsteps),
                                            int(precision), _stream(stream)))

    def step_profile(self, state: Sod2dState, nsteps: int, precision: int = FP64, stream=None):
        """Mean ms per launch of (fused RHS, gather/RK stage, entropy viscosity + dt)."""
        ms = (C.c_float * 3)()
        st = state.struct()
        _lib.check(_lib.load().sod_step_profile(self.handle, C.byref(st), C.c_void_p(_ptr(state.dt)), int(nsteps),
                                               int(precision), _stream(stream), ms))
        return tuple(float(x) for x in ms)

    def rk4_main_host(self, host: dict, dt: float, precision: int = FP64, stream=None) -> float:
        """sod_rk4_main_host on host arrays (numpy, reference layouts; pinned for speed)."""
        st = _lib.SodState(*(int(host[f].ctypes.data) if host.get(f) is not None else 0 for f in Sod2dState.FIELDS))
        dtn = C.c_double(0.0)
        _lib.check(_lib.load().sod_rk4_main_host(self.handle, C.byref(st), C.c_double(dt), C.byref(dtn),
                                                int(precision), _stream(stream)))
        return dtn.value

    def autotune(self, state: Sod2dState, precision: int = FP64, stream=None):
        """Pick elements per CTA and the stage launch shape by timing the candidates; returns
        (elements per CTA, fastest fused-RHS ms)."""
        best = C.c_int(0); ms = C.c_float(0.0)
        st = state.struct()
        _lib.check(_lib.load().sod_autotune(self.handle, C.byref(st), int(precision), C.byref(best), C.byref(ms),
                                           _stream(stream)))
        return best.value, ms.value

    def autotune_table(self, precision: int = FP64):
        """The last autotuner sweep: [(elements per CTA, CTAs per SM of the one-launch stage or 0 for
        two launches, ms per stage)]."""
        cap = 64
        e = (C.c_int32 * cap)(); c = (C.c_int32 * cap)(); t = (C.c_float * cap)()
        n = _lib.load().sod_autotune_table(self.handle, int(precision), cap, e, c, t)
        if n < 0:
            _lib.check(n)
        return [(int(e[q]), int(c[q]), float(t[q])) for q in range(min(n, cap))]

    def set_stage_launch(self, precision: int, ctas_per_sm: int):
        """0: two launches per RK stage; n > 0: one cooperative launch with n CTAs per SM."""
        _lib.check(_lib.load().sod_set_stage_launch(self.handle, int(precision), int(ctas_per_sm)))

    def compute_field_derivs(self, rho, u, leviCivi=None, stream=None):
        """compute_fieldDerivs on device tensors rho (npoin) and u (3, npoin) = Fortran (npoin,3):
        returns (gradRho (3,npoin), curlU (3,npoin), divU, Qcrit).  leviCivi: (3,3,3) array
        or None for the reference's symbol."""
        torch = _torch()
        N = self.npoin
        g = torch.empty(3, N, dtype=torch.float64, device="cuda")
        c = torch.empty(3, N, dtype=torch.float64, device="cuda")
        dv = torch.empty(N, dtype=torch.float64, device="cuda")
        qc = torch.empty(N, dtype=torch.float64, device="cuda")
        lv = None if leviCivi is None else np.asfortranarray(leviCivi, dtype=np.float64).ravel(order="F")
        _lib.check(_lib.load().sod_compute_field_derivs(
            self.handle, C.c_void_p(_ptr(_contig(rho))), C.c_void_p(_ptr(_contig(u))),
            _np_ptr(lv) if lv is not None else None, *(C.c_void_p(_ptr(t)) for t in (g, c, dv, qc)), _stream(stream)))
        return g, c, dv, qc

    def set_rhs_config(self, precision: int, config: int):
        """Pins the fused-RHS configuration of a precision (sod_set_rhs_config)."""
        _lib.check(_lib.load().sod_set_rhs_config(self.handle, int(precision), int(config)))

    def rhs(self, state: Sod2dState, precision: int = FP64, stream=None):
        torch = _torch()
        N = self.npoin
        out = dict(Rmass=torch.zeros(N, dtype=torch.float64, device="cuda"),
                   Rmom=torch.zeros(3, N, dtype=torch.float64, device="cuda"),
                   Rener=torch.zeros(N, dtype=torch.float64, device="cuda"),
                   Reta=torch.zeros(N, dtype=torch.float64, device="cuda"))
        _lib.check(_lib.load().sod_rhs(self.handle, *(C.c_void_p(_ptr(t)) for t in (
            state.rho, state.q, state.E, state.mu_e, state.mu_factor, out["Rmass"], out["Rmom"], out["Rener"],
            out["Reta"])), int(precision), _stream(stream)))
        return out

    def tgv_diagnostics(self, state: Sod2dState, rho0: float, volT: float = 0.0, stream=None) -> dict:
        """volAvg_EK / visc_dissipationRate of the state: EK, eps_S, eps_D, eps_T (volT <= 0:
        the summed gpvol)."""
        torch = _torch()
        out = torch.zeros(5, dtype=torch.float64, device="cuda")
        _lib.check(_lib.load().sod_tgv_diagnostics(self.handle, *(C.c_void_p(_ptr(t)) for t in (
            state.rho, state.u, state.mu_fluid, state.mu_e)), C.c_double(rho0), C.c_double(volT),
            C.c_void_p(_ptr(out)), _stream(stream)))
        v = out.cpu().tolist()
        return {"EK": v[0], "eps_S": v[1], "eps_D": v[2], "eps_T": v[3], "volT": v[4]}

    # ---- adjoint (reverse mode, FP64, mu_e and dt frozen) --------------------------------
    def rhs_vjp(self, rho, q, E, mu_e, mu_factor, bar_Rmass, bar_Rmom, bar_Rener, stream=None):
        """(dR/d(rho,q,E))^T (bar_Rmass, bar_Rmom, bar_Rener) for the FP64 stage RHS of rhs()."""
        torch = _torch()
        N = self.npoin
        g_rho = torch.empty(N, dtype=torch.float64, device="cuda")
        g_q = torch.empty(3, N, dtype=torch.float64, device="cuda")
        g_E = torch.empty(N, dtype=torch.float64, device="cuda")
        args = [_contig(t) for t in (rho, q, E, mu_e, mu_factor, bar_Rmass, bar_Rmom, bar_Rener)]
        _lib.check(_lib.load().sod_rhs_vjp(self.handle, *(C.c_void_p(_ptr(t)) for t in args + [g_rho, g_q, g_E]),
                                           _stream(stream)))
        return g_rho, g_q, g_E

    def rk_4_main_record(self, state: Sod2dState, stages, update_dt: bool = True, precision: int = FP64,
                         stream=None):
        """rk_4_main that also stores the stage states Y2..Y4 in stages (15*npoin float64)."""
        st = state.struct()
        _lib.check(_lib.load().sod_rk4_main_record(self.handle, C.byref(st), C.c_void_p(_ptr(state.dt)),
                                                  C.c_void_p(_ptr(state.dt) if update_dt else 0),
                                                  C.c_void_p(_ptr(_contig(stages))), int(precision),
                                                  _stream(stream)))

    def rk4_step_vjp(self, rho, q, E, mu_e, mu_factor, dt, bar_rho, bar_q, bar_E, out=None, stages=None,
                     mu_sgs=None, stream=None):
        """Adjoint of one FP64 RK4 step from (rho, q, E) with mu_e, mu_sgs (LES, or None) and dt
        (device (1,)) frozen; stages from rk_4_main_record of the same step (recomputed when None)."""
        torch = _torch()
        N = self.npoin
        if out is None:
            out = (torch.empty(N, dtype=torch.float64, device="cuda"),
                   torch.empty(3, N, dtype=torch.float64, device="cuda"),
                   torch.empty(N, dtype=torch.float64, device="cuda"))
        args = [_contig(t) for t in (rho, q, E, mu_e)]
        args += [None if mu_sgs is None else _contig(mu_sgs)]
        args += [_contig(t) for t in (mu_factor, dt)]
        args += [None if stages is None else _contig(stages)]
        args += [_contig(t) for t in (bar_rho, bar_q, bar_E)]
        _lib.check(_lib.load().sod_rk4_step_vjp(self.handle, *(C.c_void_p(_ptr(t)) for t in args + list(out)),
                                                _stream(stream)))
        return out

    def adapt_dt(self, state: Sod2dState, stream=None):
        _lib.check(_lib.load().sod_adapt_dt_cfl(self.handle, *(C.c_void_p(_ptr(t)) for t in (
            state.u, state.csound, state.mu_fluid)), C.c_void_p(0), C.c_void_p(_ptr(state.rho)),
            C.c_void_p(_ptr(state.dt)), _stream(stream)))
        return state.dt

    # ---- per-routine entry points (reference argument lists) ----------------------------
    def full_convec_ijk(self, u, q, rho, pr, E, stream=None):
        torch = _torch()
        N = self.npoin
        Rm = torch.empty(N, dtype=torch.float64, device="cuda")
        Rmo = torch.empty(3, N, dtype=torch.float64, device="cuda")
        Re = torch.empty(N, dtype=torch.float64, device="cuda")
        _lib.check(_lib.load().sod_full_convec_ijk(self.handle, *(C.c_void_p(_ptr(t)) for t in (
            u, q, rho, pr, E, Rm, Rmo, Re)), _stream(stream)))
        return Rm, Rmo, Re

    def full_convec_ijk_H(self, u, q, rho, pr, E, stream=None):
        """full_convec_ijk_H: E is the total energy rho E."""
        torch = _torch()
        N = self.npoin
        Rm = torch.empty(N, dtype=torch.float64, device="cuda")
        Rmo = torch.empty(3, N, dtype=torch.float64, device="cuda")
        Re = torch.empty(N, dtype=torch.float64, device="cuda")
        _lib.check(_lib.load().sod_full_convec_ijk_H(self.handle, *(C.c_void_p(_ptr(t)) for t in (
            u, q, rho, pr, E, Rm, Rmo, Re)), _stream(stream)))
        return Rm, Rmo, Re

    def generic_scalar_convec_ijk(self, f, eta, u, stream=None):
        torch = _torch()
        R = torch.empty(self.npoin, dtype=torch.float64, device="cuda")
        _lib.check(_lib.load().sod_generic_scalar_convec_ijk(self.handle, *(C.c_void_p(_ptr(t)) for t in (
            f, eta, u, R)), _stream(stream)))
        return R

    def full_diffusion_ijk(self, rho_n, rho, u, Tem, mu_fluid, mu_e, mu_sgs=None, stream=None):
        torch = _torch()
        N = self.npoin
        Rm = torch.empty(N, dtype=torch.float64, device="cuda")
        Rmo = torch.empty(3, N, dtype=torch.float64, device="cuda")
        Re = torch.empty(N, dtype=torch.float64, device="cuda")
        _lib.check(_lib.load().sod_full_diffusion_ijk(self.handle, C.c_double(self.prm.Cp), C.c_double(self.prm.Prt),
                                                     *(C.c_void_p(_ptr(t)) for t in (rho_n, rho, u, Tem, mu_fluid,
                                                                                     mu_e, mu_sgs, Rm, Rmo, Re)),
                                                     _stream(stream)))
        return Rm, Rmo, Re

    def lumped_solver(self, R, stream=None):
        ncomp = 3 if R.dim() == 2 else 1
        _lib.check(_lib.load().sod_lumped_solver(self.handle, C.c_void_p(_ptr(R)), ncomp, _stream(stream)))
        return R

    def smart_visc_spectral(self, Reta, rho, u, csound, Tem, eta, stream=None):
        torch = _torch()
        mu_e = torch.zeros(64, self.nelem, dtype=torch.float64, device="cuda")
        _lib.check(_lib.load().sod_smart_visc_spectral(self.handle, *(C.c_void_p(_ptr(t)) for t in (
            Reta, rho, u, csound, Tem, eta, mu_e)), _stream(stream)))
        return mu_e


def sutherland_viscosity(Tem, mu_factor, stream=None):
    torch = _torch()
    mu = torch.empty_like(Tem)
    _lib.check(_lib.load().sod_sutherland_viscosity(int(Tem.numel()), C.c_void_p(_ptr(Tem)), C.c_void_p(_ptr(mu_factor)),
                                                   C.c_void_p(_ptr(mu)), _stream(stream)))
    return mu


def csr_spmv_scal(rdom, cdom, Mc, v, stream=None):
    torch = _torch()
    u = torch.empty(rdom.numel() - 1, dtype=torch.float64, device="cuda")
    _lib.check(_lib.load().sod_csr_spmv_scal(int(u.numel()), int(Mc.numel()), *(C.c_void_p(_ptr(t)) for t in (
        rdom, cdom, Mc, v, u)), _stream(stream)))
    return u


class Sod2dPoisson:
    """Pressure-Poisson operator and PCG of lib_sod2d_incomp over the C ABI
    (eval_laplacian_mult / eval_laplacian_diag / conjGrad_pressure_incomp)."""

    def __init__(self, mesh: "Sod2dMesh"):
        _torch()
        h = C.c_void_p(0)
        _lib.check(_lib.load().sod_poisson_create(mesh.handle, C.byref(h)))
        self.handle = h
        self.n = mesh.npoin
        self.nelem = mesh.nelem
        self._mesh = mesh  # the handle points into the mesh

    def close(self):
        if getattr(self, "handle", None) and self.handle.value:
            _lib.load().sod_poisson_destroy(self.handle)
            self.handle = C.c_void_p(0)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def apply(self, x, stream=None):
        torch = _torch()
        y = torch.empty_like(x)
        _lib.check(_lib.load().sod_poisson_apply(self.handle, C.c_void_p(_ptr(x)), C.c_void_p(_ptr(y)), _stream(stream)))
        return y

    def diag(self, stream=None):
        torch = _torch()
        d = torch.empty(self.n, dtype=torch.float64, device="cuda")
        _lib.check(_lib.load().sod_poisson_diag(self.handle, C.c_void_p(_ptr(d)), _stream(stream)))
        return d

    def solve(self, rhs, x0=None, max_iter: int = 100000, tol: float = 1e-10, mixed: bool = False, stream=None):
        """conjGrad_pressure_incomp: returns (x0 + x, iterations, final relative residual)."""
        torch = _torch()
        R = rhs.clone()
        Rp0 = torch.zeros_like(rhs) if x0 is None else x0
        it = C.c_int(0); rel = C.c_double(0.0)
        _lib.check(_lib.load().sod_conjgrad_pressure(self.handle, C.c_void_p(_ptr(Rp0)), C.c_void_p(_ptr(R)),
                                                    int(max_iter), C.c_double(tol), int(bool(mixed)), C.byref(it),
                                                    C.byref(rel), _stream(stream)))
        return R, it.value, rel.value


class Sod2dBatch:
    """Ensemble of independent periodic meshes advanced together (one launch per RK stage)."""

    def __init__(self, meshes: list, states: list, prm: TGVParams | None = None):
        _torch()
        L = _lib.load()
        self.prm = prm or TGVParams()
        members = [Sod2dMesh(m, self.prm) for m in meshes]
        arr = (C.c_void_p * len(members))(*[mm.handle.value for mm in members])
        h = C.c_void_p(0)
        _lib.check(L.sod_batch_create(arr, len(members), C.byref(h)))
        self.handle = h
        self.sizes = [(m.npoin, m.nelem) for m in meshes]
        for mm in members:
            mm.close()
        for i, st in enumerate(states):
            self.set_member(i, st)

    def close(self):
        if getattr(self, "handle", None) and self.handle.value:
            _lib.load().sod_batch_destroy(self.handle)
            self.handle = C.c_void_p(0)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def _host_struct(d: dict) -> _lib.SodState:
        return _lib.SodState(*(int(d[f].ctypes.data) if d.get(f) is not None else 0 for f in Sod2dState.FIELDS))

    def set_member(self, i: int, st: FlowState):
        d = {f: np.asfortranarray(getattr(st, f)) for f in ("rho", "q", "E", "u", "csound", "mu_fluid", "mu_factor",
                                                             "mu_e")}
        _lib.check(_lib.load().sod_batch_set_member(self.handle, int(i), C.byref(self._host_struct(d))))

    def get_member(self, i: int) -> dict:
        N, E = self.sizes[i]
        d = {f: np.zeros(N) for f in ("rho", "E", "pr", "Tem", "e_int", "eta", "csound", "machno", "mu_fluid",
                                      "Reta")}
        d["q"] = np.zeros((N, 3), order="F"); d["u"] = np.zeros((N, 3), order="F")
        d["mu_e"] = np.zeros((E, 64), order="F")
        _lib.check(_lib.load().sod_batch_get_member(self.handle, int(i), C.byref(self._host_struct(d))))
        return d

    def adapt_dt(self, stream=None):
        _lib.check(_lib.load().sod_batch_adapt_dt(self.handle, _stream(stream)))

    def dt(self) -> np.ndarray:
        out = np.zeros(len(self.sizes))
        _lib.check(_lib.load().sod_batch_get_dt(self.handle, C.c_void_p(out.ctypes.data)))
        return out

    def set_dt(self, dt):
        a = np.ascontiguousarray(dt, dtype=np.float64)
        _lib.check(_lib.load().sod_batch_set_dt(self.handle, C.c_void_p(a.ctypes.data)))

    def rk4_steps(self, nsteps: int, precision: int = FP64, stream=None):
        _lib.check(_lib.load().sod_batch_rk4_steps(self.handle, int(nsteps), int(precision), _stream(stream)))

    def autotune(self, precision: int = FP64, stream=None):
        """Tune elements per CTA and the stage launch shape on the concatenated ensemble mesh."""
        best = C.c_int(0); ms = C.c_float(0.0)
        _lib.check(_lib.load().sod_batch_autotune(self.handle, int(precision), C.byref(best), C.byref(ms),
                                                 _stream(stream)))
        return best.value, ms.value

    def _mesh(self) -> C.c_void_p:
        h = C.c_void_p(0)
        _lib.check(_lib.load().sod_batch_mesh(self.handle, C.byref(h)))
        return h

    def autotune_table(self, precision: int = FP64):
        """The last autotuner sweep of the ensemble: [(elements per CTA, CTAs per SM or 0, ms per stage)]."""
        cap = 64
        e = (C.c_int32 * cap)(); c = (C.c_int32 * cap)(); t = (C.c_float * cap)()
        n = _lib.load().sod_autotune_table(self._mesh(), int(precision), cap, e, c, t)
        if n < 0:
            _lib.check(n)
        return [(int(e[q]), int(c[q]), float(t[q])) for q in range(min(n, cap))]

    def set_stage_launch(self, precision: int, ctas_per_sm: int):
        """0: two launches per RK stage; n > 0: one cooperative launch with n CTAs per SM."""
        _lib.check(_lib.load().sod_set_stage_launch(self._mesh(), int(precision), int(ctas_per_sm)))

    def set_rhs_config(self, precision: int, config: int):
        _lib.check(_lib.load().sod_set_rhs_config(self._mesh(), int(precision), int(config)))


# ---- legacy element-loop API of the unit tests (host numpy in, host numpy out) ----------------
def _legacy_call(fn_name: str, connec, Ngp, gpcar, gpvol, fields, out_shape):
    torch = _torch()
    connec = np.asfortranarray(connec, dtype=np.int32)
    nelem, nnode = connec.shape
    gpcar = np.asfortranarray(gpcar, dtype=np.float64)
    ndime, _, ngaus, _ = gpcar.shape
    dev = lambda a, dt=np.float64: torch.from_numpy(np.ascontiguousarray(np.asarray(a, dtype=dt).ravel(order="F"))).cuda()
    args = [dev(connec, np.int32), dev(Ngp), dev(gpcar), dev(gpvol)] + [dev(f) for f in fields]
    npoin = out_shape[0]
    R = torch.zeros(int(np.prod(out_shape)), dtype=torch.float64, device="cuda")
    _lib.check(getattr(_lib.load(), fn_name)(nelem, ngaus, npoin, nnode, ndime,
                                             *(C.c_void_p(_ptr(t)) for t in args + [R]), _stream(None)))
    return R.cpu().numpy().reshape(out_shape, order="F")


def legacy_mass_convec(connec, Ngp, gpcar, gpvol, q):
    """mass_convec of the unit tests: R_a = sum_g gpvol N_a div q; q (npoin, ndime)."""
    return _legacy_call("sod_legacy_mass_convec", connec, Ngp, gpcar, gpvol, [q], (np.shape(q)[0],))


def legacy_generic_scalar_convec(connec, Ngp, gpcar, gpvol, q):
    return _legacy_call("sod_legacy_generic_scalar_convec", connec, Ngp, gpcar, gpvol, [q], (np.shape(q)[0],))


def legacy_mom_convec(connec, Ngp, gpcar, gpvol, u, q, pr):
    return _legacy_call("sod_legacy_mom_convec", connec, Ngp, gpcar, gpvol, [u, q, pr], np.shape(u))


def legacy_ener_convec(connec, Ngp, gpcar, gpvol, u, pr, E):
    return _legacy_call("sod_legacy_ener_convec", connec, Ngp, gpcar, gpvol, [u, pr, E], (np.shape(u)[0],))


def legacy_mom_diffusion(connec, Ngp, gpcar, gpvol, u, mu_e):
    return _legacy_call("sod_legacy_mom_diffusion", connec, Ngp, gpcar, gpvol, [u, mu_e], np.shape(u))


# ---- the reference's subroutines with their complete argument lists (device arrays) ----------
def _ptrs(*ts):
    return [C.c_void_p(_ptr(t)) for t in ts]


def full_convec_ijk_ref(nelem, npoin, connec, Ngp, dNgp, He, gpvol, dlxigp_ip, xgp, invAtoIJK, gmshAtoI, gmshAtoJ,
                        gmshAtoK, u, q, rho, pr, E, index_base: int = 1, total_enthalpy: bool = False, stream=None):
    """full_convec_ijk (elem_convec.f90:211-224) or, with total_enthalpy, full_convec_ijk_H
    (:20-33), called as the reference calls it: every argument a CUDA tensor holding the Fortran
    array's memory (connec (nelem,64) column-major, ids index_base-based; u, q (npoin,3) ...).
    Returns (Rmass, Rmom, Rener) with Rmom in (npoin,3) memory order."""
    torch = _torch()
    f64 = dict(dtype=torch.float64, device="cuda")
    Rm, Rmo, Re = torch.empty(npoin, **f64), torch.empty(3 * npoin, **f64), torch.empty(npoin, **f64)
    fn = _lib.load().sod_full_convec_ijk_H_ref if total_enthalpy else _lib.load().sod_full_convec_ijk_ref
    _lib.check(fn(int(nelem), int(npoin), int(index_base), *_ptrs(connec, Ngp, dNgp, He, gpvol, dlxigp_ip, xgp,
                                                                   invAtoIJK, gmshAtoI, gmshAtoJ, gmshAtoK, u, q, rho,
                                                                   pr, E, Rm, Rmo, Re), _stream(stream)))
    return Rm, Rmo, Re


def generic_scalar_convec_ijk_ref(nelem, npoin, connec, Ngp, dNgp, He, gpvol, dlxigp_ip, xgp, invAtoIJK, gmshAtoI,
                                  gmshAtoJ, gmshAtoK, q, eta, u, index_base: int = 1, stream=None):
    """generic_scalar_convec_ijk (elem_convec.f90:462-476) with its argument list; returns Rconvec."""
    torch = _torch()
    R = torch.empty(npoin, dtype=torch.float64, device="cuda")
    _lib.check(_lib.load().sod_generic_scalar_convec_ijk_ref(
        int(nelem), int(npoin), int(index_base), *_ptrs(connec, Ngp, dNgp, He, gpvol, dlxigp_ip, xgp, invAtoIJK,
                                                        gmshAtoI, gmshAtoJ, gmshAtoK, q, eta, u, R), _stream(stream)))
    return R


def full_diffusion_ijk_ref(nelem, npoin, connec, Ngp, He, gpvol, dlxigp_ip, invAtoIJK, gmshAtoI, gmshAtoJ, gmshAtoK,
                           Cp, Pr, rho_n, rho, u, Tem, mu_fluid, mu_e, mu_sgs, Ml, index_base: int = 1, stream=None):
    """full_diffusion_ijk (elem_diffu.f90:12-25) with its argument list; returns (Rmass, Rmom, Rener)."""
    torch = _torch()
    f64 = dict(dtype=torch.float64, device="cuda")
    Rm, Rmo, Re = torch.empty(npoin, **f64), torch.empty(3 * npoin, **f64), torch.empty(npoin, **f64)
    L = _lib.load()
    _lib.check(L.sod_full_diffusion_ijk_ref(
        int(nelem), int(npoin), int(index_base), *_ptrs(connec, Ngp, He, gpvol, dlxigp_ip, invAtoIJK, gmshAtoI,
                                                        gmshAtoJ, gmshAtoK), C.c_double(Cp), C.c_double(Pr),
        *_ptrs(rho_n, rho, u, Tem, mu_fluid, mu_e, mu_sgs, Ml, Rm, Rmo, Re), _stream(stream)))
    return Rm, Rmo, Re


def smart_visc_spectral_ref(nelem, npoin, npoin_w, connec, lpoin_w, Reta, Ngp, coord, dNgp, gpvol, wgp, gamma_gas,
                            rho, u, csound, Tem, eta, helem_l, helem, Ml, invAtoIJK, gmshAtoI, gmshAtoJ, gmshAtoK,
                            prm: TGVParams | None = None, index_base: int = 1, stream=None):
    """smart_visc_spectral (mod_entropy_viscosity.f90:14-28) with its argument list (helem_l is
    the dummy named helem, helem the one named helem_k); prm gives the mod_numerical_params
    values and nscbc_Rgas_inf.  Returns mu_e in (nelem,64) memory order."""
    torch = _torch()
    mu_e = torch.empty(64 * nelem, dtype=torch.float64, device="cuda")
    p = params_struct(prm or TGVParams())
    _lib.check(_lib.load().sod_smart_visc_spectral_ref(
        int(nelem), int(npoin), int(npoin_w), int(index_base), *_ptrs(connec, lpoin_w, Reta, Ngp, coord, dNgp, gpvol,
                                                                      wgp), C.c_double(gamma_gas),
        *_ptrs(rho, u, csound, Tem, eta, helem_l, helem, Ml, mu_e, invAtoIJK, gmshAtoI, gmshAtoJ, gmshAtoK),
        C.c_void_p(0), C.byref(p), _stream(stream)))
    return mu_e
