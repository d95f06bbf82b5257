"""The oracle's boundary routines (mod_bc_routines.f90) against an independent numpy
restatement and the wall invariants, and the channel mesh's boundary arrays (no GPU)."""
import numpy as np
import pytest

from sod2d_refmap_b200 import mesh as M

CODES = (M.BC_FAR_FIELD, M.BC_OUTLET_INCOMP, M.BC_NON_SLIP_ADIABATIC, M.BC_NON_SLIP_HOT, M.BC_NON_SLIP_COLD,
         M.BC_SLIP_ADIABATIC, M.BC_SLIP_WALL_MODEL, M.BC_TOP_ABL)


def random_case(seed=3, n=2):
    """A channel mesh with every code drawn per boundary node, a perturbed state, and lnbn
    redirected to other boundary nodes for a few of them (the routine's copy-first order)."""
    rng = np.random.default_rng(seed)
    m = M.channel_box(n, jitter=0.05, seed=seed)
    prm = M.TGVParams()
    st = M.taylor_green_state(m, prm, pert_amp=5e-2, seed=seed)
    codes = m.extra["bou_codes_nodes"].copy()
    bnd = np.flatnonzero(codes < M.MAX_NUM_BOU_CODES)
    codes[bnd] = rng.choice(CODES, size=bnd.size)
    lnbn = m.extra["lnbn_nodes"].copy()
    redirect = rng.choice(bnd, size=8, replace=False)
    lnbn[redirect] = rng.choice(bnd, size=8)
    nrm = rng.standard_normal((m.npoin, 3))
    nrm /= np.linalg.norm(nrm, axis=1)[:, None]
    ub = np.asfortranarray(rng.uniform(-1.0, 1.0, (m.npoin, 3)))
    u_old = np.asfortranarray(st.u + rng.uniform(-0.1, 0.1, (m.npoin, 3)))
    return m, prm, st, codes, lnbn, np.asfortranarray(nrm), ub, u_old


def numpy_bc(codes, lnbn, nrm, ub, bc, rho, q, u, pr, E):
    """temporary_bc_routine_dirichlet_prim restated with numpy (mod_bc_routines.f90:17-180)."""
    rho, q, u, pr, E = rho.copy(), q.copy(), u.copy(), pr.copy(), E.copy()
    b = codes < M.MAX_NUM_BOU_CODES
    gi = bc["gamma_inf"]
    rho2 = np.where(b, rho[lnbn], 0.0)
    q2 = np.where(b[:, None], q[lnbn], 0.0)
    E2 = np.where(b, E[lnbn], 0.0)
    with np.errstate(divide="ignore", invalid="ignore"):
        u2 = q2 / rho2[:, None]
        p2 = rho2 * (gi - 1.0) * (E2 / rho2 - 0.5 * np.sum(u2 * u2, axis=1))
    for n in np.flatnonzero(b):
        c = codes[n]
        if c == M.BC_FAR_FIELD:
            E_inf = bc["rho_inf"] * 0.5 * bc["u_inf"] ** 2 + bc["p_inf"] / (gi - 1.0)
            c2 = np.sqrt(gi * p2[n] / rho2[n])
            sl = min(bc["u_inf"] - bc["c_inf"], u2[n, 0] - c2)
            sr = max(u2[n, 0] + c2, bc["u_inf"] + bc["c_inf"])
            rho[n] = (sr * rho2[n] - sl * bc["rho_inf"] + bc["rho_inf"] * bc["u_inf"] - q2[n, 0]) / (sr - sl)
            E[n] = (sr * E2[n] - sl * E_inf + bc["u_inf"] * (E_inf + bc["p_inf"]) - u2[n, 0] * (E2[n] + p2[n])) / (sr - sl)
            for d in range(3):
                sl = min(ub[n, d] - bc["c_inf"], u2[n, d] - c2)
                sr = max(u2[n, d] + c2, ub[n, d] + bc["c_inf"])
                q[n, d] = (sr * q2[n, d] - sl * bc["rho_inf"] * ub[n, d] + bc["rho_inf"] * ub[n, d] ** 2
                           - u2[n, d] * q2[n, d]) / (sr - sl)
            u[n] = q[n] / rho[n]
            pr[n] = rho[n] * (gi - 1.0) * (E[n] / rho[n] - 0.5 * np.dot(u[n], u[n]))
        elif c == M.BC_NON_SLIP_ADIABATIC:
            q[n] = 0.0; u[n] = 0.0; rho[n] = bc["rho_inf"]
        elif c in (M.BC_NON_SLIP_HOT, M.BC_NON_SLIP_COLD):
            q[n] = 0.0; u[n] = 0.0
            rho[n] = bc["p_inf"] / bc["Rgas_inf"] / (bc["T_H"] if c == M.BC_NON_SLIP_HOT else bc["T_C"])
            E[n] = bc["p_inf"] / (gi - 1.0)
        elif c in (M.BC_SLIP_ADIABATIC, M.BC_SLIP_WALL_MODEL):
            E[n] -= rho[n] * 0.5 * np.dot(u[n], u[n])
            q[n] -= np.dot(nrm[n], q[n]) * nrm[n]
            rho[n] = bc["rho_inf"]
            u[n] = q[n] / rho[n]
            E[n] += rho[n] * 0.5 * np.dot(u[n], u[n])
    return rho, q, u, pr, E


def test_bc_dirichlet_prim_vs_numpy(oracle):
    m, prm, st, codes, lnbn, nrm, ub, u_old = random_case()
    bc = M.bc_params(prm)
    bnd = oracle.Boundaries(codes, lnbn, nrm, ub, bc)
    args = [np.array(a, order="F", copy=True) for a in (st.rho, st.q, u_old, st.pr, st.E)]
    ref = numpy_bc(codes, lnbn, nrm, ub, bc, *[a.copy(order="F") for a in args])
    oracle.bc_dirichlet_prim(bnd, *args)
    for name, a, r in zip(("rho", "q", "u", "pr", "E"), args, ref):
        np.testing.assert_allclose(a, r, rtol=1e-14, atol=1e-14 * np.abs(r).max(), err_msg=name)
    inner = codes >= M.MAX_NUM_BOU_CODES
    assert np.array_equal(args[0][inner], st.rho[inner]) and np.array_equal(args[4][inner], st.E[inner])


def test_bc_wall_invariants(oracle):
    m, prm, st, codes, lnbn, nrm, ub, u_old = random_case(seed=5)
    bc = M.bc_params(prm)
    bnd = oracle.Boundaries(codes, lnbn, nrm, ub, bc)
    rho, q, u, pr, E = [np.array(a, order="F", copy=True) for a in (st.rho, st.q, u_old, st.pr, st.E)]
    oracle.bc_dirichlet_prim(bnd, rho, q, u, pr, E)
    ns = np.isin(codes, (M.BC_NON_SLIP_ADIABATIC, M.BC_NON_SLIP_HOT, M.BC_NON_SLIP_COLD))
    assert np.all(q[ns] == 0.0) and np.all(u[ns] == 0.0)
    assert np.all(rho[codes == M.BC_NON_SLIP_ADIABATIC] == bc["rho_inf"])
    hot = codes == M.BC_NON_SLIP_HOT
    np.testing.assert_allclose(rho[hot] * bc["Rgas_inf"] * bc["T_H"], bc["p_inf"], rtol=1e-15)
    slip = np.isin(codes, (M.BC_SLIP_ADIABATIC, M.BC_SLIP_WALL_MODEL))
    assert np.abs(np.sum(q[slip] * nrm[slip], axis=1)).max() < 1e-14 * np.abs(q).max()
    passive = np.isin(codes, (M.BC_OUTLET_INCOMP, M.BC_TOP_ABL))
    assert np.array_equal(rho[passive], st.rho[passive]) and np.array_equal(q[passive], st.q[passive])


def test_bc_fix_residuals(oracle):
    m, prm, st, codes, lnbn, nrm, ub, _ = random_case(seed=7)
    bnd = oracle.Boundaries(codes, lnbn, nrm, ub, M.bc_params(prm))
    rng = np.random.default_rng(1)
    Rm, Re, R = rng.standard_normal(m.npoin), rng.standard_normal(m.npoin), rng.standard_normal(m.npoin)
    Rmo = np.asfortranarray(rng.standard_normal((m.npoin, 3)))
    Rm0, Re0, R0, Rmo0 = Rm.copy(), Re.copy(), R.copy(), Rmo.copy()
    oracle.bc_fix_residual(bnd, Rm, Rmo, Re)
    oracle.bc_fix_residual_entropy(bnd, R)
    ns = np.isin(codes, (M.BC_NON_SLIP_ADIABATIC, M.BC_NON_SLIP_HOT, M.BC_NON_SLIP_COLD))
    iso = np.isin(codes, (M.BC_NON_SLIP_HOT, M.BC_NON_SLIP_COLD))
    assert np.all(Rm[ns] == 0) and np.all(Rmo[ns] == 0) and np.all(R[ns] == 0) and np.all(Re[iso] == 0)
    assert np.array_equal(Rm[~ns], Rm0[~ns]) and np.array_equal(R[~ns], R0[~ns])
    assert np.array_equal(Re[~iso], Re0[~iso]) and np.array_equal(Rmo[~ns], Rmo0[~ns])


def test_channel_mesh_boundary_arrays():
    n = 3
    m = M.channel_box(n, jitter=0.05, seed=2)
    mm = 3 * n
    assert m.npoin == mm * (mm + 1) * mm
    codes, lnbn, nrm = m.extra["bou_codes_nodes"], m.extra["lnbn_nodes"], m.extra["normals"]
    y = m.coord[:, 1]
    assert np.all(y[codes == M.BC_NON_SLIP_ADIABATIC] == 0.0)
    assert np.allclose(y[codes == M.BC_SLIP_ADIABATIC], m.L)
    assert (codes < M.MAX_NUM_BOU_CODES).sum() == 2 * mm * mm
    # nearBoundaryNode: the interior node atoIJK(nnode) of the highest element holding the node
    b = np.flatnonzero(codes < M.MAX_NUM_BOU_CODES)
    assert np.all(codes[lnbn[b]] == M.MAX_NUM_BOU_CODES)
    for nd in b[:: max(1, b.size // 17)]:
        e = np.flatnonzero((m.connec == nd).any(axis=1)).max()
        assert lnbn[nd] == m.connec[e, m.tables.atoIJK[63]]
    assert np.all(np.abs(nrm[b, 1]) == 1.0) and np.all(nrm[codes >= M.MAX_NUM_BOU_CODES] == 0.0)


def test_channel_steps_oracle(oracle):
    """Three rk_4_main steps of the oracle on a channel with a no-slip and a slip wall stay
    finite, keep the no-slip wall at rest and conserve nothing spurious at inner nodes."""
    m = M.channel_box(3, jitter=0.05, seed=4)
    prm = M.TGVParams()
    st = M.taylor_green_state(m, prm, pert_amp=1e-2, seed=4)
    om = oracle.OracleMesh(m)
    bnd = oracle.Boundaries(m.extra["bou_codes_nodes"], m.extra["lnbn_nodes"], m.extra["normals"],
                            np.zeros((m.npoin, 3), order="F"), M.bc_params(prm))
    dt = oracle.adapt_dt(om, st, prm)
    oracle.rk4(om, prm, st, dt, nsteps=3, bnd=bnd)
    codes = m.extra["bou_codes_nodes"]
    assert np.isfinite(st.rho).all() and np.isfinite(st.mu_e).all()
    assert np.all(st.q[codes == M.BC_NON_SLIP_ADIABATIC] == 0.0)
    top = codes == M.BC_SLIP_ADIABATIC
    assert np.abs(st.q[top, 1]).max() < 1e-15
