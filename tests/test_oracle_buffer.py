"""The oracle's updateBuffer (time_integ.f90:510-589) against an independent numpy restatement,
and its properties: the identity (up to rounding) outside the zones, the free-stream state at
the far end of a zone, and rk_4_main with the zone on (the free-stream density deep in a zone)."""
import numpy as np
import pytest

from _util import rel_l2


def np_update_buffer(coord, u_buffer, prm, rho, q, E):
    sides = (("east", 0, 1), ("west", 0, -1), ("north", 1, 1), ("south", 1, -1), ("top", 2, 1), ("bottom", 2, -1))
    xi = np.ones(len(rho))
    for name, ax, sgn in sides:
        if not prm["on_" + name]:
            continue
        mn, sz = prm[name[0] + "_min"], prm[name[0] + "_size"]
        xs = coord[:, ax]
        inside = xs > mn if sgn > 0 else xs < mn
        xb = np.where(inside, (xs - mn) / sz if sgn > 0 else (mn - xs) / sz, 0.0)
        f = (1.0 - 0.01 * xb * xb) * (1.0 - (1.0 - np.exp(10.0 * xb * xb)) / (1.0 - np.exp(10.0)))
        xi = np.where(inside, np.minimum(f, xi), xi)
    E_inf = prm["rho_inf"] * 0.5 * prm["u_inf"] ** 2 + prm["p_inf"] / (prm["gamma_inf"] - 1.0)
    ur = u_buffer * rho[:, None]
    return (prm["rho_inf"] + xi * (rho - prm["rho_inf"]), ur + xi[:, None] * (q - ur), E_inf + xi * (E - E_inf), xi)


@pytest.fixture(scope="module")
def case(oracle):
    from sod2d_refmap_b200 import mesh as M
    m = M.periodic_box(3, jitter=0.05, seed=3)
    prm = M.TGVParams()
    st = M.taylor_green_state(m, prm, pert_amp=1e-2, seed=3)
    L = 2.0 * np.pi
    # zones whose far ends lie just beyond the outermost nodes (xb <= 0.995: xi in (0, 1], down
    # to ~0.1 there; the factor stays near 1 until xb approaches 1)
    lo, hi = m.coord.min(axis=0), m.coord.max(axis=0)
    bp = M.buffer_params(prm, east=(0.6 * L, (hi[0] - 0.6 * L) / 0.995),
                         south=(0.4 * L, (0.4 * L - lo[1]) / 0.995), top=(0.7 * L, (hi[2] - 0.7 * L) / 0.995))
    rng = np.random.default_rng(3)
    ub = np.asfortranarray(np.column_stack([np.full(m.npoin, 1.0), rng.uniform(-0.1, 0.1, (m.npoin, 2))]))
    return m, prm, st, bp, ub


def test_update_buffer_matches_numpy(case, oracle):
    m, prm, st, bp, ub = case
    buf = oracle.BufferZone(m.coord, ub, bp)
    rho, q, E = st.rho.copy(), np.array(st.q, order="F", copy=True), st.E.copy()
    oracle.update_buffer(buf, rho, q, E)
    r2, q2, E2, xi = np_update_buffer(m.coord, ub, bp, st.rho, st.q, st.E)
    assert 0 < (xi < 1).sum() < m.npoin
    for a, b in ((rho, r2), (q, q2), (E, E2)):
        assert rel_l2(a, b) < 1e-15
    out = xi == 1.0
    assert np.allclose(rho[out], st.rho[out], rtol=1e-15, atol=0)
    assert np.allclose(E[out], st.E[out], rtol=1e-15, atol=0)


def test_far_end_is_free_stream(oracle):
    from sod2d_refmap_b200 import mesh as M
    m = M.channel_box(2, seed=1)  # walls at y = 0 and y = L: nodes on y = L exist
    prm = M.TGVParams()
    st = M.taylor_green_state(m, prm, pert_amp=1e-2, seed=1)
    L = 2.0 * np.pi
    bp = M.buffer_params(prm, u_inf=0.5, north=(0.5 * L, 0.5 * L))  # y = L is the zone's far end (xb = 1)
    ub = np.zeros((m.npoin, 3), order="F"); ub[:, 0] = 0.5
    rho, q, E = st.rho.copy(), np.array(st.q, order="F", copy=True), st.E.copy()
    oracle.update_buffer(oracle.BufferZone(m.coord, ub, bp), rho, q, E)
    far = np.isclose(m.coord[:, 1], L, rtol=0, atol=1e-12)
    assert far.any()
    E_inf = prm.rho0 * 0.5 * 0.25 + prm.p0 / (prm.gamma_gas - 1.0)
    assert np.allclose(rho[far], prm.rho0, rtol=1e-14)
    assert np.allclose(E[far], E_inf, rtol=1e-14)
    assert np.allclose(q[far, 0], 0.5 * st.rho[far], rtol=1e-14)
    assert np.allclose(q[far, 1:], 0.0, atol=1e-14)


def test_rk4_with_buffer_relaxes_the_zone(case, oracle):
    from sod2d_refmap_b200 import mesh as M
    m, prm, st0, bp, ub = case
    om = oracle.OracleMesh(m)
    dt = oracle.adapt_dt(om, st0, prm)
    a, b = st0.copy(), st0.copy()
    oracle.rk4(om, prm, a, dt, nsteps=2)
    oracle.rk4(om, prm, b, dt, nsteps=2, buf=oracle.BufferZone(m.coord, ub, bp))
    xi = np_update_buffer(m.coord, ub, bp, st0.rho, st0.q, st0.E)[3]
    assert 0 < xi.min() and (xi < 0.5).any()
    # the last updateBuffer of the step scales rho - rho_inf by xi: the density deviation is
    # smallest deep in the zones
    dev = np.abs(b.rho - prm.rho0)
    assert dev[xi < 0.2].max() < dev[xi == 1.0].max()
    assert rel_l2(b.rho, a.rho) > 1e-8
    assert np.isfinite(b.mu_e).all() and (b.rho > 0).all()
