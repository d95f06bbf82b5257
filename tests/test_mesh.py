"""Mesh generator, gmsh ordering, seeds and TGV state (no GPU)."""
import numpy as np

from sod2d_refmap_b200 import mesh as M


def test_gmsh_hex_order_p3():
    t = M.gmsh_hex_table(3)
    assert t.shape == (64, 3) and len({tuple(r) for r in t}) == 64
    # corners first in gmsh order (genHighOrderHexGmsh, mod_ijk_indices.f90:584-593)
    assert t[:8].tolist() == [[0, 0, 0], [3, 0, 0], [3, 3, 0], [0, 3, 0], [0, 0, 3], [3, 0, 3], [3, 3, 3], [0, 3, 3]]
    # first edge (1->2) interior nodes, then the volume nodes last
    assert t[8].tolist() == [1, 0, 0] and t[9].tolist() == [2, 0, 0]
    assert all(1 <= v <= 2 for r in t[56:] for v in r)


def test_a2ijk_is_permutation():
    a = M.a2ijk_table(3)
    assert sorted(a.tolist()) == list(range(64))


def test_periodic_box_topology():
    m = M.periodic_box(3)
    assert m.npoin == 9 ** 3 and m.nelem == 27 and m.npoin_orig == 10 ** 3
    counts = np.bincount(m.connec.ravel(order="F"), minlength=m.npoin)
    # every unique node is shared: 8 (vertex), 4 (edge), 2 (face) or 1 (interior) elements
    assert set(np.unique(counts)) == {1, 2, 4, 8}
    assert counts.sum() == 64 * m.nelem
    # master coordinates lie in [0, L)
    assert m.coord.min() >= 0.0 and m.coord.max() < m.L


def test_jitter_periodic_consistent():
    m = M.periodic_box(4, jitter=0.05, seed=1)
    disp = m.coord_orig - M.periodic_box(4).coord_orig
    # every orig image of a unique node moves by the same displacement
    for c in range(3):
        d = np.zeros(m.npoin); d[m.master] = disp[:, c]
        assert np.allclose(disp[:, c], d[m.master])
    hnode = (1 - 1 / np.sqrt(5)) / 2 * m.L / 4
    assert np.abs(disp).max() <= 3 * 0.05 * hnode + 1e-15


def test_splitmix_deterministic():
    ids = np.arange(5, dtype=np.int64)
    a = M.uniform01(7, 1, ids)
    b = M.uniform01(7, 1, ids[::-1])[::-1]
    assert np.array_equal(a, b) and (a >= 0).all() and (a < 1).all()
    # SplitMix64 reference value for key 0 (Steele et al. 2014)
    assert int(M.splitmix64(np.array([0], dtype=np.uint64))[0]) == 0xE220A8397B1DCDAF


def test_tgv_state():
    m = M.periodic_box(2)
    prm = M.TGVParams()
    st = M.taylor_green_state(m, prm)
    assert np.allclose(st.q, st.rho[:, None] * st.u)
    assert abs(st.pr.mean() - prm.p0) < 1.0
    assert np.allclose(st.Tem, st.pr / (st.rho * prm.Rgas))
