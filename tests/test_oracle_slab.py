"""The slab method used to compare the GPU residual with the oracle on the 64^3 benchmark mesh:
on an 8^3 jittered periodic box, the oracle's stage residual on a 4-layer slab equals its
residual on the whole mesh at the slab-interior nodes (the nodes whose elements all lie in the
slab), up to the summation order of the scatter."""
import numpy as np

from _util import rel_l2, slab_oracle, slab_state


def test_slab_interior_equals_full_mesh(oracle):
    from sod2d_refmap_b200 import mesh as M
    m = M.periodic_box(8, jitter=0.05, seed=1)
    prm = M.TGVParams()
    st = M.taylor_green_state(m, prm)
    om = oracle.OracleMesh(m)
    dt = oracle.adapt_dt(om, st, prm)
    oracle.rk4(om, prm, st, dt, nsteps=1)          # a state with mu_e > 0
    assert float(np.abs(st.mu_e).max()) > 0.0
    full = oracle.rhs_stage(om, prm, st)
    som, nodes, E, idx = slab_oracle(oracle, M, m, 4)
    assert len(idx) == 11 * 24 * 24
    part = oracle.rhs_stage(som, prm, slab_state(st, nodes, E, st.mu_e))
    for f in range(5):
        assert rel_l2(part[f, idx], full[f, nodes[idx]]) < 1e-14, f
    # a node on the slab's faces misses the contributions of the elements outside it
    face = np.setdiff1d(np.arange(len(nodes)), idx)
    assert rel_l2(part[0, face], full[0, nodes[face]]) > 1e-3
