"""The oracle's compute_fieldDerivs (mod_postpro.f90:12-139) on fields the p = 3 elements
represent exactly (undistorted channel mesh, fields polynomial in the wall-normal coordinate y):
gradRho, the reference's curl sum_jk leviCivi(i,j,k) du_j/dx_k, the split divergence
(div(rho u) + rho div u)/2 and Q = -1/2 du_i/dx_j du_j/dx_i against their closed forms (1e-10)."""
import numpy as np


def linear_case(M):
    m = M.channel_box(2, jitter=0.0, seed=1)
    y = m.coord[:, 1]
    a, b, c, d = 0.3, 0.05, -0.2, 0.1
    rho = 1.0 + b * y
    u = np.asfortranarray(np.column_stack([a * y, d * y, c * y]))
    exact = dict(gradRho=np.column_stack([0 * y, b + 0 * y, 0 * y]),
                 curlU=np.column_stack([-c + 0 * y, 0 * y, a + 0 * y]),
                 divU=0.5 * d * (2.0 + 3.0 * b * y), Qcrit=-0.5 * d * d + 0 * y)
    return m, rho, u, exact


def test_field_derivs_exact_on_polynomial_fields(oracle):
    from sod2d_refmap_b200 import mesh as M
    m, rho, u, exact = linear_case(M)
    g, c, dv, qc = oracle.compute_field_derivs(oracle.OracleMesh(m), rho, u)
    for got, ref in ((g, exact["gradRho"]), (c, exact["curlU"]), (dv, exact["divU"]), (qc, exact["Qcrit"])):
        assert np.abs(got - ref).max() <= 1e-10 * max(1.0, np.abs(ref).max())


def test_levi_civita_argument(oracle):
    """The symbol is an argument: its negative flips the curl and nothing else."""
    from sod2d_refmap_b200 import mesh as M
    m, rho, u, _ = linear_case(M)
    om = oracle.OracleMesh(m)
    a = oracle.compute_field_derivs(om, rho, u)
    b = oracle.compute_field_derivs(om, rho, u, levi=-oracle.levi_civita())
    assert np.array_equal(b[1], -a[1])
    for q in (0, 2, 3):
        assert np.array_equal(a[q], b[q])
