"""Legacy element-loop API (sod_legacy_*) through the C ABI against the unit tests' data, the
companion-script residuals and the oracle.

Bounds: the unit tests' own check |sum_a R_a| < 1e-14 and the script residuals to 1e-14
(absolute, residuals of order 1); on a 3-D HEX64 mesh with random fields the CUDA result matches
the oracle to 1e-12 relative (FP64, different summation order inside an element).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASES = ["mass_convec", "generic_scalar_convec", "mom_convec", "ener_convec", "mom_diffu"]


@pytest.fixture(scope="module")
def S():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from sod2d_refmap_b200 import build, solver
    build.build()
    return solver


def _call(S, name, c, connec, Ngp, gpcar, gpvol):
    a = lambda k: np.array(c[k])
    if name == "mass_convec":
        return S.legacy_mass_convec(connec, Ngp, gpcar, gpvol, a("q"))
    if name == "generic_scalar_convec":
        return S.legacy_generic_scalar_convec(connec, Ngp, gpcar, gpvol, a("q"))
    if name == "mom_convec":
        return S.legacy_mom_convec(connec, Ngp, gpcar, gpvol, a("u"), a("q"), a("pr"))
    if name == "ener_convec":
        return S.legacy_ener_convec(connec, Ngp, gpcar, gpvol, a("u"), a("pr"), a("E"))
    return S.legacy_mom_diffusion(connec, Ngp, gpcar, gpvol, a("u"), a("mu_e"))


@pytest.mark.parametrize("name", CASES)
def test_legacy_unit_test_cases(S, kats, oracle, name):
    c = kats["legacy_" + name]
    connec, Ngp, gpcar, gpvol = (np.array(c[k]) for k in ("connec", "Ngp", "gpcar", "gpvol"))
    R = _call(S, name, c, connec, Ngp, gpcar, gpvol)
    if "R_expected" in c:
        assert np.abs(R - np.array(c["R_expected"])).max() < 1e-14
    assert np.all(np.abs(np.atleast_1d(R.sum(axis=0))) < c["sum_tol"])
    if name == "mom_diffu":
        ref = oracle.legacy_mom_diffusion(connec, Ngp, gpcar, gpvol, np.array(c["u"]), np.array(c["mu_e"]))
        assert np.abs(R - ref).max() < 1e-14


def test_legacy_hex64_random_fields_vs_oracle(S, oracle):
    """3-D HEX64 elements (collocated: Ngp = identity, gpcar = He dN) with random fields."""
    from sod2d_refmap_b200 import mesh as M
    m = M.periodic_box(2, jitter=0.05, seed=5)
    om = oracle.OracleMesh(m)
    T = m.tables
    dN = np.asarray(T.dNgp)                                   # (3, 64, 64)
    gpcar = np.einsum("rkge,kag->rage", om.He, dN)            # (3, 64, 64, nelem)
    Ngp = np.eye(64)
    gpvol = om.gpvol
    connec = np.asfortranarray(m.connec + 1)
    rng = np.random.default_rng(3)
    N = m.npoin
    q, u = rng.standard_normal((N, 3)), rng.standard_normal((N, 3))
    pr, E = rng.uniform(0.5, 1.5, N), rng.uniform(1.0, 2.0, N)
    mu_e = rng.uniform(0.0, 0.1, m.nelem)
    pairs = [
        (S.legacy_mass_convec(connec, Ngp, gpcar, gpvol, q), oracle.legacy_mass_convec(connec, Ngp, gpcar, gpvol, q)),
        (S.legacy_mom_convec(connec, Ngp, gpcar, gpvol, u, q, pr),
         oracle.legacy_mom_convec(connec, Ngp, gpcar, gpvol, u, q, pr)),
        (S.legacy_ener_convec(connec, Ngp, gpcar, gpvol, u, pr, E),
         oracle.legacy_ener_convec(connec, Ngp, gpcar, gpvol, u, pr, E)),
        (S.legacy_mom_diffusion(connec, Ngp, gpcar, gpvol, u, mu_e),
         oracle.legacy_mom_diffusion(connec, Ngp, gpcar, gpvol, u, mu_e)),
    ]
    for got, ref in pairs:
        assert np.linalg.norm(got - ref) <= 1e-12 * np.linalg.norm(ref)


def test_legacy_rejects_bad_connectivity(S, kats):
    from sod2d_refmap_b200 import _lib
    c = kats["legacy_mass_convec"]
    connec = np.array(c["connec"])
    connec[1, 2] = 99  # outside 1..npoin: flagged by the counting pass, nothing else runs
    with pytest.raises(_lib.SodError):
        S.legacy_mass_convec(connec, np.array(c["Ngp"]), np.array(c["gpcar"]), np.array(c["gpvol"]), np.array(c["q"]))
