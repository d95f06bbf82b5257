"""The allocation-free full_convec_ijk entry point against the regular one.

sod_full_convec_ijk_noalloc serves callers that cannot allocate device memory (their device
memory belongs to the OpenACC runtime or to a fixed pool of the host code), so it keeps its
scratch in a static device array instead of a SodMesh.  It must give the same residuals as
sod_full_convec_ijk on the same reference-layout inputs, call after call (the shared scratch
keeps the previous call's contents).  This file is collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-12  # same FP64 arithmetic; only the element loop's data layout differs


def _setup():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from sod2d_refmap_b200 import build, mesh as M, solver as S, _lib
    build.build()
    m = M.periodic_box(3, jitter=0.05, seed=4)
    prm = M.TGVParams()
    gm = S.Sod2dMesh(m, prm)
    geo = gm.geometry()
    st = M.taylor_green_state(m, prm)
    rng = np.random.default_rng(5)
    N = m.npoin
    f64 = lambda a: torch.from_numpy(np.ascontiguousarray(np.asarray(a, dtype=np.float64).ravel(order="F"))).cuda()
    i32 = lambda a: torch.from_numpy(np.ascontiguousarray(np.asarray(a, dtype=np.int32).ravel(order="F"))).cuda()
    u = np.asfortranarray(st.u + 0.01 * rng.standard_normal((N, 3)))
    inp = dict(u=f64(u), q=f64(st.q), rho=f64(st.rho), pr=f64(st.pr), E=f64(3.5 * st.pr / st.rho))
    T = m.tables
    mesh = dict(connec=i32(np.asarray(m.connec) + 1), He=f64(geo["He"]), gpvol=f64(geo["gpvol"]),
                dl=f64(T.dlxigp_ip), gI=i32(T.gmshAtoI + 1), gJ=i32(T.gmshAtoJ + 1), gK=i32(T.gmshAtoK + 1))
    return torch, S, _lib, m, gm, inp, mesh


def _noalloc(torch, _lib, m, mesh, inp, nelem=None):
    N = m.npoin
    out = [torch.full((N,), np.nan, dtype=torch.float64, device="cuda"),
           torch.full((3 * N,), np.nan, dtype=torch.float64, device="cuda"),
           torch.full((N,), np.nan, dtype=torch.float64, device="cuda")]
    p = lambda t: C.c_void_p(int(t.data_ptr()))
    rc = _lib.load().sod_full_convec_ijk_noalloc(
        m.nelem if nelem is None else nelem, N, 1, p(mesh["connec"]), p(mesh["He"]), p(mesh["gpvol"]),
        p(mesh["dl"]), p(mesh["gI"]), p(mesh["gJ"]), p(mesh["gK"]), p(inp["u"]), p(inp["q"]), p(inp["rho"]),
        p(inp["pr"]), p(inp["E"]), p(out[0]), p(out[1]), p(out[2]),
        C.c_void_p(int(torch.cuda.current_stream().cuda_stream)))
    return rc, out


def test_noalloc_matches_regular_entry_point_twice():
    torch, S, _lib, m, gm, inp, mesh = _setup()
    N = m.npoin
    Rm, Rmo, Re = gm.full_convec_ijk(inp["u"].view(3, N), inp["q"].view(3, N), inp["rho"], inp["pr"], inp["E"])
    ref = [Rm, Rmo.reshape(-1), Re]
    for call in range(2):
        rc, out = _noalloc(torch, _lib, m, mesh, inp)
        assert rc == 0, _lib.load().sod_last_error()
        torch.cuda.synchronize()
        for got, want in zip(out, ref):
            err = float((got - want).norm() / want.norm())
            assert err <= TOL, (call, err)


def test_noalloc_rejects_oversized_mesh():
    torch, S, _lib, m, gm, inp, mesh = _setup()
    rc, _ = _noalloc(torch, _lib, m, mesh, inp, nelem=4097)
    assert rc == -1
    assert b"4096 elements" in _lib.load().sod_last_error()
