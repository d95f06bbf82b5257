"""Error behaviour of the C ABI without a GPU: invalid arguments are rejected with SOD_ERR_ARG
and a message before any device work (the reference has no error returns; it stops the
program, so every caller-visible failure here is a return code plus sod_last_error())."""
import ctypes as C

import pytest

SOD_ERR_ARG = -1


@pytest.fixture(scope="module")
def L():
    from sod2d_refmap_b200 import build, _lib
    build.build()
    return _lib.load()


def _msg(L):
    f = L.sod_last_error
    f.restype = C.c_char_p
    return f().decode()


def test_null_mesh_and_state_rejected(L):
    assert L.sod_rk4_main(None, None, None, None, 0, None) == SOD_ERR_ARG
    assert "null" in _msg(L)
    assert L.sod_rk4_steps(None, None, None, 1, 0, None) == SOD_ERR_ARG
    assert L.sod_rhs(None, None, None, None, None, None, None, None, None, None, 0, None) == SOD_ERR_ARG
    assert L.sod_rhs_vjp(*([None] * 13)) == SOD_ERR_ARG


def test_mesh_description_validated(L):
    from sod2d_refmap_b200 import _lib
    d = _lib.SodMeshDesc()
    d.nelem, d.npoin, d.porder, d.index_base = 8, 216, 4, 0
    out = C.c_void_p(0)
    assert L.sod_mesh_create(C.byref(d), None, C.byref(out)) == SOD_ERR_ARG
    assert "porder" in _msg(L)
    d.porder, d.index_base = 3, 2
    assert L.sod_mesh_create(C.byref(d), None, C.byref(out)) == SOD_ERR_ARG
    assert out.value is None


def test_allocation_free_entry_rejects_oversize(L):
    buf = (C.c_double * 8)()
    p = C.cast(buf, C.c_void_p)
    too_many = 4097  # SOD_NOALLOC_MAX_ELEM + 1
    rc = L.sod_full_convec_ijk_noalloc(too_many, 27 * too_many, 0, p, p, p, p, p, p, p, p, p, p, p, p, p, p, p, None)
    assert rc == SOD_ERR_ARG
    assert "4096" in _msg(L)


def test_legacy_entry_points_validate_sizes(L):
    buf = (C.c_double * 8)()
    p = C.cast(buf, C.c_void_p)
    # nnode above 64 and ndime outside {2, 3} are refused before any device call
    assert L.sod_legacy_mass_convec(2, 4, 6, 65, 2, p, p, p, p, p, p, None) == SOD_ERR_ARG
    assert L.sod_legacy_mass_convec(2, 4, 6, 4, 4, p, p, p, p, p, p, None) == SOD_ERR_ARG
    assert L.sod_legacy_mom_convec(2, 4, 6, 4, 2, p, p, p, p, p, p, None, p, None) == SOD_ERR_ARG  # pr null


def test_batch_and_poisson_validate(L):
    out = C.c_void_p(0)
    assert L.sod_batch_create(None, 0, C.byref(out)) == SOD_ERR_ARG
    assert L.sod_poisson_create(None, C.byref(out)) == SOD_ERR_ARG
