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


def _box_desc(mesh):
    """A SodMeshDesc over a generated periodic box, with the arrays kept alive on the side."""
    import numpy as np
    from sod2d_refmap_b200 import _lib
    T, keep = mesh.tables, []

    def ptr(a):
        keep.append(a)
        return a.ctypes.data

    d = _lib.SodMeshDesc()
    d.nelem, d.npoin, d.npoin_orig, d.porder, d.index_base = mesh.nelem, mesh.npoin, mesh.npoin_orig, 3, 0
    arrays = dict(connec=np.asfortranarray(mesh.connec, dtype=np.int32),
                  connec_orig=np.asfortranarray(mesh.connec_orig, dtype=np.int32),
                  coord_orig=np.asfortranarray(mesh.coord_orig, dtype=np.float64),
                  dlxigp_ip=np.asfortranarray(T.dlxigp_ip), wgp=np.ascontiguousarray(T.wgp),
                  gmshAtoI=np.ascontiguousarray(T.gmshAtoI, dtype=np.int32),
                  gmshAtoJ=np.ascontiguousarray(T.gmshAtoJ, dtype=np.int32),
                  gmshAtoK=np.ascontiguousarray(T.gmshAtoK, dtype=np.int32))
    for k, a in arrays.items():
        setattr(d, k, ptr(a))
    return d, arrays, keep


@pytest.mark.parametrize("case", ["nelem0", "no_geometry", "ijk_range", "ijk_duplicate", "connec_range",
                                  "unreferenced_node"])
def test_mesh_tables_and_connectivity_validated(L, case):
    """Each malformed description is refused with SOD_ERR_ARG and its own message, and no handle is
    returned: the checks run on the host before the first device allocation."""
    from sod2d_refmap_b200 import mesh as M
    d, arrays, keep = _box_desc(M.periodic_box(2))
    expect = {"nelem0": "positive", "no_geometry": "either He+gpvol", "ijk_range": "out of range at local node",
              "ijk_duplicate": "two local nodes", "connec_range": "connec(", "unreferenced_node": "not referenced"}
    if case == "nelem0":
        d.nelem = 0
    elif case == "no_geometry":
        d.coord_orig = None
    elif case == "ijk_range":
        arrays["gmshAtoI"][5] = 4
    elif case == "ijk_duplicate":
        for k in ("gmshAtoI", "gmshAtoJ", "gmshAtoK"):
            arrays[k][7] = arrays[k][3]
    elif case == "connec_range":
        arrays["connec"][1, 10] = d.npoin
    elif case == "unreferenced_node":
        d.npoin += 1
    out = C.c_void_p(0)
    assert L.sod_mesh_create(C.byref(d), None, C.byref(out)) == SOD_ERR_ARG
    assert expect[case] in _msg(L)
    assert out.value is None
    del keep
