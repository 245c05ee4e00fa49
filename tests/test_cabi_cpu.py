"""C-ABI checks that need no GPU: the library loads, exports every function
include/cfdb.h declares, builds host geometry identical to the oracle's, and
rejects bad arguments with status codes instead of aborting."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest


def test_library_exports_every_header_function(cfdb):
    names = cfdb.capi.header_functions()
    assert len(names) > 40
    L = cfdb.lib()
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    unbound = [n for n in names if n not in cfdb.capi.PROTOTYPES]
    assert not unbound, unbound


def test_abi_version(cfdb):
    assert cfdb.lib().cfdb_abi_version() == 1


@pytest.mark.parametrize("shape,spacing", [((5, 6, 7), (0.2, 1 / 6, 1 / 7)), ((4, 4, 8), (1.0, 1.0, 1.0))])
def test_structured_geometry_bit_identical_to_oracle(cfdb, oracle, shape, spacing):
    m = cfdb.Mesh.structured(None, *shape, *spacing)
    o = oracle.Mesh(*shape, *spacing).geometry()
    cap = cfdb.capi
    pairs = [(cap.GEOM_NORMAL, "normal"), (cap.GEOM_NORMAL_ALT, "normal_alt"), (cap.GEOM_AREA, "area"),
             (cap.GEOM_ALPHA_D, "alpha_d"), (cap.GEOM_LEN_C2F, "len_c2f"), (cap.GEOM_VOLUME, "volume"),
             (cap.GEOM_CENTER, "center"), (cap.GEOM_IS_BOUNDARY, "is_boundary")]
    for which, key in pairs:
        assert np.array_equal(m.geometry(which), o[key]), key
    ids, ibf = m.ids()
    assert np.array_equal(ids, o["ids"]) and np.array_equal(ibf, o["ids_bound_free"])


@pytest.mark.parametrize("compat", [False, True])
def test_vertex_geometry_bit_identical_to_oracle(cfdb, oracle, compat):
    from cfdarcov2_b200.workloads import jittered_vertices
    n = 5
    V = jittered_vertices(n, amp=0.05 if compat else 0.2, seed=2)
    m = cfdb.Mesh.from_vertices(None, n, n, n, 1 / n, 1 / n, 1 / n, V, compat_area=compat)
    o = oracle.Mesh(n, n, n, 1 / n, 1 / n, 1 / n, vertices=V, compat_area=compat).geometry()
    cap = cfdb.capi
    for which, key in [(cap.GEOM_NORMAL_ALT, "normal_alt"), (cap.GEOM_AREA, "area"), (cap.GEOM_ALPHA_D, "alpha_d"),
                       (cap.GEOM_VOLUME, "volume"), (cap.GEOM_LEN_C2F, "len_c2f")]:
        assert np.array_equal(m.geometry(which), o[key]), key


def test_tangled_vertices_rejected(cfdb):
    from cfdarcov2_b200.workloads import jittered_vertices
    V = jittered_vertices(4, amp=0.0).reshape(5, 5, 5, 3).copy()
    V[2, 2, 2, 0] += 0.6  # push an interior vertex through its neighbours
    with pytest.raises(cfdb.CfdbError) as e:
        cfdb.Mesh.from_vertices(None, 4, 4, 4, 0.25, 0.25, 0.25, V.reshape(-1, 3))
    assert e.value.code == cfdb.capi.EINVAL and "tangled" in str(e.value)


def test_bad_arguments_return_status(cfdb):
    L = cfdb.lib()
    h = C.c_void_p()
    assert L.cfdb_mesh_create_structured(None, 0, 4, 4, 1.0, 1.0, 1.0, C.byref(h)) == cfdb.capi.EINVAL
    assert "dimensions" in cfdb.capi.last_error()
    assert L.cfdb_mesh_create_structured(None, 4, 4, 4, -1.0, 1.0, 1.0, C.byref(h)) == cfdb.capi.EINVAL
    assert L.cfdb_mesh_create_structured(None, 4, 4, 4, 1.0, 1.0, 1.0, None) == cfdb.capi.EINVAL
    assert L.cfdb_mesh_create_structured(None, 1 << 12, 1 << 12, 1 << 8, 1.0, 1.0, 1.0, C.byref(h)) == cfdb.capi.EINVAL
    # device calls on a host-only mesh or without a context fail cleanly
    m = cfdb.Mesh.structured(None, 4, 4, 4, 1.0, 1.0, 1.0)
    assert L.cfdb_op_lapl(None, m.h, 0, None, None, 7) == cfdb.capi.EINVAL
    assert L.cfdb_heat_step(None, m.h, 0, 1, None, None, 1.0, 1.0) == cfdb.capi.EINVAL
    assert L.cfdb_sync(None) == cfdb.capi.EINVAL
    assert L.cfdb_mesh_info(None, None, None, None) == cfdb.capi.EINVAL


def test_mesh_info_and_wave_dt(cfdb):
    m = cfdb.Mesh.structured(None, 8, 4, 2, 0.125, 0.25, 0.5)
    dims = (C.c_int64 * 3)()
    sp = (C.c_double * 3)()
    uni = C.c_int()
    assert cfdb.lib().cfdb_mesh_info(m.h, dims, sp, C.byref(uni)) == 0
    assert list(dims) == [8, 4, 2] and list(sp) == [0.125, 0.25, 0.5] and uni.value == 1
    assert m.wave_dt(0.4, c_const=2.0) == pytest.approx(0.4 / (2 * (8 + 4 + 2)))


def test_wave_dt_matches_oracle_on_vertex_mesh(cfdb, oracle):
    from cfdarcov2_b200.workloads import jittered_vertices
    n = 6
    V = jittered_vertices(n, seed=2)
    m = cfdb.Mesh.from_vertices(None, n, n, n, 1 / n, 1 / n, 1 / n, V)
    o = oracle.Mesh(n, n, n, 1 / n, 1 / n, 1 / n, vertices=V)
    rng = np.random.default_rng(0)
    c = np.exp(0.2 * rng.standard_normal(m.n))
    assert m.wave_dt(0.4, c=c) == pytest.approx(o.wave_dt(0.4, c=c), rel=1e-15)


def test_missing_library_fails_loudly(cfdb, monkeypatch, tmp_path):
    """No fallback: with libcfdb.so absent every entry into the library raises
    ImportError naming the build command (the package itself still imports,
    because the build module lives in it)."""
    cap = cfdb.capi
    monkeypatch.setattr(cap, "LIB_PATH", str(tmp_path / "libcfdb.so"))
    monkeypatch.setattr(cap, "_lib", None)
    with pytest.raises(ImportError, match="cfdarcov2_b200.build"):
        cap.lib()
    with pytest.raises(ImportError):
        cfdb.Mesh.structured(None, 4, 4, 4, 1.0, 1.0, 1.0)
