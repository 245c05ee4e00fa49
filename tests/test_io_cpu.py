"""Output files of the reference's IO layer written by libcfdb without VTK or
nlohmann::json (include/io_operators_tmpl.hpp): the .vti image of a field
(store_history) and mesh.json (store_mesh), numbered as
Mesh3D::init_basic_internals (src/mesh3d.cpp:323-416).  Host-only, CPU."""
from __future__ import annotations

import json
import re

import numpy as np
import pytest


def read_vti(path):
    data = open(path, "rb").read()
    head = data[: data.index(b"<AppendedData")].decode()
    i = data.index(b"_", data.index(b"<AppendedData"))
    nbytes = int(np.frombuffer(data[i + 1: i + 9], np.uint64)[0])
    arr = np.frombuffer(data[i + 9: i + 9 + nbytes], np.float32)
    assert data[i + 9 + nbytes:].strip().startswith(b"</AppendedData>")
    return head, arr


def test_vti_point_order_header_and_range(cfdb, tmp_path):
    X, Y, Z = 5, 3, 7
    vals = np.random.default_rng(1).standard_normal(X * Y * Z).astype(np.float32)
    p = tmp_path / "res_0.vti"
    cfdb.write_vti(p, "rho", vals, X, Y, Z)
    head, img = read_vti(p)
    assert 'type="ImageData"' in head and 'header_type="UInt64"' in head
    assert f'WholeExtent="0 {X - 1} 0 {Y - 1} 0 {Z - 1}"' in head
    assert 'Spacing="1 1 1"' in head and 'Name="rho"' in head and 'type="Float32"' in head
    lo = float(re.search(r'RangeMin="([^"]+)"', head).group(1))
    hi = float(re.search(r'RangeMax="([^"]+)"', head).group(1))
    assert lo == pytest.approx(vals.min(), rel=1e-7) and hi == pytest.approx(vals.max(), rel=1e-7)
    # VTK image points run x fastest; point (x, y, z) holds cell Z*Y*x + Z*y + z
    x, y, z = np.meshgrid(np.arange(X), np.arange(Y), np.arange(Z), indexing="ij")
    assert np.array_equal(img[x + X * (y + Y * z)], vals[Z * Y * x + Z * y + z])


def test_vti_rejects_bad_sizes_and_paths(cfdb, tmp_path):
    with pytest.raises(ValueError):
        cfdb.write_vti(tmp_path / "a.vti", "T", np.zeros(5), 2, 2, 2)
    with pytest.raises(cfdb.CfdbError) as e:
        cfdb.write_vti(tmp_path / "no_such_dir" / "a.vti", "T", np.zeros(8), 2, 2, 2)
    assert e.value.code == cfdb.capi.EIO


def test_mesh_json_numbering(cfdb, tmp_path):
    X, Y, Z = 3, 2, 4
    dx, dy, dz = 0.5, 0.25, 0.125
    p = tmp_path / "mesh.json"
    cfdb.write_mesh_json(p, X, Y, Z, dx, dy, dz)
    m = json.loads(p.read_text())
    nv, nf, nn = (X + 1) * (Y + 1) * (Z + 1), X * Y * (Z + 1) + Z * Y * (X + 1) + X * Z * (Y + 1), X * Y * Z
    assert (len(m["vertexes"]), len(m["face"]), len(m["nodes"])) == (nv, nf, nn)
    assert (m["x"], m["y"], m["z"]) == (X, Y, Z)
    assert m["lx"] == pytest.approx(X * dx) and m["lz"] == pytest.approx(Z * dz)
    V = np.array(m["vertexes"])
    vid = lambda x, y, z: x * (Z + 1) * (Y + 1) + y * (Z + 1) + z  # noqa: E731
    assert np.allclose(V[vid(2, 1, 3)], [2 * dx, 1 * dy, 3 * dz])
    seen = np.zeros(nf, int)
    for x in range(X):
        for y in range(Y):
            for z in range(Z):
                cid = Z * Y * x + Z * y + z
                node = m["nodes"][cid]
                corners = [vid(x + i, y + j, z + k) for i in (0, 1) for j in (0, 1) for k in (0, 1)]
                assert node["vertexes"] == corners
                fz = (Z + 1) * Y * x + (Z + 1) * y + z
                fy = X * Y * (Z + 1) + X * (Y + 1) * z + (Y + 1) * x + y
                fx = X * Y * (Z + 1) + X * (Y + 1) * Z + (X + 1) * Z * y + (X + 1) * z + x
                assert node["face"] == [fz, fz + 1, fy, fy + 1, fx, fx + 1]
                for k, f in enumerate(node["face"]):
                    face = m["face"][f]
                    assert cid in face["nodes_id"]
                    seen[f] += 1
                    # a face's four corners are corners of the cell, on the plane of its axis
                    pts = V[face["vertexes_id"]]
                    assert set(face["vertexes_id"]) <= set(corners)
                    axis = 2 - k // 2  # faces 0,1: z; 2,3: y; 4,5: x
                    assert np.ptp(pts[:, axis]) == 0
    # interior faces belong to two cells (lower cell first), boundary faces to one
    for f, face in enumerate(m["face"]):
        assert len(face["nodes_id"]) == seen[f] and face["nodes_id"] == sorted(face["nodes_id"])


def test_mesh_json_takes_given_vertices(cfdb, tmp_path):
    from cfdarcov2_b200.workloads import jittered_vertices
    n = 3
    Vx = jittered_vertices(n, seed=4)
    p = tmp_path / "mesh.json"
    cfdb.write_mesh_json(p, n, n, n, 1 / n, 1 / n, 1 / n, Vx)
    V = np.array(json.loads(p.read_text())["vertexes"])
    assert np.allclose(V, np.asarray(Vx).reshape(-1, 3).astype(np.float32), rtol=0, atol=1e-7)


@pytest.mark.parametrize("dtype,fields", [(np.float32, 4), (np.float64, 5), (np.float32, 1)])
def test_checkpoint_round_trip(cfdb, tmp_path, dtype, fields):
    """cfdb_state_save / cfdb_state_load: values, step and time come back
    exactly; no temporary file is left behind."""
    nx, ny, nz = 5, 3, 4
    rng = np.random.default_rng(21)
    v = rng.standard_normal(fields * nx * ny * nz).astype(dtype)
    p = tmp_path / "state.ckpt"
    cfdb.save_state(p, v, nx, ny, nz, fields, step=123, t=0.0625)
    got, step, t = cfdb.load_state(p, nx, ny, nz, fields, dtype=dtype)
    assert np.array_equal(got, v) and step == 123 and t == 0.0625
    assert sorted(q.name for q in tmp_path.iterdir()) == ["state.ckpt"]
    assert p.stat().st_size == 64 + v.nbytes


def test_checkpoint_rejects_mismatch_and_damage(cfdb, tmp_path):
    cap = cfdb.capi
    nx, ny, nz = 4, 4, 4
    v = np.arange(2 * nx * ny * nz, dtype=np.float32)
    p = tmp_path / "s.ckpt"
    cfdb.save_state(p, v, nx, ny, nz, 2, step=7, t=1.5)
    for args in [(nx, ny, nz, 3, np.float32), (nx, ny, 8, 2, np.float32), (nx, ny, nz, 2, np.float64)]:
        with pytest.raises(cap.CfdbError) as e:
            cfdb.load_state(p, *args[:4], dtype=args[4])
        assert e.value.code == cap.EINVAL
    data = p.read_bytes()
    (tmp_path / "short.ckpt").write_bytes(data[:-8])
    (tmp_path / "foreign.ckpt").write_bytes(b"NOTACKPT" + data[8:])
    for name in ["short.ckpt", "foreign.ckpt", "missing.ckpt"]:
        with pytest.raises(cap.CfdbError) as e:
            cfdb.load_state(tmp_path / name, nx, ny, nz, 2)
        assert e.value.code == cap.EIO, name
    with pytest.raises(cap.CfdbError) as e:
        cfdb.save_state(tmp_path / "no_such_dir" / "x.ckpt", v, nx, ny, nz, 2)
    assert e.value.code == cap.EIO
