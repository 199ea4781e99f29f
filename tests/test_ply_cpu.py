"""PLY load/save in the reference's layout (src/gaussian_model.cpp:860-1060): round trips, the
property order savePly writes, the channel-major SH mapping, other encodings, and errors."""
import numpy as np
import pytest

from omnigs_b200 import ply


def _random(P, M, seed=0):
    r = np.random.default_rng(seed)
    f = lambda *s: r.standard_normal(s).astype(np.float32)  # noqa: E731
    return ply.PlyGaussians(xyz=f(P, 3), features_dc=f(P, 1, 3), features_rest=f(P, M - 1, 3), opacity=f(P, 1),
                            scaling=f(P, 3), rotation=f(P, 4))


def _header(path):
    with open(path, "rb") as fh:
        data = fh.read()
    return data[:data.index(b"end_header\n")].decode().splitlines()


@pytest.mark.parametrize("M", [1, 4, 16])
def test_round_trip_is_exact(tmp_path, M):
    g = _random(37, M, seed=M)
    p = str(tmp_path / "scene.ply")
    ply.write_ply(p, g)
    h = ply.read_ply(p)
    assert (h.P, h.M) == (37, M)
    for k in ("xyz", "features_dc", "features_rest", "opacity", "scaling", "rotation"):
        np.testing.assert_array_equal(getattr(h, k), getattr(g, k), err_msg=k)


def test_header_matches_the_reference_property_order(tmp_path):
    p = str(tmp_path / "scene.ply")
    ply.write_ply(p, _random(5, 16))
    hdr = _header(p)
    assert hdr[:3] == ["ply", "format binary_little_endian 1.0", "element vertex 5"]
    names = [ln.split()[2] for ln in hdr[3:]]
    assert all(ln.startswith("property float ") for ln in hdr[3:])
    expect = (["x", "y", "z", "nx", "ny", "nz", "f_dc_0", "f_dc_1", "f_dc_2"] + [f"f_rest_{i}" for i in range(45)]
              + ["opacity", "scale_0", "scale_1", "scale_2", "rot_0", "rot_1", "rot_2", "rot_3"])
    assert names == expect
    import os
    assert os.path.getsize(p) == len("\n".join(hdr + ["end_header"]).encode()) + 1 + 5 * len(expect) * 4


def _write_custom(path, fmt, props, rows, extra_elements=""):
    """A PLY file with the given (name, type) vertex properties and row values."""
    hdr = ["ply", f"format {fmt} 1.0", f"element vertex {len(rows)}"]
    hdr += [f"property {t} {n}" for n, t in props]
    hdr += [extra_elements] if extra_elements else []
    hdr += ["end_header"]
    with open(path, "wb") as fh:
        fh.write(("\n".join(hdr) + "\n").encode())
        if fmt == "ascii":
            fh.write(("\n".join(" ".join(repr(float(v)) if t in ("float", "double") else str(int(v))
                                         for v, (_, t) in zip(r, props)) for r in rows) + "\n").encode())
        else:
            order = "<" if fmt == "binary_little_endian" else ">"
            code = {"float": "f4", "double": "f8", "uchar": "u1", "int": "i4"}
            dt = np.dtype([(n, order + code[t]) for n, t in props])
            rec = np.array([tuple(r) for r in rows], dtype=dt)
            fh.write(rec.tobytes())


def _scene_props(M, with_extras=False):
    props = [("x", "float"), ("y", "float"), ("z", "float")]
    if with_extras:
        props += [("red", "uchar"), ("nx", "double")]
    props += [(f"f_dc_{c}", "float") for c in range(3)]
    props += [(f"f_rest_{i}", "float") for i in range(3 * (M - 1))]
    props += [("opacity", "float")] + [(f"scale_{i}", "float") for i in range(3)]
    props += [(f"rot_{i}", "float") for i in range(4)]
    return props


@pytest.mark.parametrize("fmt", ["binary_little_endian", "binary_big_endian", "ascii"])
def test_channel_major_sh_and_other_encodings(tmp_path, fmt):
    M, P = 4, 3
    props = _scene_props(M, with_extras=True)
    rows = []
    for p in range(P):
        row = []
        for name, t in props:
            if name.startswith("f_rest_"):
                i = int(name[7:])
                c, k = divmod(i, M - 1)  # f_rest_{c (M-1) + k} = coefficient k + 1 of channel c
                row.append(100 * p + 10 * (k + 1) + c)
            elif name.startswith("f_dc_"):
                row.append(100 * p + int(name[5:]))
            elif name == "red":
                row.append(7)
            else:
                row.append(p + 0.25)
        rows.append(row)
    path = str(tmp_path / "c.ply")
    _write_custom(path, fmt, props, rows)
    g = ply.read_ply(path)
    assert (g.P, g.M) == (P, M)
    sh = np.concatenate([g.features_dc, g.features_rest], axis=1)  # [P, M, 3] coefficient-major
    for p in range(P):
        for k in range(M):
            for c in range(3):
                assert sh[p, k, c] == 100 * p + 10 * k + c, (p, k, c)
    np.testing.assert_array_equal(g.xyz, np.array([[p + 0.25] * 3 for p in range(P)], np.float32))


def test_elements_after_the_vertices_are_ignored(tmp_path):
    g = _random(4, 1)
    p = str(tmp_path / "s.ply")
    props = _scene_props(1)
    rows = [[*g.xyz[i], *g.features_dc[i, 0], *g.opacity[i], *g.scaling[i], *g.rotation[i]] for i in range(4)]
    _write_custom(p, "binary_little_endian", props, rows, extra_elements="element face 0\nproperty list uchar int vertex_indices")
    h = ply.read_ply(p)
    np.testing.assert_array_equal(h.xyz, g.xyz)
    np.testing.assert_array_equal(h.rotation, g.rotation)


def test_errors(tmp_path):
    bad = tmp_path / "bad.ply"
    bad.write_bytes(b"not a ply\n")
    with pytest.raises(ValueError, match="magic"):
        ply.read_ply(str(bad))
    # missing opacity
    props = [pr for pr in _scene_props(1) if pr[0] != "opacity"]
    p = str(tmp_path / "noop.ply")
    _write_custom(p, "binary_little_endian", props, [[0.0] * len(props)])
    with pytest.raises(ValueError, match="opacity"):
        ply.read_ply(p)
    # 10 f_rest values: not (degree + 1)^2 - 1 coefficients x 3
    props = [pr for pr in _scene_props(1)] + [(f"f_rest_{i}", "float") for i in range(10)]
    p = str(tmp_path / "rest.ply")
    _write_custom(p, "binary_little_endian", props, [[0.0] * len(props)])
    with pytest.raises(ValueError, match="f_rest"):
        ply.read_ply(p)
    # truncated data
    p = str(tmp_path / "trunc.ply")
    ply.write_ply(p, _random(8, 4))
    data = open(p, "rb").read()
    open(p, "wb").write(data[:-10])
    with pytest.raises(ValueError, match="truncated"):
        ply.read_ply(p)


def test_activated_values_follow_the_model_activations():
    g = _random(50, 16, seed=3)
    a = g.activated()
    np.testing.assert_allclose(a.scales, np.exp(g.scaling), rtol=1e-6)
    np.testing.assert_allclose(a.opacities, 1 / (1 + np.exp(-g.opacity.astype(np.float64))), rtol=1e-6)
    np.testing.assert_allclose(np.linalg.norm(a.rotations, axis=1), 1.0, rtol=1e-6)
    assert a.shs.shape == (50, 16, 3)
    np.testing.assert_array_equal(a.shs[:, 0], g.features_dc[:, 0])
    np.testing.assert_array_equal(a.shs[:, 1:], g.features_rest)
