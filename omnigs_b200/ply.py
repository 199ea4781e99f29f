"""PLY load/save of a Gaussian scene in the reference's layout (src/gaussian_model.cpp:860-976
loadPly, :978-1060 savePly; the common 3D Gaussian splatting format).

One ``vertex`` element of FP32 properties, in this order when written:
``x y z  nx ny nz  f_dc_0..2  f_rest_0..(3(M-1)-1)  opacity  scale_0..2  rot_0..3``.  The values
are the model's raw parameters: opacity before the sigmoid, log scales, unnormalised rotation
(r, x, y, z).  The SH coefficients are stored channel-major: ``f_dc_c`` is coefficient 0 of
channel c and ``f_rest_{c (M-1) + k}`` coefficient k + 1 of channel c, while the model holds them
coefficient-major ([P, M, 3]; gaussian_model.cpp:948-954 transposes on load, :984-985 on save).
The normals are written as zeros and ignored on load.

``read_ply`` accepts binary (little or big endian) and ASCII files; properties of any numeric PLY
type are converted to float32, extra vertex properties are ignored, and elements other than
``vertex`` are skipped when their size can be computed (scalar properties only).
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

_PLY_TYPES = {
    "char": "i1", "int8": "i1", "uchar": "u1", "uint8": "u1",
    "short": "i2", "int16": "i2", "ushort": "u2", "uint16": "u2",
    "int": "i4", "int32": "i4", "uint": "u4", "uint32": "u4",
    "float": "f4", "float32": "f4", "double": "f8", "float64": "f8",
}


@dataclass
class PlyGaussians:
    """Raw parameters of P Gaussians as the reference's model holds them."""
    xyz: np.ndarray            # [P, 3]
    features_dc: np.ndarray    # [P, 1, 3]
    features_rest: np.ndarray  # [P, M - 1, 3]
    opacity: np.ndarray        # [P, 1], before the sigmoid
    scaling: np.ndarray        # [P, 3], log scales
    rotation: np.ndarray       # [P, 4], unnormalised (r, x, y, z)

    @property
    def P(self) -> int:
        return int(self.xyz.shape[0])

    @property
    def M(self) -> int:
        return 1 + int(self.features_rest.shape[1])

    def activated(self):
        """The rasterizer's inputs (scenes.Gaussians): sigmoid opacity, exp scales, normalised
        rotations (gaussian_model.cpp:54-77), SH [P, M, 3]."""
        from .scenes import Gaussians

        rot = self.rotation.astype(np.float32)
        norm = np.maximum(np.linalg.norm(rot, axis=1, keepdims=True), np.float32(1e-12))
        return Gaussians(
            means3D=np.ascontiguousarray(self.xyz, dtype=np.float32),
            scales=np.exp(self.scaling).astype(np.float32),
            rotations=(rot / norm).astype(np.float32),
            opacities=(1.0 / (1.0 + np.exp(-self.opacity.astype(np.float64)))).astype(np.float32),
            shs=np.ascontiguousarray(np.concatenate([self.features_dc, self.features_rest], axis=1), dtype=np.float32))


def _parse_header(f):
    if f.readline().strip() != b"ply":
        raise ValueError("not a PLY file (missing 'ply' magic)")
    fmt, elements = None, []
    while True:
        line = f.readline()
        if not line:
            raise ValueError("PLY header has no end_header")
        words = line.decode("ascii", "replace").split()
        if not words or words[0] in ("comment", "obj_info"):
            continue
        if words[0] == "end_header":
            break
        if words[0] == "format":
            fmt = words[1]
        elif words[0] == "element":
            elements.append({"name": words[1], "count": int(words[2]), "props": []})
        elif words[0] == "property":
            if not elements:
                raise ValueError("PLY property before any element")
            if words[1] == "list":
                elements[-1]["props"].append((words[4], None))
            else:
                if words[1] not in _PLY_TYPES:
                    raise ValueError(f"unknown PLY property type {words[1]!r}")
                elements[-1]["props"].append((words[2], _PLY_TYPES[words[1]]))
    if fmt not in ("binary_little_endian", "binary_big_endian", "ascii"):
        raise ValueError(f"unsupported PLY format {fmt!r}")
    return fmt, elements


def _read_vertices(path: str) -> dict:
    with open(path, "rb") as f:
        fmt, elements = _parse_header(f)
        names = [e["name"] for e in elements]
        if "vertex" not in names:
            raise ValueError("PLY file has no vertex element")
        vi = names.index("vertex")
        for e in elements[:vi + 1]:
            if any(t is None for _, t in e["props"]):
                raise ValueError(f"PLY element {e['name']!r} before the vertices has list properties")
        vert = elements[vi]
        if fmt == "ascii":
            skip = sum(e["count"] for e in elements[:vi])
            lines = f.read().decode("ascii").splitlines()[skip:skip + vert["count"]]
            data = np.array([ln.split() for ln in lines], dtype=np.float64).reshape(vert["count"], len(vert["props"]))
            return {name: data[:, i] for i, (name, _) in enumerate(vert["props"])}
        order = "<" if fmt == "binary_little_endian" else ">"
        for e in elements[:vi]:
            f.seek(e["count"] * np.dtype([(n, order + t) for n, t in e["props"]]).itemsize, 1)
        dt = np.dtype([(n, order + t) for n, t in vert["props"]])
        buf = f.read(dt.itemsize * vert["count"])
        if len(buf) != dt.itemsize * vert["count"]:
            raise ValueError("PLY file is truncated")
        rec = np.frombuffer(buf, dtype=dt, count=vert["count"])
        return {n: rec[n] for n in dt.names}


def read_ply(path: str) -> PlyGaussians:
    """Loads a scene written by the reference's savePly (or any file with those properties)."""
    props = _read_vertices(path)

    def cols(names):
        missing = [n for n in names if n not in props]
        if missing:
            raise ValueError(f"PLY vertex element lacks properties {missing}")
        return np.stack([np.asarray(props[n], dtype=np.float32) for n in names], axis=1)

    n_rest = 0
    while f"f_rest_{n_rest}" in props:
        n_rest += 1
    m = n_rest // 3 + 1
    if n_rest % 3 or int(round(math.sqrt(m))) ** 2 != m:
        raise ValueError(f"{n_rest} f_rest properties do not make (degree + 1)^2 - 1 coefficients x 3 channels")
    xyz = cols(["x", "y", "z"])
    P = xyz.shape[0]
    f_dc = cols([f"f_dc_{c}" for c in range(3)]).reshape(P, 1, 3)
    f_rest = (cols([f"f_rest_{i}" for i in range(n_rest)]).reshape(P, 3, m - 1).transpose(0, 2, 1)
              if n_rest else np.zeros((P, 0, 3), np.float32))
    return PlyGaussians(xyz=xyz, features_dc=np.ascontiguousarray(f_dc),
                        features_rest=np.ascontiguousarray(f_rest, dtype=np.float32),
                        opacity=cols(["opacity"]), scaling=cols([f"scale_{i}" for i in range(3)]),
                        rotation=cols([f"rot_{i}" for i in range(4)]))


def write_ply(path: str, g: PlyGaussians) -> None:
    """Writes ``g`` as binary little-endian PLY with the reference's property names and order."""
    P, M = g.P, g.M
    names = (["x", "y", "z", "nx", "ny", "nz"] + [f"f_dc_{c}" for c in range(3)]
             + [f"f_rest_{i}" for i in range(3 * (M - 1))] + ["opacity"]
             + [f"scale_{i}" for i in range(3)] + [f"rot_{i}" for i in range(4)])
    f_rest = np.asarray(g.features_rest, np.float32).reshape(P, M - 1, 3).transpose(0, 2, 1).reshape(P, -1)
    data = np.concatenate([np.asarray(g.xyz, np.float32).reshape(P, 3), np.zeros((P, 3), np.float32),
                           np.asarray(g.features_dc, np.float32).reshape(P, 3), f_rest,
                           np.asarray(g.opacity, np.float32).reshape(P, 1),
                           np.asarray(g.scaling, np.float32).reshape(P, 3),
                           np.asarray(g.rotation, np.float32).reshape(P, 4)], axis=1).astype("<f4")
    assert data.shape[1] == len(names)
    header = ["ply", "format binary_little_endian 1.0", f"element vertex {P}"]
    header += [f"property float {n}" for n in names] + ["end_header"]
    with open(path, "wb") as f:
        f.write(("\n".join(header) + "\n").encode("ascii"))
        f.write(np.ascontiguousarray(data).tobytes())
