"""CPU tests of the .ply reader and writer (host code of the library, no
device needed): the reference's own cases (tests/test_ply.cpp:20-82), and the
files against the reference's load_ply / save_ply (gaussian_cloud.cpp:236-365)
compiled from its sources, byte for byte."""
from __future__ import annotations

import math

import numpy as np
import pytest

from tests.conftest import splat_module

needs_reference = pytest.mark.skipif("not __import__('oracle.oracle', fromlist=['x']).have_reference()",
                                     reason="the reference's FP64 twin was not built here")


@pytest.fixture(scope="module")
def S():
    return splat_module()


def sample_cloud(S, degree: int, n: int = 37):
    # tests/test_ply.cpp:22-28: every attribute a different, exactly stored value.
    coeffs = (degree + 1) ** 2
    positions = np.arange(n * 3, dtype=np.float32) * np.float32(0.25)
    scales = -np.arange(n * 3, dtype=np.float32) * np.float32(0.01)
    rotations = (np.arange(n * 4) % 5).astype(np.float32)
    opacities = np.arange(n, dtype=np.float32) - np.float32(10.0)
    sh = np.array([math.sin(float(np.float32(i))) for i in range(n * coeffs * 3)], np.float32)
    return S.GaussianCloud(degree, positions, scales, rotations, opacities, sh)


def same_cloud(a, b) -> None:
    assert a.sh_degree == b.sh_degree
    for name in ("positions", "scales", "rotations", "opacities", "sh"):
        np.testing.assert_array_equal(np.asarray(getattr(a, name), np.float32), np.asarray(getattr(b, name), np.float32), name)


@pytest.mark.parametrize("degree", [0, 1, 2, 3])
def test_save_and_load_round_trip_every_attribute(S, tmp_path, degree):
    cloud = sample_cloud(S, degree)
    path = tmp_path / "roundtrip.ply"
    S.save_ply(cloud, path)
    loaded = S.load_ply(path)
    assert loaded.size() == cloud.size()
    same_cloud(loaded, cloud)


def test_rest_coefficients_are_channel_major_in_the_file(S, tmp_path):
    # tests/test_ply.cpp:46-71: one Gaussian of degree 1 in an ASCII file with a
    # comment and a face element after the vertices.
    path = tmp_path / "ascii.ply"
    header = ["ply", "format ascii 1.0", "comment written by a test", "element vertex 1"]
    header += [f"property float {p}" for p in ("x", "y", "z", "f_dc_0", "f_dc_1", "f_dc_2")]
    header += [f"property float f_rest_{i}" for i in range(9)]
    header += [f"property float {p}" for p in ("opacity", "scale_0", "scale_1", "scale_2", "rot_0", "rot_1", "rot_2", "rot_3")]
    header += ["element face 0", "property list uchar int vertex_indices", "end_header"]
    path.write_text("\n".join(header) + "\n1 2 3  0.1 0.2 0.3  10 11 12 20 21 22 30 31 32  0.5  -1 -2 -3  1 0 0 0\n")
    c = S.load_ply(path)
    assert c.size() == 1 and c.sh_degree == 1
    np.testing.assert_array_equal(c.positions, np.float32([1, 2, 3]))
    assert c.sh[0 * 3 + 0] == np.float32(0.1)  # DC red
    assert c.sh[1 * 3 + 0] == 10.0  # coefficient 1 red
    assert c.sh[1 * 3 + 1] == 20.0  # coefficient 1 green
    assert c.sh[3 * 3 + 2] == 32.0  # coefficient 3 blue
    assert c.opacities[0] == 0.5
    np.testing.assert_array_equal(c.scales, np.float32([-1, -2, -3]))


def test_loader_refuses_files_that_are_not_splats(S, tmp_path):
    # tests/test_ply.cpp:73-82: a mesh's vertices have no splat properties.
    path = tmp_path / "mesh.ply"
    path.write_text("ply\nformat ascii 1.0\nelement vertex 1\nproperty float x\nproperty float y\nproperty float z\n"
                    "end_header\n0 0 0\n")
    with pytest.raises(S.SplatError, match="missing property: "):
        S.load_ply(path)
    with pytest.raises(S.SplatError):
        S.load_ply(tmp_path / "absent.ply")
    (tmp_path / "text.ply").write_text("not a ply file\n")
    with pytest.raises(S.SplatError, match="not a PLY"):
        S.load_ply(tmp_path / "text.ply")


def test_binary_properties_of_other_types_are_converted(S, tmp_path):
    # A binary file with a double, a uchar and an unused int16 among the floats.
    names = ["x", "y", "z", "f_dc_0", "f_dc_1", "f_dc_2", "opacity", "scale_0", "scale_1", "scale_2",
             "rot_0", "rot_1", "rot_2", "rot_3"]
    types = {"x": ("double", "<f8"), "opacity": ("uchar", "u1"), "extra": ("short", "<i2")}
    columns = names[:3] + ["extra"] + names[3:]
    header = "ply\nformat binary_little_endian 1.0\nelement vertex 2\n"
    header += "".join(f"property {types.get(c, ('float', '<f4'))[0]} {c}\n" for c in columns) + "end_header\n"
    dtype = np.dtype([(c, types.get(c, ("float", "<f4"))[1]) for c in columns])
    rows = np.zeros(2, dtype)
    for i in range(2):
        for j, c in enumerate(columns):
            rows[c][i] = (i + 1) * 10 + j
    path = tmp_path / "types.ply"
    path.write_bytes(header.encode() + rows.tobytes())
    c = S.load_ply(path)
    assert c.size() == 2 and c.sh_degree == 0
    np.testing.assert_array_equal(c.positions.reshape(2, 3)[:, 0], np.float32([10, 20]))
    np.testing.assert_array_equal(c.opacities, np.float32([rows["opacity"][0], rows["opacity"][1]]))
    np.testing.assert_array_equal(c.sh.reshape(2, 3)[:, 0], rows["f_dc_0"].astype(np.float32))


@needs_reference
@pytest.mark.parametrize("degree", [0, 1, 2, 3])
def test_files_equal_the_references(S, tmp_path, degree):
    from oracle import oracle as O

    cloud = sample_cloud(S, degree, n=211)
    ref_cloud = O.Cloud(degree, cloud.positions, cloud.scales, cloud.rotations, cloud.opacities, cloud.sh)
    ours, theirs = tmp_path / "ours.ply", tmp_path / "theirs.ply"
    S.save_ply(cloud, ours)
    O.ref_save_ply(ref_cloud, theirs)
    assert ours.read_bytes() == theirs.read_bytes()
    # Each reader on the other's file.
    same_cloud(S.load_ply(theirs), cloud)
    back = O.ref_load_ply(ours)
    same_cloud(S.GaussianCloud(back.sh_degree, back.positions, back.scales, back.rotations, back.opacities, back.sh), cloud)
