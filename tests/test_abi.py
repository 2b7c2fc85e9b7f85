"""CPU tests of the drop-in boundary: the C-ABI library loads without a GPU,
exports every entry point include/*.h declares, and refuses bad arguments and
unsupported options before it touches a device (the reference throws for
these: trainer.cpp:174,276,571)."""
from __future__ import annotations

import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

from tests.conftest import ROOT, splat_module


def declared_functions() -> list[str]:
    """Entry points of the headers that declare an extern "C" ABI (header-only
    inline helpers such as splat_detmath.h export nothing)."""
    names = []
    for header in sorted((ROOT / "include").glob("*.h")):
        text = header.read_text()
        if 'extern "C"' not in text:
            continue
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[a-z_0-9]+\s*\**\s*(splat_[a-z_0-9]+)\s*\(", text, flags=re.M):
            names.append(m.group(1))
    return names


def test_library_exports_every_declared_entry_point():
    lib = ctypes.CDLL(str(ROOT / "vibe-splat_b200" / "libsplat_b200.so"))
    public = declared_functions()
    assert len(public) >= 29
    missing = [n for n in public if not hasattr(lib, n)]
    assert not missing, missing


def test_defaults_are_the_reference_defaults():
    s = splat_module()
    o = s._Options()
    s._lib.splat_trainer_options_default(ctypes.byref(o))
    assert abs(o.lambda_ssim - 0.2) < 1e-7 and abs(o.near_plane - 0.01) < 1e-9 and o.selective_adam == 1
    assert o.memory_budget == 2**64 - 1 and o.force_fixed_point == 0
    assert o.forward_pixels_per_thread == 1 and o.backward_pixels_per_thread == 2 and o.digit_bits == 8
    r = s._Rates()
    s._lib.splat_learning_rates_default(ctypes.byref(r))
    got = [r.position, r.scale, r.rotation, r.opacity, r.sh, r.sh_rest_scale, r.trust_region]
    np.testing.assert_allclose(got, [1.6e-4, 0.005, 0.001, 0.05, 0.025, 0.05, 0.0], rtol=1e-6)
    # DensifyOptions and RelocateOptions (densify.hpp:23-50,87-91).
    d = s._DensifyOptions()
    s._lib.splat_densify_options_default(ctypes.byref(d))
    assert (d.prune_large, d.max_gaussians, d.scored_views, d.transparent_share) == (0, 2**64 - 1, 0, 1.0)
    assert (d.explore_splits, d.explore_seeds, d.edge_split) == (0, 0, 0)
    np.testing.assert_allclose([d.gradient_threshold, d.dense_scale, d.prune_opacity, d.max_screen_radius, d.max_world_scale,
                                d.split_threshold, d.min_marked_pixels], [2e-4, 0.0, 0.005, 20.0, 0.0, 0.0, 5.0], rtol=1e-6)
    m = s._RelocateOptions()
    s._lib.splat_relocate_options_default(ctypes.byref(m))
    assert abs(m.min_opacity - 0.005) < 1e-9 and m.growth == 0.05 and m.max_gaussians == 2**64 - 1
    py = s.DensifyOptions()._c()
    assert [getattr(py, f) for f, _ in d._fields_] == [getattr(d, f) for f, _ in d._fields_]


def _tiny_cloud(s, n=4, degree=0):
    f = 3 * (degree + 1) ** 2
    return s.GaussianCloud(degree, np.zeros(n * 3, np.float32), np.zeros(n * 3, np.float32),
                           np.tile(np.array([1, 0, 0, 0], np.float32), n), np.zeros(n, np.float32),
                           np.zeros(n * f, np.float32))


def test_empty_cloud_is_refused():
    s = splat_module()
    empty = _tiny_cloud(s, 0)
    with pytest.raises(RuntimeError, match="empty"):
        s.Trainer(empty)
    c, keep = empty._c()
    h = s._P()
    status = s._lib.splat_trainer_create(ctypes.byref(c), None, ctypes.byref(h))
    assert status == s.SPLAT_ERR_INVALID and b"empty" in s._lib.splat_last_error()


def test_unsupported_options_are_refused_not_emulated():
    s = splat_module()
    for opts in (s.TrainerOptions(mip_filter_2d=True), s.TrainerOptions(position_noise=0.1),
                 s.TrainerOptions(pose_gradients=True), s.TrainerOptions(blend_lists=True, force_fixed_point=True)):
        with pytest.raises(s.UnsupportedOption):
            s.Trainer(_tiny_cloud(s), opts)


def test_inconsistent_cloud_is_refused():
    s = splat_module()
    bad = _tiny_cloud(s)
    bad.sh = np.zeros(5, np.float32)
    with pytest.raises(RuntimeError, match="inconsistent"):
        s.Trainer(bad)
    bad = _tiny_cloud(s)
    bad.sh_degree = 4
    with pytest.raises(RuntimeError):
        s.Trainer(bad)


def test_bad_digit_width_is_refused():
    s = splat_module()
    with pytest.raises(s.SplatError) as e:
        s.Trainer(_tiny_cloud(s), s.TrainerOptions(digit_bits=5))
    assert e.value.status == s.SPLAT_ERR_INVALID


def test_stage_entry_points_check_arguments():
    s = splat_module()
    with pytest.raises(s.SplatError):
        s.radix_sort_device(0, 0, 0, 0, 10, 0)
    with pytest.raises(s.SplatError):
        s.radix_sort_device(0, 0, 0, 0, 10, 65, key_bytes=8)
    # One key needs no work and touches no memory.
    s.radix_sort_device(0, 0, 0, 0, 1, 32)


def test_sorts_refuse_unaligned_arrays():
    # Vector loads and bulk copies need 16-byte aligned arrays; the check comes
    # before any device work.
    s = splat_module()
    for key_bytes in (4, 8):
        with pytest.raises(s.SplatError, match="16-byte aligned"):
            s.radix_sort_device(0x1004, 0x2000, 0x3000, 0x4000, 10, 16, key_bytes=key_bytes)
    fn = s._lib.splat_radix_sort_u32_noalloc
    assert fn(s._P(0x1000), s._P(0x2008), s._P(0x3000), s._P(0x4000), 10, 16, 8, None) == s.SPLAT_ERR_INVALID
    assert "16-byte aligned" in s._lib.splat_last_error().decode()


def test_cpp_face_compiles_links_and_draws_as_the_reference(tmp_path):
    # include/splat_trainer.hpp, the reference-shaped C++ class over the ABI,
    # compiles as C++20, links against the library and runs its host-only
    # part: the generator's picks, which the CPU reference draws the same.
    import shutil
    import subprocess

    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("no C++ compiler")
    source = tmp_path / "face.cpp"
    source.write_text('#include "splat_trainer.hpp"\n#include <cstdio>\n'
                      "int main() {\n  splat_b200::Rng rng(8);\n"
                      "  for (int k = 0; k < 5; ++k) std::printf(\"%zu \", rng.pick(1000));\n"
                      "  splat_densify_options d = splat_b200::default_densify_options();\n"
                      "  splat_relocate_options r = splat_b200::default_relocate_options();\n"
                      "  splat_session_options so = splat_b200::default_session_options();\n"
                      "  if (so.iterations != 15000) return 1;\n"
                      "  std::printf(\"%g %g\\n\", d.gradient_threshold, r.growth);\n}\n")
    lib = ROOT / "vibe-splat_b200"
    exe = tmp_path / "face"
    subprocess.run([gxx, "-std=c++20", "-I", str(ROOT / "include"), str(source), "-L", str(lib), "-lsplat_b200",
                    f"-Wl,-rpath,{lib}", "-o", str(exe)], check=True, capture_output=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()
    splat = splat_module()
    rng = splat.Rng(8)
    assert [int(v) for v in out[:5]] == [rng.pick(1000) for _ in range(5)]
    assert float(out[5]) == pytest.approx(2e-4) and float(out[6]) == pytest.approx(0.05)
