"""CPU tests: the oracle pinned against the reference's own implementation.

  * The reference's FP64 twin (src/train/reference.cpp, compiled unmodified into
    oracle/_ref) against central finite differences, as the reference's own
    tests do (tests/test_train.cpp:86-142).
  * This repository's FP32 restatement (oracle/splat_oracle.c) against that FP64
    twin with the reference's GPU tolerances (tests/test_train.cpp:218-293).
  * The deterministic exp/log against a double-precision libm.
  * The committed golden fixtures (tests/golden/) against both, so the oracle
    is pinned where the reference tree is absent too.
"""
from __future__ import annotations

import numpy as np
import pytest

from tests.conftest import check_close

needs_reference = pytest.mark.skipif("not __import__('oracle.oracle', fromlist=['x']).have_reference()",
                                     reason="the reference's FP64 twin was not built here")


@pytest.fixture(scope="module")
def O():
    from oracle import oracle

    return oracle


def _functional(O, cloud, view, adjoint):
    rgb, _, _ = O.ref_render(cloud, view, no_cutoffs=True)
    return float((adjoint.reshape(-1, 3) * rgb).sum())


def _finite_differences(O, cloud, member: str, view, adjoint, step: float):
    values = getattr(cloud, member)
    out = np.zeros(values.size)
    for i in range(values.size):
        original = values[i]
        values[i] = original + np.float32(step)
        up = float(values[i])
        high = _functional(O, cloud, view, adjoint)
        values[i] = original - np.float32(step)
        down = float(values[i])
        low = _functional(O, cloud, view, adjoint)
        values[i] = original
        out[i] = (high - low) / (up - down)
    return out


@needs_reference
def test_reference_gradients_match_finite_differences(O):
    # tests/test_train.cpp:86-113.
    view = O.train_camera(40, 32)
    adjoint = O.normal_adjoint(9, 40 * 32)
    cloud = O.random_cloud(12, 0, 3)
    g = O.ref_gradients(cloud, view, adjoint, no_cutoffs=True)
    for member in ("positions", "scales", "rotations", "opacities"):
        check_close(getattr(g, member), _finite_differences(O, cloud, member, view, adjoint, 2e-3), member, 0.999, 0.01)
    degree3 = O.random_cloud(12, 3, 6)
    g3 = O.ref_gradients(degree3, view, adjoint, no_cutoffs=True)
    check_close(g3.positions, _finite_differences(O, degree3, "positions", view, adjoint, 2e-3), "positions, degree 3",
                0.999, 0.01)
    check_close(g3.sh, _finite_differences(O, degree3, "sh", view, adjoint, 2e-3), "sh degree 3", 0.999, 0.01)


@needs_reference
def test_reference_loss_adjoint_matches_finite_differences(O):
    # tests/test_train.cpp:115-142.
    rng = np.random.default_rng(21)
    w, h = 18, 14
    rgb = rng.uniform(0.1, 0.9, (w * h, 3))
    target = O.smooth_target(w, h, 5)
    for lam in (1.0, 0.2):
        base = O.ref_loss(rgb, w, h, target, lam)
        analytic, numeric = [], []
        for i in range(0, w * h, 7):
            for c in range(3):
                changed = rgb.copy()
                changed[i, c] += 1e-5
                high = O.ref_loss(changed, w, h, target, lam)[0]
                changed[i, c] -= 2e-5
                low = O.ref_loss(changed, w, h, target, lam)[0]
                numeric.append((high - low) / 2e-5)
                analytic.append(base[3][i, c])
        check_close(analytic, numeric, "pure SSIM" if lam == 1.0 else "L1 + SSIM", 0.9999, 0.001)


def _oracle_pipeline(O, cloud, view, sh_storage="f32"):
    splats, reach, keys = O.preprocess(cloud, view, sh_storage=sh_storage)
    order = O.stable_order(keys)
    tiles, values = O.bin_entries(splats, reach, keys[order], order, view)
    by_tile = O.stable_order(tiles)
    tiles, values = tiles[by_tile], values[by_tile]
    tc = ((view.width + 15) // 16) * ((view.height + 15) // 16)
    ranges = O.ranges(tiles, tc)
    image, stops = O.forward(splats, values, ranges, view, degree=cloud.sh_degree)
    return splats, reach, keys, tiles, values, ranges, image, stops


@needs_reference
@pytest.mark.parametrize("case", [(100, 75, 300, 1, 7, 0.0), (80, 60, 400, 1, 17, 5.0), (64, 48, 200, 3, 29, 0.0)])
def test_restatement_forward_matches_reference(O, case):
    # tests/test_train.cpp:218-235 and :353-370: max |rgb| < 1e-3, |log T| < 1e-2.
    w, h, n, degree, seed, opacity = case
    view = O.train_camera(w, h)
    cloud = O.random_cloud(n, degree, seed)
    if opacity:
        cloud.opacities[:] = opacity
    rgb, logT, stop = O.ref_render(cloud, view)
    *_, image, stops = _oracle_pipeline(O, cloud, view)
    assert np.abs(image[:, :3] - rgb).max() < 1e-3
    assert np.abs(image[:, 3] - logT).max() < 1e-2


@needs_reference
def test_restatement_loss_and_backward_match_reference(O):
    # tests/test_train.cpp:256-293 at the restatement's level: loss within 1e-3,
    # raw sums carried through the reference's own chain rule would be needed for
    # parameter gradients, so the screen-space colour sums are compared instead
    # with the FP64 twin's SH gradient at degree 0 (basis C0 times the colour sum).
    view = O.train_camera(72, 56)
    target = O.smooth_target(72, 56, 11)
    cloud = O.random_cloud(60, 0, 13)
    rgb, _, _ = O.ref_render(cloud, view)
    loss, l1, ssim, adjoint = O.ref_loss(rgb, 72, 56, target, 0.2)
    splats, reach, keys, tiles, values, ranges, image, stops = _oracle_pipeline(O, cloud, view)
    adj, ssim_sum, l1_sum = O.loss(image, target, view, 0.2)
    P = 72 * 56
    assert abs(l1_sum / (3 * P) - l1) < 1e-3 and abs(ssim_sum / (3 * P) - ssim) < 1e-3
    np.testing.assert_allclose(adj[:, :3], adjoint, atol=1e-7, rtol=1e-3)
    cpu = O.ref_gradients(cloud, view, adjoint)
    for fixed in (False, True):
        raw = O.backward(splats, values, ranges, view, image, adj, stops, fixed, cloud.count)
        colour = raw[:, 6:9].astype(np.float64)
        if fixed:
            colour /= float(np.float32(3.0) * np.float32(72) * np.float32(56) * np.float32(64.0))
        visible = keys != 0xFFFFFFFF
        colour_grad = np.where(splats[:, 4:7] > 0, colour, 0.0) * 0.28209479177387814
        check_close(colour_grad[visible].ravel(), cpu.sh.reshape(-1, 3)[visible].ravel(), "sh dc", 0.999,
                    0.1 if fixed else 0.02)


def test_detmath_accuracy(O):
    x = np.linspace(-80, 80, 400_001).astype(np.float32)
    e, _ = O.detmath(x)
    ref = np.exp(x.astype(np.float64))
    assert (np.abs(e - ref) / ref).max() < 2.5e-7
    y = np.concatenate([np.linspace(1e-3, 1.0, 200_001), np.linspace(1.0, 1e4, 200_001)]).astype(np.float32)
    _, lg = O.detmath(y)
    ref = np.log(y.astype(np.float64))
    assert np.abs(lg - ref).max() < 2e-6
    assert np.all(np.abs(lg - ref) <= 2.5e-7 * np.maximum(np.abs(ref), 1.0))
    e, _ = O.detmath(np.array([np.nan, -1e30, 1e30], np.float32))
    assert np.isnan(e[0]) and 0 < e[1] < 1e-37 and e[2] > 1e38


def test_fixtures_follow_the_reference_helpers(O):
    c = O.random_cloud(3, 1, 7)
    assert c.positions.size == 9 and c.sh.size == 36
    assert np.all(np.abs(c.positions[0::3]) <= 1.4) and np.all((c.positions[2::3] >= 3) & (c.positions[2::3] <= 6))
    t = O.smooth_target(8, 4, 11)
    assert t.size == 128 and np.all(t[3::4] == 255)
    # std::mt19937(5489)'s 10000th output is 4123659995 (C++ standard, [rand.predef]).
    assert int(O.mt19937(5489, 10000)[-1]) == 4123659995


def test_golden_fixtures(O):
    from tests.golden.check import check_golden

    check_golden(O)


@needs_reference
def test_reference_marked_pixels_count_what_the_image_gets_wrong(O):
    # reference.cpp:248-276, the expectation of Trainer::score_view's test
    # (tests/test_train.cpp:588-621): a Gaussian's count is at most the
    # pixels of the image, every count is whole, a share above 1 marks
    # nothing and a lower share marks at least as much.
    view = O.train_camera(72, 56)
    target = O.smooth_target(72, 56, 43)
    cloud = O.random_cloud(60, 1, 47)
    half = O.ref_marked_pixels(cloud, view, target, 0.5)
    assert half.sum() > 0.0
    assert np.all(half == np.round(half)) and np.all(half <= 72 * 56)
    assert O.ref_marked_pixels(cloud, view, target, 1.5).sum() == 0.0
    assert np.all(O.ref_marked_pixels(cloud, view, target, 0.25) >= half)
