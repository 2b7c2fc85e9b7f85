"""The training session and its schedule (TrainSession, src/train/train.cpp
:474-760; src/train/schedule.cpp).

CPU: the schedule's host parts (resolution_switches, GrowthBudget) against the
reference's schedule.cpp compiled from its sources, and the oracle's
restatements of half_size and neighbour_distances pinned on cases whose
answer is known. GPU: frequency_energy, half_size and initial_cloud on the
device against the reference and the restatements, and a whole session's
schedule (views, sizes, rates, SH degree, densification rounds, the adaptive
image sizes) against the reference's rules.
"""

from __future__ import annotations

import ctypes
import math

import numpy as np
import pytest

from tests.conftest import splat_module
from tests.helpers import to_camera

needs_reference = pytest.mark.skipif("not __import__('oracle.oracle', fromlist=['x']).have_reference()",
                                     reason="the reference sources are not available")

_libm = ctypes.CDLL("libm.so.6")
_libm.logf.restype = ctypes.c_float
_libm.logf.argtypes = [ctypes.c_float]


def host_logf(values) -> np.ndarray:
    """The host C library's logf, as the reference calls std::log on a float."""
    return np.array([_libm.logf(float(v)) for v in np.asarray(values, np.float32).ravel()], np.float32)


@pytest.fixture(scope="module")
def O():
    from oracle import oracle as o

    return o


def spectrum_images(size=64, seed=9):
    import random

    rng = random.Random(seed)
    noise = np.zeros((size, size, 4), np.uint8)
    smooth = np.zeros((size, size, 4), np.uint8)
    for y in range(size):
        for x in range(size):
            value = int(127.5 * (1.0 + math.sin(0.2 * x) * math.cos(0.1 * y)))
            for c in range(3):
                noise[y, x, c] = rng.randrange(256)
                smooth[y, x, c] = value
    return noise.ravel(), smooth.ravel()


# ----------------------------------------------------------------- CPU


@needs_reference
def test_schedule_host_parts_match_the_reference(O):
    # resolution_switches and GrowthBudget, host code in the product, against
    # schedule.cpp compiled from the reference's sources: the same numbers,
    # including the reference test's values (test_densify.cpp:306-335).
    splat = splat_module()
    assert splat.resolution_switches(4.0, 2.0, 1.0) == pytest.approx((0.5, 0.0), abs=1e-12)
    for full, half, quarter in [(4.0, 2.0, 1.0), (10.0, 9.0, 7.5), (10.0, 2.0, 1.0), (8.0, 8.0, 8.0), (5.0, 1.2, 0.7),
                                (3.3, 3.0, 2.9), (1.0, 0.0, 0.0)]:
        assert splat.resolution_switches(full, half, quarter) == O.ref_resolution_switches(full, half, quarter)
    cases = [(1000, 5.0, [], 1.0, 0.0), (1000, 5.0, [], 4.0, 0.0), (1000, 5.0, [1000, 0], 1.0, 1.0), (1000, 8.0, [], 1.0, 1.0),
             (1000, 0.0, [5], 1.0, 1.0), (123457, 4.0, [300, 20000, 7], 2.0, 0.37), (10, 5.0, [1, 2, 3, 4], 4.0, 0.9)]
    for initial, factor, observed, image_factor, progress in cases:
        assert splat.growth_limit(initial, factor, observed, image_factor, progress) == \
            O.ref_growth_limit(initial, factor, observed, image_factor, progress)
    assert splat.growth_limit(1000, 5.0, [], 4.0, 0.0)[0] == 1000 + 4000 // 16


def test_restated_half_size_and_neighbours_are_pinned():
    # The oracle's restatements, on cases whose answer is known: a 2x2 block
    # mean rounded half up; on a lattice of spacing s every point's three
    # nearest neighbours are s away (corners included); a lone far point
    # falls back to the grid's cell size.
    from oracle import oracle as o

    img = np.zeros((2, 4, 4), np.uint8)
    img[0, 0, 0], img[0, 1, 0], img[1, 0, 0], img[1, 1, 0] = 1, 2, 3, 4  # (1+2+3+4+2)/4 = 3
    img[:, 2:, 1] = 255
    out = o.half_size(img.ravel(), 4, 2).reshape(1, 2, 4)
    assert out[0, 0, 0] == 3 and out[0, 1, 1] == 255 and out[0, 0, 1] == 0
    grid = np.stack(np.meshgrid(np.arange(6), np.arange(5), np.arange(4), indexing="ij"), -1).reshape(-1, 3) * 0.25
    d = o.neighbour_distances(grid)
    np.testing.assert_allclose(d, 0.25, rtol=1e-7)


# ----------------------------------------------------------------- GPU


@pytest.mark.gpu
def test_frequency_energy_on_the_gpu_matches_the_reference(splat, O):
    # The spectrum energies within the frequencies of 1/1, 1/2, 1/4 size, on
    # the reference test's noise and smooth images and on camera-sized
    # photos (mirrored to a power of two): within 1e-9 relative of the
    # reference's CPU FFT; the switches they give, within 1e-9.
    noise, smooth = spectrum_images()
    for image, w, h in [(noise, 64, 64), (smooth, 64, 64)]:
        mine = splat.frequency_energy(image, w, h)
        ref = O.ref_frequency_energy(image, w, h)
        np.testing.assert_allclose(mine, ref, rtol=1e-9)
        assert mine[0] > mine[1] > mine[2]
        np.testing.assert_allclose(splat.resolution_switches(*mine), O.ref_resolution_switches(*ref), atol=1e-9)
    assert splat.resolution_switches(*splat.frequency_energy(noise, 64, 64))[0] < 0.25
    assert splat.resolution_switches(*splat.frequency_energy(smooth, 64, 64))[0] > 0.7
    for w, h, seed in [(100, 60, 1), (321, 217, 2), (1237, 822, 3)]:
        target = O.smooth_target(w, h, seed)
        np.testing.assert_allclose(splat.frequency_energy(target, w, h, (1, 2, 4, 8)),
                                   O.ref_frequency_energy(target, w, h, (1, 2, 4, 8)), rtol=1e-9)


@pytest.mark.gpu
def test_half_size_and_initial_cloud_on_the_gpu(splat, O):
    # half_size on the device, bit for bit against the restatement (odd sizes
    # drop the last row and column); initial_cloud with its neighbour search
    # on the device: positions, sizes (the host's logf of the restated
    # distances), DC colour and opacity bit for bit.
    rng = np.random.default_rng(4)
    for w, h in [(64, 48), (101, 77), (1237, 822)]:
        img = rng.integers(0, 256, w * h * 4, dtype=np.uint8)
        np.testing.assert_array_equal(splat.half_size(img, w, h), O.half_size(img, w, h))
    clusters = rng.normal(0.0, 1.0, (40, 3)) * 3.0
    points = np.concatenate([clusters[rng.integers(0, 40, 2500)] + rng.normal(0, 0.05, (2500, 3)),
                             rng.uniform(-10, 10, (12, 3)), np.array([[50.0, 50.0, 50.0]])])
    points[7] = points[8]  # a duplicate: distance 0 to its twin
    colors = rng.integers(0, 256, (points.shape[0], 3), dtype=np.uint8)
    cloud = splat.initial_cloud(points, colors, 2)
    n = points.shape[0]
    np.testing.assert_array_equal(cloud.positions, points.astype(np.float32).ravel())
    expected = host_logf(O.neighbour_distances(points))
    np.testing.assert_array_equal(cloud.scales.reshape(n, 3), np.repeat(expected[:, None], 3, axis=1))
    dc = (colors.astype(np.float32) / np.float32(255.0) - np.float32(0.5)) / np.float32(0.28209479177387814)
    np.testing.assert_array_equal(cloud.sh.reshape(n, 27)[:, :3], dc)
    assert np.all(cloud.sh.reshape(n, 27)[:, 3:] == 0)
    assert np.all(cloud.opacities == host_logf([np.float32(0.1) / (np.float32(1.0) - np.float32(0.1))])[0])
    np.testing.assert_array_equal(cloud.rotations.reshape(n, 4), np.tile([1, 0, 0, 0], (n, 1)).astype(np.float32))


def _small_scene(O, views=8, width=160, height=120, points=3000, seed=3):
    rng = np.random.default_rng(seed)
    cams, images = [], []
    for k in range(views):
        angle = 2 * math.pi * k / views
        eye = np.array([4 * math.sin(angle), -1.0, -4 * math.cos(angle)])
        fx = (width / 2) / math.tan(math.radians(27.5))
        cams.append(splat_module().Camera.look_at(eye, np.zeros(3), np.array([0.0, -1.0, 0.0]), fx, width, height))
        images.append(O.smooth_target(width, height, seed + k))
    pts = rng.normal(0.0, 0.8, (points, 3))
    colors = rng.integers(0, 256, (points, 3), dtype=np.uint8)
    return pts, colors, cams, images


@pytest.mark.gpu
def test_session_schedule_follows_the_reference(splat, O):
    # A 400-iteration session on a small scene: each step trains on the view
    # TrainSession's shuffle gives, at the size the coarse-to-fine schedule
    # gives (quarter until 15 %, half until 35 %), with the position rate's
    # exponential decay and the SH degree's ramp; densification runs at every
    # interval from densifyFrom to densifyUntil and grows the cloud; the loss
    # stays finite and the probe's PSNR improves.
    pts, colors, cams, images = _small_scene(O)
    iterations = 400
    options = splat.SessionOptions(iterations=iterations, sh_degree=2, seed=5, densify_interval=50, score_views=2,
                                   report_every=100, dense_fraction=0.01)
    session = splat.Session(pts, colors, cams, images, extent=4.0, typical_depth=4.5, options=options)
    order = O.ref_view_order(5, len(cams), iterations)
    start, end = 1.6e-4 * 4.0, 1.6e-6 * 4.0
    densify_from, densify_until = min(500, iterations // 20 + 1), iterations // 2
    sh_interval = max(1, min(1000, iterations // 10))
    rounds, psnr = 0, []
    for it in range(1, iterations + 1):
        stats = session.step()
        st = session.state()
        assert st.iteration == it and math.isfinite(stats.loss)
        assert st.view == order[it - 1], f"iteration {it}"
        progress = (it - 1) / (iterations - 1)
        level = 1 if progress < 0.15 else 0 if progress < 0.35 else 2
        assert st.level == level, f"iteration {it}"
        decay = min(max(progress, 0.0), 1.0)
        assert st.position_rate == np.float32(start * math.pow(end / start, decay))
        active = ctypes.c_int32()
        splat._lib.splat_trainer_info(session.trainer()._h, None, None, ctypes.byref(active), None, None, None)
        assert active.value == min((it - 1) // sh_interval, 2)
        if densify_from <= it <= densify_until and it % 50 == 0:
            rounds += 1
        assert st.densify_rounds == rounds
        if st.report_iteration == it:
            psnr.append(st.probe_psnr)
    assert rounds == len([i for i in range(densify_from, densify_until + 1) if i % 50 == 0])
    assert session.state().gaussians != pts.shape[0]
    assert len(psnr) == 4 and psnr[-1] > psnr[0]
    with pytest.raises(splat.SplatError):
        session.step()


@pytest.mark.gpu
def test_adaptive_session_sizes_come_from_the_spectra(splat, O):
    # With the adaptive schedule the coarse levels end where the sampled
    # photos' spectra say (train.cpp:429-437), computed on the GPU: within
    # 1e-9 of the reference's FFT and switches; relocation mode runs.
    pts, colors, cams, images = _small_scene(O, views=16, width=96, height=64)
    options = splat.SessionOptions(iterations=60, adaptive_schedule=True, densify_mode=1, densify_interval=10, report_every=0)
    session = splat.Session(pts, colors, cams, images, extent=4.0, typical_depth=4.5, options=options)
    energy = np.zeros(3)
    for i in range(0, 16, max(16 // 8, 1)):
        energy += O.ref_frequency_energy(images[i], 96, 64)
    expected = O.ref_resolution_switches(*energy)
    st = session.state()
    np.testing.assert_allclose([st.coarse_until[0], st.coarse_until[1]], expected, atol=1e-9)
    while not session.finished():
        session.step()
    assert session.state().densify_rounds > 0
    assert np.isfinite(session.trainer().render(to_camera(O.train_camera(96, 64)))).all()


@pytest.mark.gpu
def test_multi_view_session_takes_the_reference_order_in_groups(splat, O):
    # views_per_step = 4: each step trains on the next four views of the
    # order TrainSession's shuffle gives, in one batched step (64-bit
    # tile|depth keys), at the schedule's size for that iteration.
    pts, colors, cams, images = _small_scene(O)
    iterations, batch = 120, 4
    options = splat.SessionOptions(iterations=iterations, seed=9, views_per_step=batch, densify_interval=40, score_views=2,
                                   report_every=0, dense_fraction=0.01)
    session = splat.Session(pts, colors, cams, images, extent=4.0, typical_depth=4.5, options=options)
    order = O.ref_view_order(9, len(cams), iterations * batch)
    for it in range(1, iterations + 1):
        stats = session.step()
        st = session.state()
        assert math.isfinite(stats.loss)
        assert st.views_in_step == batch and st.view == order[it * batch - 1], f"iteration {it}"
        progress = (it - 1) / (iterations - 1)
        assert st.level == (1 if progress < 0.15 else 0 if progress < 0.35 else 2)
    assert session.state().densify_rounds == len([i for i in range(min(500, iterations // 20 + 1), iterations // 2 + 1)
                                                  if i % 40 == 0])
