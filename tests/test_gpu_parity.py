"""GPU parity: the CUDA step against the reference's FP64 twin (with the
reference's own tolerances, tests/test_train.cpp) and against the FP32 CPU
restatement (bit for bit on integer results, given the device's own projected
splats). Every call goes through the C ABI."""
from __future__ import annotations

import itertools
import math

import numpy as np
import pytest

from tests.conftest import check_close
from tests.helpers import device_projection, oracle_entries, tile_count, to_camera, to_cloud

pytestmark = pytest.mark.gpu


def _run_oracle_forward(oracle, trainer, cloud, view, n):
    splats, reach, keys = device_projection(trainer, n)
    tiles, values, ranges = oracle_entries(oracle, splats, reach, keys, view)
    image, stops = oracle.forward(splats, values, ranges, view)
    return splats, reach, keys, tiles, values, ranges, image, stops


@pytest.mark.parametrize("sort_form", [0, 1])
def test_forward_matches_reference_and_restatement(splat, oracle, sort_form):
    # tests/test_train.cpp:218-235: 100x75, 300 Gaussians, degree 1, seed 7.
    view = oracle.train_camera(100, 75)
    cloud = oracle.random_cloud(300, 1, 7)
    opts = splat.TrainerOptions(sort_form=sort_form)
    trainer = splat.Trainer(to_cloud(cloud), opts)
    gpu = trainer.render(to_camera(view)).reshape(-1, 4)
    rgb, logT, _ = oracle.ref_render(cloud, view)
    worst = np.abs(gpu[:, :3] - rgb).max()
    worst_log = np.abs(gpu[:, 3] - logT).max()
    print(f"  forward: worst difference from CPU {worst:.6f}, log transmittance {worst_log:.6f}")
    assert worst < 1e-3 and worst_log < 1e-2

    # Bit for bit against the restatement, given the device's own splats.
    n = cloud.count
    splats, reach, keys, tiles, values, ranges, image, stops = _run_oracle_forward(oracle, trainer, cloud, view, n)
    dev_ranges = trainer.debug_download(splat.DEBUG_RANGES, np.uint32).reshape(-1, 2)[: tile_count(view)]
    dev_values = trainer.debug_download(splat.DEBUG_ENTRY_VALUES, np.uint32)
    dev_keys = trainer.debug_download(splat.DEBUG_ENTRY_KEYS, np.uint64 if sort_form == 1 else np.uint32)
    assert dev_values.size == values.size
    np.testing.assert_array_equal(dev_values, values)
    dev_tiles = (dev_keys >> np.uint64(32)).astype(np.uint32) if sort_form == 1 else dev_keys
    np.testing.assert_array_equal(dev_tiles, tiles)
    np.testing.assert_array_equal(dev_ranges, ranges)
    np.testing.assert_array_equal(trainer.debug_download(splat.DEBUG_STOPS, np.uint32), stops)
    np.testing.assert_array_equal(gpu.view(np.uint32), image.view(np.uint32))


def test_preprocess_matches_restatement(splat, oracle):
    view = oracle.train_camera(100, 75)
    cloud = oracle.random_cloud(300, 3, 21)
    trainer = splat.Trainer(to_cloud(cloud), splat.TrainerOptions(sh_storage=splat.SH_F32))
    trainer.render(to_camera(view))
    splats, reach, keys = device_projection(trainer, cloud.count)
    o_splats, o_reach, o_keys = oracle.preprocess(cloud, view, sh_storage="f32")
    np.testing.assert_array_equal(keys, o_keys)
    visible = keys != 0xFFFFFFFF
    assert visible.sum() > 100
    np.testing.assert_array_equal(splats[visible].view(np.uint32), o_splats[visible].view(np.uint32))
    np.testing.assert_array_equal(reach[visible].view(np.uint32), o_reach[visible].view(np.uint32))


@pytest.mark.parametrize("fixed", [False, True])
def test_loss_and_gradients_match_reference(splat, oracle, fixed):
    # tests/test_train.cpp:256-293: 72x56, 60 Gaussians degree 1 seed 13,
    # target seed 11, penalties 0.01; float atomics cosine > 0.999 and length
    # within 2%, fixed point cosine > 0.97 and length within 10%.
    view = oracle.train_camera(72, 56)
    target = oracle.smooth_target(72, 56, 11)
    cloud = oracle.random_cloud(60, 1, 13)
    rgb, _, _ = oracle.ref_render(cloud, view)
    loss, l1, ssim, adjoint = oracle.ref_loss(rgb, 72, 56, target, 0.2)
    cpu = oracle.ref_gradients(cloud, view, adjoint, opacity_reg=0.01, scale_reg=0.01)
    opts = splat.TrainerOptions(force_fixed_point=fixed, opacity_reg=0.01, scale_reg=0.01)
    trainer = splat.Trainer(to_cloud(cloud), opts)
    assert trainer.uses_fixed_point() == fixed
    stats = trainer.compute_gradients(to_camera(view), target)
    assert abs(stats.loss - loss) < 1e-3
    assert abs(stats.l1 - l1) < 1e-3
    assert abs(stats.ssim - ssim) < 1e-3
    g = trainer.gradients()
    cos, ratio = (0.97, 0.1) if fixed else (0.999, 0.02)
    check_close(g.positions, cpu.positions, "positions", cos, ratio)
    check_close(g.scales, cpu.scales, "scales", cos, ratio)
    check_close(g.rotations, cpu.rotations, "rotations", cos, ratio)
    check_close(g.opacities, cpu.opacities, "opacities", cos, ratio)
    check_close(g.sh, cpu.sh, "sh", cos, ratio)


def test_fixed_point_sums_are_bit_exact(splat, oracle):
    # Fixed-point sums: the same integers as the restatement's per-warp
    # quantisation, given the device's splats, image, stops and adjoint.
    view = oracle.train_camera(80, 60)
    target = oracle.smooth_target(80, 60, 19)
    cloud = oracle.random_cloud(400, 1, 17)
    cloud.opacities[:] = 2.0
    trainer = splat.Trainer(to_cloud(cloud), splat.TrainerOptions(force_fixed_point=True))
    trainer.compute_gradients(to_camera(view), target)
    n = cloud.count
    splats, reach, keys = device_projection(trainer, n)
    tiles, values, ranges = oracle_entries(oracle, splats, reach, keys, view)
    image = trainer.debug_download(splat.DEBUG_IMAGE, np.float32).reshape(-1, 4)
    stops = trainer.debug_download(splat.DEBUG_STOPS, np.uint32)
    adjoint = trainer.debug_download(splat.DEBUG_ADJOINT, np.float32).reshape(-1, 4)
    o_image, o_stops = oracle.forward(splats, values, ranges, view)
    np.testing.assert_array_equal(image.view(np.uint32), o_image.view(np.uint32))
    np.testing.assert_array_equal(stops, o_stops)
    raw = trainer.debug_download(splat.DEBUG_RAW, np.int32)[: n * 16].reshape(n, 16)
    o_raw = oracle.backward(splats, values, ranges, view, image, adjoint, stops, True, n)
    assert np.count_nonzero(raw) > 100
    np.testing.assert_array_equal(raw[:, :14], o_raw[:, :14])
    # The adjoint against the restatement's loss (floats, order of sums differs).
    o_adj, _, _ = oracle.loss(image, target, view, 0.2)
    np.testing.assert_allclose(adjoint[:, :3], o_adj[:, :3], rtol=1e-4, atol=1e-9)


def test_early_stop_case(splat, oracle):
    # tests/test_train.cpp:353-403: opaque Gaussians, most pixels stop early.
    view = oracle.train_camera(80, 60)
    target = oracle.smooth_target(80, 60, 19)
    cloud = oracle.random_cloud(400, 1, 17)
    cloud.opacities[:] = 5.0
    rgb, logT, stop = oracle.ref_render(cloud, view)
    assert (stop > 0).sum() > stop.size // 10
    loss, _, _, adjoint = oracle.ref_loss(rgb, 80, 60, target, 0.2)
    cpu = oracle.ref_gradients(cloud, view, adjoint)
    contributions = oracle.ref_contributions(cloud, view)
    for fixed in (False, True):
        trainer = splat.Trainer(to_cloud(cloud), splat.TrainerOptions(force_fixed_point=fixed))
        gpu = trainer.render(to_camera(view)).reshape(-1, 4)
        assert np.abs(gpu[:, :3] - rgb).max() < 1e-3
        assert np.abs(gpu[:, 3] - logT).max() < 1e-2
        stats = trainer.compute_gradients(to_camera(view), target)
        assert abs(stats.loss - loss) < 1e-3
        g = trainer.gradients()
        d = trainer.densify_stats()
        cos, ratio = (0.97, 0.1) if fixed else (0.999, 0.02)
        check_close(d.contribution, contributions, "contribution", cos, ratio)
        absolute = np.hypot(cpu.absolute_centre[0::2] * 0.5 * 80, cpu.absolute_centre[1::2] * 0.5 * 60)
        check_close(d.absolute_gradient_sum, absolute, "absolute", cos, ratio)
        check_close(g.positions, cpu.positions, "positions", cos, ratio)
        check_close(g.scales, cpu.scales, "scales", cos, ratio)
        check_close(g.rotations, cpu.rotations, "rotations", cos, ratio)
        check_close(g.opacities, cpu.opacities, "opacities", cos, ratio)
        check_close(g.sh, cpu.sh, "sh", cos, ratio)


def test_adam_first_step_and_unseen_view(splat, oracle):
    # tests/test_train.cpp:450-491.
    view = oracle.train_camera(40, 32)
    target = oracle.smooth_target(40, 32, 2)
    cloud = oracle.random_cloud(8, 1, 5)
    trainer = splat.Trainer(to_cloud(cloud))
    trainer.compute_gradients(to_camera(view), target)
    g = trainer.gradients()
    rates = splat.LearningRates(sh=0.02, sh_rest_scale=0.05)
    trainer.apply_gradients(rates)
    after = trainer.cloud()
    moved = 0
    for i in range(cloud.sh.size):
        if g.sh[i] == 0.0:
            continue
        dc = i % 12 < 3
        rate = rates.sh if dc else rates.sh * rates.sh_rest_scale
        expected = cloud.sh[i] - (rate if g.sh[i] > 0 else -rate)
        tol = 2e-5 if dc else max(2e-5, abs(expected) / 512.0)
        assert abs(after.sh[i] - expected) <= tol
        moved += 1
    assert moved > 0
    for i in range(cloud.count):
        if g.opacities[i] == 0.0:
            continue
        assert abs(after.opacities[i] - (cloud.opacities[i] - (rates.opacity if g.opacities[i] > 0 else -rates.opacity))) < 2e-5
    # A view that sees none of them moves nothing, despite the momentum.
    away = to_camera(view)
    rot = np.diag([-1.0, 1.0, -1.0, 1.0]).astype(np.float32)  # 180 degrees about y
    away.view = rot @ away.view
    trainer.compute_gradients(away, target)
    trainer.apply_gradients(rates)
    unseen = trainer.cloud()
    np.testing.assert_array_equal(unseen.positions, after.positions)
    np.testing.assert_array_equal(unseen.opacities, after.opacities)
    np.testing.assert_array_equal(unseen.sh, after.sh)


def test_degenerate_gaussians_do_not_spread(splat, oracle):
    # tests/test_train.cpp:544-586.
    view = oracle.train_camera(72, 56)
    target = oracle.smooth_target(72, 56, 37)
    healthy = oracle.random_cloud(40, 1, 41)
    clean = splat.Trainer(to_cloud(healthy))
    expected = clean.render(to_camera(view))
    bad = healthy.copy()
    n, f = healthy.count, 12
    extra = 5
    bad.positions = np.concatenate([healthy.positions, np.zeros(extra * 3, np.float32)])
    bad.scales = np.concatenate([healthy.scales, np.full(extra * 3, np.log(0.3), np.float32)])
    bad.rotations = np.concatenate([healthy.rotations, np.tile(np.array([1, 0, 0, 0], np.float32), extra)])
    bad.opacities = np.concatenate([healthy.opacities, np.full(extra, 2.0, np.float32)])
    bad.sh = np.concatenate([healthy.sh, np.zeros(extra * f, np.float32)])
    for i in range(n, n + extra):
        bad.positions[i * 3 + 2] = 4.0
    bad.positions[n * 3] = np.nan
    bad.scales[(n + 1) * 3] = 200.0
    bad.rotations[(n + 2) * 4] = 1e-5
    bad.opacities[n + 3] = np.nan
    bad.sh[(n + 4) * f] = np.nan
    trainer = splat.Trainer(to_cloud(bad))
    rendered = trainer.render(to_camera(view))
    np.testing.assert_array_equal(rendered.view(np.uint32), expected.view(np.uint32))
    stats = trainer.compute_gradients(to_camera(view), target)
    assert np.isfinite(stats.loss)
    g = trainer.gradients()
    assert np.isfinite(g.positions).all() and np.isfinite(g.sh).all()


def test_graph_form_matches_plain_form(splat, oracle):
    view = oracle.train_camera(96, 80)
    target = oracle.smooth_target(96, 80, 3)
    cloud = oracle.random_cloud(500, 2, 23)
    rates = splat.LearningRates(position=1e-3)
    results = []
    for graph in (False, True):
        opts = splat.TrainerOptions(force_fixed_point=True, use_graph=graph, sh_storage=splat.SH_F32,
                                    state_storage=splat.STATE_F32)
        t = splat.Trainer(to_cloud(cloud), opts)
        losses = [t.step(to_camera(view), target, rates).loss for _ in range(5)]
        results.append((losses, t.cloud()))
    assert results[0][0] == results[1][0]
    for a, b in zip((results[0][1].positions, results[0][1].sh), (results[1][1].positions, results[1][1].sh)):
        np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("sh_storage,state_storage,selective", [
    ("SH_F16", "STATE_BF16_PAIR", True),
    ("SH_BF16", "STATE_BF16_PAIR", False),
    ("SH_F32", "STATE_F32", True),
])
def test_fused_step_matches_split_step(splat, oracle, sh_storage, state_storage, selective):
    # The one-kernel step and the three-kernel step: the same bits, including
    # non-selective Adam (momentum on unseen Gaussians) and the penalties.
    # Fixed-point sums, so that both runs start from the same gradients (float
    # atomics add in an order that changes from run to run).
    view = oracle.train_camera(96, 80)
    target = oracle.smooth_target(96, 80, 3)
    cloud = oracle.random_cloud(700, 3, 41)
    rates = splat.LearningRates(position=1e-3)
    results = []
    for split in (False, True):
        opts = splat.TrainerOptions(sh_storage=getattr(splat, sh_storage), state_storage=getattr(splat, state_storage),
                                    selective_adam=selective, force_fixed_point=True, split_step=split,
                                    opacity_reg=0.0 if selective else 0.01, scale_reg=0.0 if selective else 0.01)
        t = splat.Trainer(to_cloud(cloud), opts)
        t.set_active_sh_degree(2)
        losses = [t.step(to_camera(view), target, rates).loss for _ in range(4)]
        results.append((losses, t.cloud()))
    assert results[0][0] == results[1][0]
    for name in ("positions", "scales", "rotations", "opacities", "sh"):
        np.testing.assert_array_equal(getattr(results[0][1], name), getattr(results[1][1], name), err_msg=name)


@pytest.mark.parametrize("fixed", [False, True])
def test_selective_step_moves_exactly_the_reached_gaussians(splat, oracle, fixed):
    # Selective Adam steps the Gaussians the view reached (some backward sum
    # non-zero) from a list of them: with float and fixed-point sums, every
    # Gaussian whose sums are all zero keeps its parameters bit for bit, and
    # every reached one moves. Dense, opaque Gaussians hide most of the cloud.
    view = oracle.train_camera(96, 80)
    target = oracle.smooth_target(96, 80, 5)
    cloud = oracle.random_cloud(6000, 3, 77)
    cloud.opacities[:] = 4.0
    rates = splat.LearningRates(position=1e-3)
    t = splat.Trainer(to_cloud(cloud), splat.TrainerOptions(force_fixed_point=fixed))
    t.step(to_camera(view), target, rates)
    before = t.cloud()
    t.step(to_camera(view), target, rates)
    after = t.cloud()
    n = cloud.count
    raw = t.debug_download(splat.DEBUG_RAW, np.uint32)[: n * 16].reshape(n, 16)[:, :14]
    nonzero = raw != 0 if fixed else raw.view(np.float32) != 0.0
    reached = nonzero.any(axis=1)
    # Sums 0-8 feed the parameter gradients; 9-13 are statistics only.
    steered = nonzero[:, :9].any(axis=1)
    print(f"  {int(reached.sum())} of {n} Gaussians reached, {int(steered.sum())} with a parameter gradient")
    assert reached.sum() > 100 and (~reached).sum() > 100
    moved = np.zeros(n, bool)
    for name, per in (("positions", 3), ("scales", 3), ("rotations", 4), ("opacities", 1), ("sh", 3 * 16)):
        b = getattr(before, name).reshape(n, per)
        a = getattr(after, name).reshape(n, per)
        np.testing.assert_array_equal(a[~reached], b[~reached], err_msg=name)
        moved |= (a != b).any(axis=1)
    assert moved[steered].mean() > 0.99


def test_training_lowers_the_loss(splat, oracle):
    # In the spirit of tests/test_train.cpp:493-520: fit a rendered view.
    view = oracle.train_camera(96, 72)
    truth = oracle.random_cloud(300, 1, 99)
    ref_rgb, _, _ = oracle.ref_render(truth, view)
    target = np.concatenate([np.clip(np.rint(ref_rgb * 255), 0, 255), np.full((ref_rgb.shape[0], 1), 255)], axis=1)
    target = target.astype(np.uint8).ravel()
    start = oracle.random_cloud(300, 1, 5)
    trainer = splat.Trainer(to_cloud(start))
    rates = splat.LearningRates(position=1e-3)
    first = last = None
    for it in range(300):
        s = trainer.step(to_camera(view), target, rates)
        assert np.isfinite(s.loss)
        first = s.loss if first is None else first
        last = s.loss
    print(f"  overfitting one view: loss {first:.4f} -> {last:.4f}")
    assert last < first * 0.6


def test_detmath_bit_exact_on_device(splat, oracle):
    import torch

    x = np.concatenate([np.linspace(-90, 90, 100001), np.linspace(1e-6, 2, 100001),
                        np.random.default_rng(1).normal(0, 5, 100000)]).astype(np.float32)
    xd = torch.from_numpy(x).cuda()
    e, l = torch.empty_like(xd), torch.empty_like(xd)
    splat.detmath_device(xd.data_ptr(), e.data_ptr(), l.data_ptr(), x.size)
    he, hl = oracle.detmath(x)
    np.testing.assert_array_equal(e.cpu().numpy().view(np.uint32), he.view(np.uint32))
    np.testing.assert_array_equal(l.cpu().numpy().view(np.uint32), hl.view(np.uint32))


@pytest.mark.parametrize("count", [2, 255, 256, 4096, 4097, 100_000, (1 << 20) + 7])
@pytest.mark.parametrize("key_bits", [8, 32])
def test_radix_sort_matches_stable_sort(splat, oracle, count, key_bits):
    # tests/test_radix_sort.cpp:15-60.
    import torch

    mask = 0xFFFFFFFF if key_bits == 32 else 0x0F
    keys = oracle.mt19937(count * 31 + key_bits, count) & np.uint32(mask)
    order = oracle.stable_order(keys)
    k = torch.from_numpy(keys.view(np.int32)).cuda()
    v = torch.arange(count, dtype=torch.int32, device="cuda")
    tk, tv = torch.empty_like(k), torch.empty_like(v)
    splat.radix_sort_device(k.data_ptr(), v.data_ptr(), tk.data_ptr(), tv.data_ptr(), count, key_bits)
    got_k = k.cpu().numpy().view(np.uint32)
    got_v = v.cpu().numpy().view(np.uint32)
    np.testing.assert_array_equal(got_k, keys[order])
    np.testing.assert_array_equal(got_v, order)


@pytest.mark.parametrize("digit_bits", [6, 7, 8])
def test_radix_sort_u64_tile_depth_keys(splat, digit_bits):
    import torch

    rng = np.random.default_rng(digit_bits)
    count = 300_001
    tiles = rng.integers(0, 4056, count, dtype=np.uint64)
    depth = rng.integers(0, 1 << 32, count, dtype=np.uint64) | np.uint64(0xFFFF0000)  # many ties in the high bits
    depth[::7] = depth[0]
    keys = (tiles << np.uint64(32)) | depth
    order = np.argsort(keys, kind="stable").astype(np.uint32)
    k = torch.from_numpy(keys.view(np.int64)).cuda()
    v = torch.arange(count, dtype=torch.int32, device="cuda")
    tk, tv = torch.empty_like(k), torch.empty_like(v)
    splat.radix_sort_device(k.data_ptr(), v.data_ptr(), tk.data_ptr(), tv.data_ptr(), count, 44, key_bytes=8,
                            digit_bits=digit_bits)
    np.testing.assert_array_equal(k.cpu().numpy().view(np.uint64), keys[order])
    np.testing.assert_array_equal(v.cpu().numpy().view(np.uint32), order)


def test_autotune_changes_nothing_but_the_sort_settings(splat, oracle):
    view = oracle.train_camera(96, 80)
    target = oracle.smooth_target(96, 80, 3)
    cloud = oracle.random_cloud(400, 2, 31)
    opts = splat.TrainerOptions(force_fixed_point=True, use_graph=True)
    tuned = splat.Trainer(to_cloud(cloud), opts)
    result = tuned.autotune(to_camera(view), target, repeats=1)
    assert result["sort_form"] in (0, 1) and result["digit_bits"] in (6, 7, 8)
    assert all(v > 0 for v in result["ms"].values())
    after = tuned.cloud()
    np.testing.assert_array_equal(after.positions, cloud.positions)
    assert np.all(tuned.densify_stats().visits == 0)
    plain = splat.Trainer(to_cloud(cloud), splat.TrainerOptions(force_fixed_point=True))
    rates = splat.LearningRates(position=1e-3)
    for _ in range(3):
        a = tuned.step(to_camera(view), target, rates)
        b = plain.step(to_camera(view), target, rates)
        assert a.loss == b.loss and a.tile_entries == b.tile_entries
    np.testing.assert_array_equal(tuned.cloud().positions, plain.cloud().positions)


@pytest.mark.parametrize("exact", [True, False])
def test_pixel_layouts_agree(splat, oracle, exact):
    # One or two pixels per thread: the same per-pixel arithmetic, so the same
    # image bit for bit; float sums in another order, so gradients to rounding.
    view = oracle.train_camera(100, 75)
    target = oracle.smooth_target(100, 75, 5)
    cloud = oracle.random_cloud(500, 1, 37)
    out = []
    for layout in (1, 2):
        t = splat.Trainer(to_cloud(cloud), splat.TrainerOptions(exact_math=exact, forward_pixels_per_thread=layout,
                                                                backward_pixels_per_thread=layout))
        image = t.render(to_camera(view))
        stats = t.compute_gradients(to_camera(view), target)
        out.append((image, stats, t.gradients()))
    np.testing.assert_array_equal(out[0][0].view(np.uint32), out[1][0].view(np.uint32))
    assert abs(out[0][1].loss - out[1][1].loss) < 1e-6
    for name in ("positions", "scales", "rotations", "opacities", "sh"):
        check_close(getattr(out[0][2], name), getattr(out[1][2], name), name, 0.99999, 1e-4)


@pytest.mark.parametrize("exact", [True, False])
def test_tile_batch_and_launch_forms_agree(splat, oracle, exact):
    # The two-pixel kernels at every tile edge, batch depth, launch form and
    # form of the backward's sums:
    # each pixel blends the same splats in the same order with the same
    # arithmetic, so the image is the same bits as the one-pixel reference
    # layout's; float sums in another order, so gradients to rounding. The
    # view (100x75) leaves partial tiles at both edges for either tile edge.
    view = oracle.train_camera(100, 75)
    target = oracle.smooth_target(100, 75, 5)
    cloud = oracle.random_cloud(500, 1, 37)
    base = splat.Trainer(to_cloud(cloud), splat.TrainerOptions(exact_math=exact))
    image0 = base.render(to_camera(view))
    base.compute_gradients(to_camera(view), target)
    g0 = base.gradients()
    for tile, batch, persistent, grouped in itertools.product((16, 32), (128, 256), (False, True), (False, True)):
                opts = splat.TrainerOptions(exact_math=exact, forward_pixels_per_thread=2, backward_pixels_per_thread=2,
                                            tile_size=tile, batch_depth=batch, persistent_raster=persistent,
                                            grouped_backward=grouped)
                t = splat.Trainer(to_cloud(cloud), opts)
                image = t.render(to_camera(view))
                np.testing.assert_array_equal(image.view(np.uint32), image0.view(np.uint32),
                                              err_msg=f"tile {tile} batch {batch} persistent {persistent}")
                t.compute_gradients(to_camera(view), target)
                g = t.gradients()
                for name in ("positions", "scales", "rotations", "opacities", "sh"):
                    check_close(getattr(g, name), getattr(g0, name),
                                f"{name} t{tile} b{batch} p{int(persistent)} g{int(grouped)}", 0.99999, 1e-4)


@pytest.mark.parametrize("tile,persistent", [(16, False), (32, True)])
def test_backward_takes_the_heaviest_tiles_first(splat, oracle, tile, persistent):
    # The two-pixel compositing records, per tile, the entries its backward
    # walks (range end minus the least stop of the tile's pixels); the
    # backward takes the tiles in half-octave classes of that work, heaviest
    # first: every tile once, and a later tile never more than a class above
    # an earlier one (sqrt 2, plus slack for the SFU log2 at class edges).
    view = oracle.train_camera(150, 100)
    target = oracle.smooth_target(150, 100, 6)
    cloud = oracle.random_cloud(4000, 1, 41)
    t = splat.Trainer(to_cloud(cloud), splat.TrainerOptions(exact_math=False, forward_pixels_per_thread=2,
                                                            backward_pixels_per_thread=2, tile_size=tile,
                                                            persistent_raster=persistent))
    t.compute_gradients(to_camera(view), target)
    gw, gh = -(-150 // tile), -(-100 // tile)
    tiles = gw * gh
    schedule = t.debug_download(splat.DEBUG_TILE_SCHEDULE, np.uint32)[: 2 * tiles]
    work, order = schedule[:tiles], schedule[tiles:]
    assert np.array_equal(np.sort(order), np.arange(tiles, dtype=np.uint32))
    ranges = t.debug_download(splat.DEBUG_RANGES, np.uint32)[: 2 * tiles].reshape(tiles, 2)
    stops = t.debug_download(splat.DEBUG_STOPS, np.uint32)[: 150 * 100].reshape(100, 150)
    for k in range(tiles):
        ty, tx = divmod(k, gw)
        least = stops[ty * tile:(ty + 1) * tile, tx * tile:(tx + 1) * tile].min()
        assert work[k] == ranges[k, 1] - min(least, ranges[k, 1]), k
    walked = work[order].astype(np.float64)
    assert walked.max() > 0
    lightest = np.minimum.accumulate(walked)
    assert (walked[1:] <= 1.5 * lightest[:-1] + 1.0).all()


def test_batched_persistent_matches_single_views(splat, oracle):
    # Several views of uneven size in one persistent launch per stage, 32 x 32
    # tiles: each view's loss equals that view's alone (the same tiles, lists
    # and arithmetic), whichever block took which tile.
    cloud = oracle.random_cloud(3000, 1, 19)
    views = [oracle.train_camera(w, h) for (w, h) in ((64, 48), (100, 75), (48, 96))]
    targets = [oracle.smooth_target(v.width, v.height, 3 + k) for k, v in enumerate(views)]
    opts = splat.TrainerOptions(sort_form=splat.SORT_TILE_DEPTH_64, exact_math=False, forward_pixels_per_thread=2,
                                backward_pixels_per_thread=2, tile_size=32, persistent_raster=True)
    single = splat.Trainer(to_cloud(cloud), opts)
    alone = [single.compute_gradients(to_camera(v), t).loss for v, t in zip(views, targets)]
    batch = splat.Trainer(to_cloud(cloud), opts)
    stats = batch.step_batch([to_camera(v) for v in views], targets, splat.LearningRates())
    for a, b in zip([s.loss for s in stats], alone):
        assert abs(a - b) < 1e-6


def _relative_error(a, b) -> float:
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("layout", [1, 2])
def test_chosen_form_against_fp64(splat, oracle, layout):
    # The precision form (BF16 SH above DC, SFU exp/log, float sums) against the
    # FP64 twin given the same BF16-rounded coefficients: rendered image PSNR
    # and the relative error of every gradient group (norm of the difference
    # over the norm of the FP64 gradient).
    w, h = 160, 120
    view = oracle.train_camera(w, h)
    target = oracle.smooth_target(w, h, 29)
    cloud = oracle.random_cloud(3000, 3, 31)
    cloud.sh = oracle.round_sh_like_device(cloud.sh, 3, "bf16")
    rgb, _, _ = oracle.ref_render(cloud, view)
    _, _, _, adjoint = oracle.ref_loss(rgb, w, h, target, 0.2)
    cpu = oracle.ref_gradients(cloud, view, adjoint)
    opts = splat.TrainerOptions(sh_storage=splat.SH_BF16, exact_math=False, use_graph=True,
                                forward_pixels_per_thread=layout, backward_pixels_per_thread=layout)
    trainer = splat.Trainer(to_cloud(cloud), opts)
    image = trainer.render(to_camera(view)).reshape(-1, 4)[:, :3].astype(np.float64)
    mse = float(np.mean((image - rgb.reshape(-1, 3)) ** 2))
    psnr = 10.0 * np.log10(1.0 / max(mse, 1e-30))
    trainer.compute_gradients(to_camera(view), target)
    g = trainer.gradients()
    errors = {name: _relative_error(getattr(g, name), getattr(cpu, name))
              for name in ("positions", "scales", "rotations", "opacities", "sh")}
    print(f"  layout {layout}: render PSNR vs FP64 {psnr:.1f} dB; gradient relative errors "
          + ", ".join(f"{k} {v:.2e}" for k, v in errors.items()))
    assert psnr > 60.0
    for name, err in errors.items():
        assert err < 1e-3, f"{name}: relative error {err}"


def test_prefetched_targets_change_nothing(splat, oracle):
    # step(next_target=...) copies the next target during the step; the results
    # are those of plain steps, also when the next call uses another target.
    view = oracle.train_camera(96, 80)
    targets = [oracle.smooth_target(96, 80, s) for s in (3, 4, 5)]
    cloud = oracle.random_cloud(500, 1, 43)
    rates = splat.LearningRates(position=1e-3)
    order = [0, 1, 2, 0, 1]
    runs = []
    for prefetch in (False, True):
        opts = splat.TrainerOptions(force_fixed_point=True, use_graph=True)
        t = splat.Trainer(to_cloud(cloud), opts)
        losses = []
        for i, k in enumerate(order):
            # The prefetch names target (k + 1) % 3, which is not the next one at i = 2.
            nxt = targets[(k + 1) % 3] if prefetch else None
            losses.append(t.step(to_camera(view), targets[k], rates, next_target=nxt).loss)
        runs.append((losses, t.cloud()))
    assert runs[0][0] == runs[1][0]
    np.testing.assert_array_equal(runs[0][1].positions, runs[1][1].positions)
    np.testing.assert_array_equal(runs[0][1].sh, runs[1][1].sh)


def test_config1_plain_small_case(splat, oracle):
    # The plain method's small case: L1 loss only, fixed-point backward, against
    # the FP64 twin (the reference's tolerances) and, bit for bit, against the
    # restatement's fixed-point sums.
    from tests.helpers import config1_scene

    cloud, view, target = config1_scene(oracle, 101)
    rgb, _, _ = oracle.ref_render(cloud, view)
    loss, l1, _, adjoint = oracle.ref_loss(rgb, 128, 128, target, 0.0)
    cpu = oracle.ref_gradients(cloud, view, adjoint)
    trainer = splat.Trainer(to_cloud(cloud), splat.TrainerOptions(force_fixed_point=True, lambda_ssim=0.0))
    image = trainer.render(to_camera(view)).reshape(-1, 4)
    assert np.max(np.abs(image[:, :3] - rgb.reshape(-1, 3))) < 1e-3
    stats = trainer.compute_gradients(to_camera(view), target)
    assert abs(stats.loss - loss) < 1e-3 and abs(stats.l1 - l1) < 1e-3
    g = trainer.gradients()
    for name in ("positions", "scales", "rotations", "opacities", "sh"):
        check_close(getattr(g, name), getattr(cpu, name), name, 0.97, 0.1)
    n = cloud.count
    splats, reach, keys = device_projection(trainer, n)
    tiles, values, ranges = oracle_entries(oracle, splats, reach, keys, view)
    dimage = trainer.debug_download(splat.DEBUG_IMAGE, np.float32).reshape(-1, 4)
    stops = trainer.debug_download(splat.DEBUG_STOPS, np.uint32)
    dadjoint = trainer.debug_download(splat.DEBUG_ADJOINT, np.float32).reshape(-1, 4)
    raw = trainer.debug_download(splat.DEBUG_RAW, np.int32)[: n * 16].reshape(n, 16)
    o_raw = oracle.backward(splats, values, ranges, view, dimage, dadjoint, stops, True, n)
    assert np.count_nonzero(raw) > 1000
    np.testing.assert_array_equal(raw[:, :14], o_raw[:, :14])


@pytest.mark.parametrize("exact", [True, False])
def test_blend_lists_match_recompute(splat, oracle, exact):
    # The store-everything variant against the reverse-sweep recompute: the
    # same image (the same compositing), the same gradients up to the order of
    # float sums and the transmittance's rounding (division vs exp/log).
    view = oracle.train_camera(128, 96)
    target = oracle.smooth_target(128, 96, 7)
    cloud = oracle.random_cloud(2000, 2, 53)
    out = []
    for lists in (False, True):
        t = splat.Trainer(to_cloud(cloud), splat.TrainerOptions(exact_math=exact, blend_lists=lists,
                                                                backward_pixels_per_thread=1))
        image = t.render(to_camera(view))
        stats = t.compute_gradients(to_camera(view), target)
        out.append((image, stats, t.gradients()))
    np.testing.assert_array_equal(out[0][0].view(np.uint32), out[1][0].view(np.uint32))
    assert out[0][1].loss == out[1][1].loss
    for name in ("positions", "scales", "rotations", "opacities", "sh"):
        check_close(getattr(out[1][2], name), getattr(out[0][2], name), name, 0.99999, 1e-3)


def test_batched_step_sums_the_views(splat, oracle):
    # Several views in one step (uneven sizes, 64-bit tile|depth keys): each
    # view's loss equals its single-view loss, and the first Adam step moves
    # every parameter by -lr * sign(sum over views of its gradient).
    base = oracle.train_camera(96, 72)
    views = [base,
             oracle.View(base.view, base.position, 50.0, 50.0, 40.0, 30.0, 80, 60),
             oracle.View(base.view, base.position, 70.0, 70.0, 56.0, 40.0, 112, 80)]
    targets = [oracle.smooth_target(v.width, v.height, 60 + i) for i, v in enumerate(views)]
    cloud = oracle.random_cloud(600, 1, 61)
    opts = dict(force_fixed_point=True, sort_form=splat.SORT_TILE_DEPTH_64, sh_storage=splat.SH_F32,
                state_storage=splat.STATE_F32)
    single = splat.Trainer(to_cloud(cloud), splat.TrainerOptions(**opts))
    losses, total = [], None
    for v, t in zip(views, targets):
        losses.append(single.compute_gradients(to_camera(v), t).loss)
        g = single.gradients()
        parts = [np.asarray(getattr(g, name), np.float64) for name in ("positions", "opacities", "sh")]
        total = parts if total is None else [a + b for a, b in zip(total, parts)]
    rates = splat.LearningRates(position=1e-3, opacity=0.05, sh=0.02, sh_rest_scale=1.0)
    batch = splat.Trainer(to_cloud(cloud), splat.TrainerOptions(**opts, use_graph=True))
    stats = batch.step_batch([to_camera(v) for v in views], targets, rates)
    for s, l in zip(stats, losses):
        assert abs(s.loss - l) < 1e-6
    after = batch.cloud()
    for name, g, lr in zip(("positions", "opacities", "sh"), total, (1e-3, 0.05, 0.02)):
        before = np.asarray(getattr(cloud, name), np.float64)
        moved = np.asarray(getattr(after, name), np.float64) - before
        clear = np.abs(g) > 1e-3 * np.max(np.abs(g))
        assert clear.sum() > 50, name
        np.testing.assert_allclose(moved[clear], -lr * np.sign(g[clear]), rtol=1e-3, atol=1e-6, err_msg=name)


@pytest.mark.parametrize("state", ["STATE_BF16_PAIR", "STATE_F32"])
def test_apply_changes_gathers_the_state(splat, oracle, state):
    # Densification keeps the survivors' Adam moments (gathered on the GPU
    # through the source table), starts new Gaussians at zero, and takes the
    # parameters from the new cloud.
    view = oracle.train_camera(96, 80)
    target = oracle.smooth_target(96, 80, 3)
    cloud = oracle.random_cloud(500, 2, 71)
    rates = splat.LearningRates(position=1e-3)
    t = splat.Trainer(to_cloud(cloud), splat.TrainerOptions(state_storage=getattr(splat, state)))
    for _ in range(3):
        t.step(to_camera(view), target, rates)
    old = [t.debug_download(splat.DEBUG_STATE + g, np.uint32) for g in range(5)]
    source = np.array(list(range(0, 500, 2)) + [-1] * 30 + list(range(499, 300, -3)), np.int32)
    new_n = source.size
    fresh = oracle.random_cloud(new_n, 2, 72)
    t.apply_changes(to_cloud(fresh), source)
    np.testing.assert_array_equal(t.cloud().positions, fresh.positions)
    new = [t.debug_download(splat.DEBUG_STATE + g, np.uint32) for g in range(5)]
    copies = 2 if state == "STATE_F32" else 1
    kept = source >= 0
    for g, stride in enumerate((3, 3, 4, 1)):
        o = old[g][: copies * 500 * stride].reshape(copies, 500, stride)
        n = new[g][: copies * new_n * stride].reshape(copies, new_n, stride)
        np.testing.assert_array_equal(n[:, kept], o[:, source[kept]])
        assert not n[:, ~kept].any()
    # The SH state: rows of 28 words (27 at degree 2, padded to 16 bytes), row
    # counts rounded up to 128.
    width = 28
    old_rows, new_rows = 512, ((new_n + 127) // 128) * 128
    o = old[4][: copies * old_rows * width].reshape(copies, old_rows, width)
    n = new[4][: copies * new_rows * width].reshape(copies, new_rows, width)
    np.testing.assert_array_equal(n[:, :new_n][:, kept], o[:, source[kept]])
    assert not n[:, :new_n][:, ~kept].any()
    assert not n[:, new_n:].any()
    assert np.any(o[:, source[kept]])
    assert np.isfinite(t.step(to_camera(view), target, rates).loss)


@pytest.mark.parametrize("fixed", [False, True])
def test_gradients_against_central_differences(splat, oracle, fixed):
    # The adjoint against FP64 central differences of the twin's loss (h = 1e-4)
    # on 256 randomly chosen parameters of a 20000-Gaussian, SH degree 3 scene
    # (loss 0.8 L1 + 0.2 (1 - SSIM)); float sums against the reference's
    # finite-difference criterion for its oracle (tests/test_train.cpp:99-112):
    # cosine > 0.999, length within 1%.
    import concurrent.futures
    import os

    w = h = 256
    view = oracle.train_camera(w, h)
    target = oracle.smooth_target(w, h, 91)
    cloud = oracle.random_cloud(20000, 3, 93)
    trainer = splat.Trainer(to_cloud(cloud), splat.TrainerOptions(force_fixed_point=fixed, sh_storage=splat.SH_F32))
    trainer.compute_gradients(to_camera(view), target)
    g = trainer.gradients()
    names = ("positions", "scales", "rotations", "opacities", "sh")
    rng = np.random.default_rng(95)
    picks = []
    for _ in range(256):
        name = names[rng.integers(0, len(names))]
        picks.append((name, int(rng.integers(0, getattr(cloud, name).size))))

    def loss_at(name, index, delta):
        c = cloud.copy()
        arr = getattr(c, name)
        arr[index] = np.float32(arr[index] + delta)
        rgb, _, _ = oracle.ref_render(c, view)
        return oracle.ref_loss(rgb, w, h, target, 0.2)[0], float(arr[index])

    def central(pick, step):
        name, index = pick
        (lp, xp), (lm, xm) = loss_at(name, index, step), loss_at(name, index, -step)
        return (lp - lm) / (xp - xm)

    with concurrent.futures.ThreadPoolExecutor(max_workers=max(1, len(os.sched_getaffinity(0)))) as pool:
        fd = np.array(list(pool.map(lambda p: central(p, 1e-4), picks)))
        fd_half = np.array(list(pool.map(lambda p: central(p, 5e-5), picks)))
    # The loss jumps where a perturbation crosses a cutoff (alpha >= 1/255, the
    # stop threshold, a tile edge); the reference checks its FP64 twin against
    # differences with the cutoffs switched off. The kernels keep them, so the
    # parameters whose differences at h and h/2 disagree by more than 1% (not
    # locally smooth) are left out; most are kept.
    smooth = np.abs(fd - fd_half) <= 0.01 * np.maximum(np.abs(fd), 1e-3 * np.max(np.abs(fd)))
    print(f"  {smooth.sum()} of {len(picks)} parameters locally smooth")
    assert smooth.sum() >= 200
    ours = np.array([float(getattr(g, name)[index]) for name, index in picks])
    # Fixed point: the reference's tolerance for its quantised sums (cosine > 0.97, 10%).
    cos, ratio = (0.97, 0.1) if fixed else (0.999, 0.01)
    check_close(ours[smooth], fd[smooth], "parameters vs central differences", cos, ratio)


@pytest.mark.gpu
def test_sm_peaks_are_plausible(splat):
    # The microbenchmarks behind the issue-bound kernels' roofline: each figure
    # between a tenth of and twice the B200's nominal rate at its top clock
    # (148 SMs, 1965 MHz: FP32 74 TFLOP/s, SFU 4.65 T ex2/s, shared memory
    # 37 TB/s, 4 warp instructions per clock per SM).
    peaks = splat.measure_sm_peaks()
    nominal = {"fp32_flops": 148 * 128 * 2 * 1.965e9, "sfu_ops": 148 * 16 * 1.965e9,
               "shared_bytes": 148 * 128 * 1.965e9, "warp_instructions": 148 * 4 * 1.965e9}
    for key, value in nominal.items():
        assert 0.1 * value < peaks[key] < 2.0 * value, (key, peaks[key], value)


@pytest.mark.parametrize("fixed", [False, True])
def test_score_view_counts_the_marked_pixels(splat, oracle, fixed):
    # tests/test_train.cpp:588-621: 72x56, 60 Gaussians degree 1 seed 47,
    # target seed 43, share 0.5, pixel weight 2; against the reference's
    # reference_marked_pixels, a pixel either way (the worst error is kept to
    # 1/65535, which moves the limit a little).
    view = oracle.train_camera(72, 56)
    target = oracle.smooth_target(72, 56, 43)
    cloud = oracle.random_cloud(60, 1, 47)
    cpu = oracle.ref_marked_pixels(cloud, view, target, 0.5)
    assert cpu.sum() > 0.0
    trainer = splat.Trainer(to_cloud(cloud), splat.TrainerOptions(force_fixed_point=fixed))
    # An ordinary iteration counts nothing.
    trainer.compute_gradients(to_camera(view), target)
    assert np.all(trainer.densify_stats().marked_pixels == 0.0)
    stats = trainer.score_view(to_camera(view), target, 0.5, 2.0)
    scored = trainer.densify_stats()
    np.testing.assert_allclose(scored.marked_pixels, 2.0 * cpu, atol=3.0)
    np.testing.assert_allclose(scored.marked_loss, 2.0 * cpu * stats.loss, atol=3.0)
    # Back to counting nothing, and the same again adds up.
    trainer.compute_gradients(to_camera(view), target)
    np.testing.assert_array_equal(trainer.densify_stats().marked_pixels, scored.marked_pixels)


def test_score_view_accumulates_the_edge_score(splat, oracle):
    # tests/test_train.cpp:623-659: a vertical edge down the middle of a
    # 96x64 target (dark left, bright right); eight small Gaussians on it and
    # eight 24 pixels to its right. The edge score is positive on the edge and
    # zero away from it; every Gaussian reaches marked pixels (the whole image
    # is wrong).
    w, h = 96, 64
    view = oracle.train_camera(w, h)  # identity pose, focal 60: pixel x = 30 x + 48 at depth 2
    target = np.full(w * h * 4, 255, np.uint8)
    for y in range(h):
        for x in range(w):
            at = (y * w + x) * 4
            target[at:at + 3] = 40 if x < w // 2 else 220
    n = 16
    positions = np.zeros((n, 3), np.float32)
    for i in range(n):
        positions[i] = (0.0 if i < 8 else 0.8, (i % 8 - 3.5) * 0.1, 2.0)
    scales = np.full((n, 3), np.log(0.02), np.float32)
    rotations = np.zeros((n, 4), np.float32)
    rotations[:, 0] = 1.0
    cloud = splat.GaussianCloud(0, positions.ravel(), scales.ravel(), rotations.ravel(), np.zeros(n, np.float32),
                                np.zeros(n * 3, np.float32))
    trainer = splat.Trainer(cloud)
    trainer.score_view(to_camera(view), target, 0.5, 1.0)
    scored = trainer.densify_stats()
    assert scored.edge_score[:8].sum() > 0.0
    assert scored.edge_score[8:].sum() == 0.0
    assert np.all(scored.marked_pixels > 0.0)


def test_score_view_refuses_bad_arguments(splat, oracle):
    view = oracle.train_camera(72, 56)
    target = oracle.smooth_target(72, 56, 43)
    trainer = splat.Trainer(to_cloud(oracle.random_cloud(60, 1, 47)))
    with pytest.raises(splat.SplatError):
        trainer.score_view(to_camera(view), target, 0.0)
    with pytest.raises(splat.SplatError):
        trainer.score_view(to_camera(view), target, float("nan"))


@pytest.mark.parametrize("kind", [0, 1, 2])
def test_pruning_keeps_the_references_survivors_and_their_state(splat, oracle, kind):
    # Trainer::remove_largest_gaussians / remove_least_contributing_gaussians /
    # remove_least_opaque_gaussians (trainer.cpp:731-747) on the GPU: the same
    # survivors as the reference's remove_* (densify.cpp:70-113) on the same
    # cloud and statistics, in their order, with their parameters and Adam
    # state bit for bit; the statistics start anew; training goes on.
    view = oracle.train_camera(72, 56)
    target = oracle.smooth_target(72, 56, 5)
    cloud = oracle.random_cloud(300, 2, 29)
    trainer = splat.Trainer(to_cloud(cloud))
    trainer.step(to_camera(view), target, splat.LearningRates())
    trainer.collect_statistics(to_camera(view), target)
    before = trainer.cloud()
    stats = trainer.densify_stats()
    states = [trainer.debug_download(splat.DEBUG_STATE + g, np.uint32) for g in range(5)]
    host = oracle.Cloud(2, before.positions, before.scales, before.rotations, before.opacities, before.sh)
    source = oracle.ref_prune(kind, host, 0.15, stats.contribution)
    prune = (trainer.remove_largest_gaussians, trainer.remove_least_contributing_gaussians,
             trainer.remove_least_opaque_gaussians)[kind]
    assert prune(0.15) == 300 - len(source) == 45
    after = trainer.cloud()
    for name, width in (("positions", 3), ("scales", 3), ("rotations", 4), ("opacities", 1), ("sh", 27)):
        old = np.asarray(getattr(before, name)).reshape(300, width)
        new = np.asarray(getattr(after, name)).reshape(len(source), width)
        np.testing.assert_array_equal(new.view(np.uint32), old[source].view(np.uint32), name)
    for g, width in enumerate((3, 3, 4, 1)):
        new = trainer.debug_download(splat.DEBUG_STATE + g, np.uint32).reshape(len(source), width)
        np.testing.assert_array_equal(new, states[g].reshape(300, width)[source], f"state group {g}")
    # SH state: a row of 28 words per Gaussian (27 at degree 2, padded to 16
    # bytes), row counts rounded up to 128.
    new_sh = trainer.debug_download(splat.DEBUG_STATE + 4, np.uint32).reshape(256, 28)[: len(source)]
    old_sh = states[4].reshape(384, 28)[source]
    np.testing.assert_array_equal(new_sh, old_sh, "SH state")
    assert np.all(trainer.densify_stats().contribution == 0.0)
    assert math.isfinite(trainer.step(to_camera(view), target, splat.LearningRates()).loss)


def test_pruning_shares_and_ties(splat, oracle):
    # Equal sizes: the lowest indices go first, as a stable sort leaves them;
    # share 0 removes nothing, share 1 all but one; a share outside [0, 1] is refused.
    cloud = oracle.random_cloud(40, 0, 3)
    cloud.scales[:] = -2.0
    trainer = splat.Trainer(to_cloud(cloud))
    assert trainer.remove_largest_gaussians(0.0) == 0
    assert trainer.remove_largest_gaussians(0.1) == 4
    np.testing.assert_array_equal(trainer.cloud().positions.reshape(-1, 3), cloud.positions.reshape(-1, 3)[4:])
    with pytest.raises(splat.SplatError):
        trainer.remove_largest_gaussians(1.5)
    assert trainer.remove_least_opaque_gaussians(1.0) == 35
    assert trainer.cloud().size() == 1


def test_settings_without_a_kernel_accept_only_neutral_values(splat, oracle):
    trainer = splat.Trainer(to_cloud(oracle.random_cloud(20, 0, 1)))
    trainer.set_exposure([1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0])
    trainer.set_sh_dropout(0.0)
    trainer.set_filter3d([])
    trainer.add_position_noise(0.0)
    for call in (lambda: trainer.set_exposure([2, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0]), lambda: trainer.set_sh_dropout(0.5),
                 lambda: trainer.set_filter3d(np.ones(20)), lambda: trainer.add_position_noise(1.0),
                 trainer.enable_second_order, trainer.update_curvature):
        with pytest.raises(splat.UnsupportedOption):
            call()


def test_graph_follows_the_active_sh_degree(splat, oracle):
    # A captured step serves one active SH degree: after set_active_sh_degree
    # the graph form recaptures, and stays bit for bit with the form that
    # launches every kernel itself (fixed-point sums, so both are exact).
    view = oracle.train_camera(96, 72)
    target = oracle.smooth_target(96, 72, 8)
    cloud = oracle.random_cloud(3000, 3, 41)
    clouds = []
    for graph in (True, False):
        t = splat.Trainer(to_cloud(cloud), splat.TrainerOptions(use_graph=graph, force_fixed_point=True, sh_storage=splat.SH_BF16))
        for degree in (0, 0, 1, 1, 3, 2):
            t.set_active_sh_degree(degree)
            assert math.isfinite(t.step(to_camera(view), target, splat.LearningRates()).loss)
        clouds.append(t.cloud())
    for name in ("positions", "scales", "rotations", "opacities", "sh"):
        np.testing.assert_array_equal(getattr(clouds[0], name), getattr(clouds[1], name), name)


def test_device_target_entry_points_match_the_host_ones(splat, oracle):
    # collect_statistics, score_view and step_batch with the targets already
    # on the device give what the host-target calls give (fixed-point sums,
    # so bit for bit).
    import torch

    views = [oracle.train_camera(80, 64), oracle.train_camera(96, 72)]
    targets = [oracle.smooth_target(80, 64, 2), oracle.smooth_target(96, 72, 3)]
    device = [torch.from_numpy(t).cuda() for t in targets]
    cloud = oracle.random_cloud(2000, 1, 17)
    opts = splat.TrainerOptions(force_fixed_point=True, sort_form=splat.SORT_TILE_DEPTH_64)
    out = []
    for on_device in (False, True):
        t = splat.Trainer(to_cloud(cloud), opts)
        if on_device:
            t.collect_statistics_device_target(to_camera(views[0]), device[0].data_ptr())
            t.score_view_device_target(to_camera(views[1]), device[1].data_ptr(), 0.5)
            t.step_batch_device_targets([to_camera(v) for v in views], [d.data_ptr() for d in device], splat.LearningRates())
        else:
            t.collect_statistics(to_camera(views[0]), targets[0])
            t.score_view(to_camera(views[1]), targets[1], 0.5)
            t.step_batch([to_camera(v) for v in views], targets, splat.LearningRates())
        out.append((t.densify_stats_raw().copy(), t.cloud()))
    np.testing.assert_array_equal(out[0][0], out[1][0])
    for name in ("positions", "scales", "opacities", "sh"):
        np.testing.assert_array_equal(getattr(out[0][1], name), getattr(out[1][1], name), name)


@pytest.mark.parametrize("graph", [False, True])
def test_step_on_a_device_target_matches_the_host_target(splat, oracle, graph):
    # A one-view step reads a device target where it is (4-byte aligned) or
    # copies it (any other address); either way the steps equal those on
    # the host target, bit for bit with fixed-point sums, graph or not.
    import torch

    view = oracle.train_camera(90, 70)
    target = oracle.smooth_target(90, 70, 4)
    cloud = oracle.random_cloud(1500, 1, 29)
    opts = splat.TrainerOptions(force_fixed_point=True, use_graph=graph)
    rates = splat.LearningRates(position=1e-3)
    size = target.size
    padded = torch.zeros(size + 1, dtype=torch.uint8, device="cuda")
    padded[1:] = torch.from_numpy(target.reshape(-1)).cuda()
    aligned = torch.from_numpy(target.reshape(-1)).cuda()
    results = []
    for where in ("host", "aligned", "unaligned"):
        t = splat.Trainer(to_cloud(cloud), opts)
        losses = []
        for _ in range(3):
            if where == "host":
                losses.append(t.step(to_camera(view), target, rates).loss)
            elif where == "aligned":
                losses.append(t.step_device_target(to_camera(view), aligned.data_ptr(), rates).loss)
            else:
                losses.append(t.step_device_target(to_camera(view), padded.data_ptr() + 1, rates).loss)
        results.append((losses, t.cloud()))
    for losses, c in results[1:]:
        assert losses == results[0][0]
        for name in ("positions", "scales", "rotations", "opacities", "sh"):
            np.testing.assert_array_equal(getattr(c, name), getattr(results[0][1], name), name)
