"""Densification (densify_cloud, src/train/densify.cpp:115-326; Trainer::densify,
trainer.cpp:710-715).

CPU: the reference's densify_cloud, compiled from its sources into the oracle
library, checked against what the reference's own tests expect
(tests/test_densify.cpp:61-476), so that the wrapper and its option layout
are pinned. GPU: splat_trainer_densify against that reference on the same
cloud, statistics and generator seed: the same counts, source table and new
cloud bit for bit, and the survivors' Adam state carried over, in the
reference's test scenarios and on random clouds with every option.
"""

from __future__ import annotations

import math

import numpy as np
import pytest

from tests.conftest import splat_module
from tests.helpers import to_camera, to_cloud

needs_reference = pytest.mark.skipif("not __import__('oracle.oracle', fromlist=['x']).have_reference()",
                                     reason="the reference sources are not available")


@pytest.fixture(scope="module")
def O():
    from oracle import oracle as o

    return o


# ----------------------------------------------------------------- scenarios


def line_of(O, count, scale, opacity=0.5, degree=0):
    """Gaussians of one size and opacity at x = 0, 1, 2, ... (test_densify.cpp:30-41)."""
    coeffs = (degree + 1) ** 2
    positions = np.zeros((count, 3), np.float32)
    positions[:, 0] = np.arange(count, dtype=np.float32)
    scales = np.full(count * 3, np.log(np.float32(scale)), np.float32)
    rotations = np.zeros((count, 4), np.float32)
    rotations[:, 0] = 1.0
    opacities = np.full(count, np.log(np.float32(opacity) / (np.float32(1.0) - np.float32(opacity))), np.float32)
    sh = np.zeros((count, coeffs * 3), np.float32)
    sh[:, 0] = np.arange(count, dtype=np.float32)
    return O.Cloud(degree, positions.ravel(), scales, rotations.ravel(), opacities, sh.ravel())


def stats_of(count, gradient):
    """Gradient sums, one visit, screen radius 1 (test_densify.cpp:43-49); the other columns 0."""
    raw = np.zeros((count, 8), np.float32)
    raw[:, 0] = gradient
    raw[:, 1] = 1.0
    raw[:, 2] = 1.0
    return raw


def options_of(**changes):
    """The reference tests' default_options() (test_densify.cpp:51-57) with changes."""
    o = splat_module().DensifyOptions(gradient_threshold=1.0, dense_scale=0.1, max_world_scale=10.0)
    for k, v in changes.items():
        setattr(o, k, v)
    return o


def scenarios(O):
    """(name, cloud, raw statistics, options, seed, what the reference's test expects)."""
    out = []
    out.append(("low gradients", line_of(O, 4, 0.05), stats_of(4, 0.5), options_of(), 1,
                dict(count=4, cloned=0, split=0, source=[0, 1, 2, 3])))
    raw = stats_of(3, 0.0)
    raw[1, 0], raw[1, 1] = 4.0, 2.0
    out.append(("clone", line_of(O, 3, 0.05), raw, options_of(), 1, dict(cloned=1, split=0, source=[0, 1, 2, -1])))
    raw = stats_of(1, 10.0)
    raw[0, 1] = 100.0
    out.append(("average", line_of(O, 1, 0.05), raw, options_of(), 1, dict(cloned=0)))
    raw = stats_of(1, 0.0)
    raw[0, 1] = 0.0
    out.append(("never seen", line_of(O, 1, 0.05), raw, options_of(), 1, dict(cloned=0)))
    raw = stats_of(2, 0.0)
    raw[0, 0] = 2.0
    out.append(("split", line_of(O, 2, 1.0), raw, options_of(), 7, dict(split=1, source=[1, -1, -1])))
    c = line_of(O, 4, 0.05)
    c.opacities[0] = np.log(np.float32(0.001) / np.float32(0.999))
    c.scales[1 * 3 + 2] = np.log(np.float32(20.0))
    raw = stats_of(4, 0.0)
    raw[2, 2] = 50.0
    out.append(("prune transparent", c, raw, options_of(max_screen_radius=20.0), 1, dict(pruned=1, source=[1, 2, 3])))
    out.append(("prune oversized", c, raw, options_of(max_screen_radius=20.0, prune_large=True), 1,
                dict(pruned=3, source=[3])))
    c = line_of(O, 4, 0.01)
    c.positions[3] = np.nan
    c.sh[2 * 3 + 1] = np.inf
    defaults = splat_module().DensifyOptions()
    out.append(("non-finite", c, stats_of(4, 0.0), defaults, 1, dict(pruned=2, source=[0, 3])))
    raw = stats_of(6, 0.0)
    raw[:, 0] = [2.0, 9.0, 3.0, 8.0, 0.0, 4.0]
    out.append(("limit", line_of(O, 6, 0.05), raw, options_of(max_gaussians=8), 1, dict(count=8, cloned=2, held_back=3)))
    out.append(("over the limit", line_of(O, 6, 0.05), raw, options_of(max_gaussians=3), 1, dict(count=6, held_back=5)))
    c = line_of(O, 4, 1.0)
    c.scales[6:12] = np.log(np.float32(0.05))
    raw = stats_of(4, 0.0)
    raw[:, 4] = [9.0, 0.0, 9.0, 0.0]
    raw[:, 0] = [0.0, 9.0, 0.0, 9.0]
    out.append(("absolute gradient", c, raw, options_of(split_threshold=4.0), 1,
                dict(split=1, cloned=1, source=[1, 2, 3, -1, -1, -1])))
    raw = stats_of(3, 2.0)
    raw[:, 5] = [60.0, 49.0, 0.0]
    out.append(("scored views", line_of(O, 3, 0.05), raw, options_of(scored_views=10, min_marked_pixels=5.0), 1,
                dict(cloned=1)))
    c = line_of(O, 5, 0.05)
    c.opacities[:4] = np.log(np.float32(0.001) / np.float32(0.999))
    raw = stats_of(5, 0.0)
    raw[:, 3] = [4.0, 1.0, 3.0, 2.0, 0.0]
    out.append(("transparent share", c, raw, options_of(transparent_share=0.5), 1, dict(pruned=2, source=[0, 2, 4])))
    raw = raw.copy()
    raw[:, 6] = [4.0, 1.0, 3.0, 2.0, 9.0]
    out.append(("transparent share, scored", c, raw, options_of(transparent_share=0.5, scored_views=1), 1,
                dict(source=[1, 3, 4])))
    c = line_of(O, 8, 1.0, 0.5, 1)
    c.scales[0:3] = np.log(np.float32(0.01))
    c.scales[3:6] = np.log(np.float32(4.0))
    out.append(("exploration", c, stats_of(8, 0.0), options_of(explore_splits=2, explore_seeds=3), 3,
                dict(split=2, seeded=3, count=13)))
    out.append(("exploration at the limit", c, stats_of(8, 0.0),
                options_of(explore_splits=2, explore_seeds=3, max_gaussians=9), 3, dict(count=9, seeded=0)))
    c = line_of(O, 1, 1.0)
    c.scales[1] = c.scales[2] = np.log(np.float32(0.2))
    raw = stats_of(1, 2.0)
    raw[:, 7] = 1.0
    out.append(("long axis", c, raw, options_of(edge_split=True), 1, dict(count=2, split=1, source=[-1, -1])))
    raw = stats_of(1000, 2.0)
    raw[:, 7] = 0.1
    raw[:500, 7] = 1.0
    out.append(("edge scores", line_of(O, 1000, 1.0), raw, options_of(edge_split=True), 1, dict()))
    raw = stats_of(100, 2.0)
    out.append(("edge scores zero", line_of(O, 100, 1.0), raw, options_of(edge_split=True), 1, dict(split=100, count=200)))
    return out


def _check_expected(name, result, expected):
    for key, value in expected.items():
        got = list(result.source) if key == "source" else result.counts[key]
        assert got == value, f"{name}: {key} {got} != {value}"


# ----------------------------------------------------------------- CPU pins


@needs_reference
def test_reference_densify_matches_its_own_tests(O):
    # The reference's densify_cloud through the oracle wrapper gives what the
    # reference's tests expect, case by case; the option structure is the
    # product's, so its layout is pinned too.
    for name, cloud, raw, options, seed, expected in scenarios(O):
        r = O.ref_densify(cloud, raw, options._c(), O.RefRng(seed))
        _check_expected(name, r, expected)
    # Edge scores: the top-scored all split, about 55% in all (test_densify.cpp:442-459).
    name, cloud, raw, options, seed, _ = [s for s in scenarios(O) if s[0] == "edge scores"][0]
    r = O.ref_densify(cloud, raw, options._c(), O.RefRng(seed))
    assert 530 <= r.counts["split"] <= 570
    assert not np.any((r.source >= 0) & (r.source < 500))
    # Long axis: children at -0.45 and +0.45 (test_densify.cpp:417-440).
    name, cloud, raw, options, seed, _ = [s for s in scenarios(O) if s[0] == "long axis"][0]
    r = O.ref_densify(cloud, raw, options._c(), O.RefRng(seed))
    assert sorted(np.round(r.cloud.positions[[0, 3]], 6)) == [-0.45, 0.45]


@needs_reference
def test_reference_densify_throws_on_an_empty_result_and_keeps_the_generator(O):
    # Everything transparent: densify_cloud returns an empty cloud (Trainer::densify
    # throws on it); two calls on one generator differ from two fresh ones.
    cloud = line_of(O, 3, 0.05, opacity=0.001)
    r = O.ref_densify(cloud, stats_of(3, 0.0), options_of()._c(), O.RefRng(1))
    assert r.counts["count"] == 0 and r.counts["pruned"] == 3
    raw = stats_of(2, 0.0)
    raw[0, 0] = 2.0
    rng = O.RefRng(7)
    first = O.ref_densify(line_of(O, 2, 1.0), raw, options_of()._c(), rng)
    second = O.ref_densify(line_of(O, 2, 1.0), raw, options_of()._c(), rng)
    assert not np.array_equal(first.cloud.positions, second.cloud.positions)


@needs_reference
def test_generator_picks_follow_the_reference():
    # splat_rng_pick is std::uniform_int_distribution<std::size_t> over
    # std::mt19937, as the session picks the views it scores (train.cpp:690-692).
    from oracle import oracle as o

    splat = splat_module()
    for seed, count in ((1, 10), (8, 1000), (12345, 3), (0, 2**40)):
        mine, ref = splat.Rng(seed), o.RefRng(seed)
        assert [mine.pick(count) for _ in range(50)] == [o.ref_rng_pick(ref, count) for _ in range(50)]


# ----------------------------------------------------------------- GPU parity


def _trainer_for(splat, O, cloud, raw, sh_storage=None):
    """A trainer on the cloud with the statistics set, and the cloud it holds."""
    opts = splat.TrainerOptions()
    if sh_storage is not None:
        opts.sh_storage = sh_storage
    trainer = splat.Trainer(to_cloud(cloud), opts)
    trainer.set_densify_stats(raw)
    held = trainer.cloud()
    return trainer, O.Cloud(cloud.sh_degree, held.positions, held.scales, held.rotations, held.opacities, held.sh)


def _assert_same_cloud(name, after, ref):
    for field in ("positions", "scales", "rotations", "opacities", "sh"):
        a = np.asarray(getattr(after, field), np.float32)
        b = np.asarray(getattr(ref, field), np.float32)
        assert a.shape == b.shape, f"{name}: {field} {a.shape} != {b.shape}"
        bad = np.flatnonzero(a.view(np.uint32) != b.view(np.uint32))
        assert bad.size == 0, f"{name}: {field} differs at {bad[:8]}: {a[bad[:8]]} != {b[bad[:8]]}"


def _densify_both(splat, O, name, cloud, raw, options, seed, sh_storage=None):
    trainer, held = _trainer_for(splat, O, cloud, raw, sh_storage)
    ref = O.ref_densify(held, raw, options._c(), O.RefRng(seed))
    result = trainer.densify(options, splat.Rng(seed))
    for key in ("count", "cloned", "split", "seeded", "pruned", "held_back"):
        assert getattr(result, key) == ref.counts[key], f"{name}: {key} {getattr(result, key)} != {ref.counts[key]}"
    np.testing.assert_array_equal(result.source, ref.source, f"{name}: source")
    _assert_same_cloud(name, trainer.cloud(), ref.cloud)
    return trainer, result, ref


@pytest.mark.gpu
def test_densify_matches_the_reference_in_its_test_scenarios(splat, O):
    # Every scenario of the reference's densify tests, on the GPU: the same
    # counts, the same source table and the same new cloud, bit for bit
    # (split children drawn from the same generator in the same order).
    for name, cloud, raw, options, seed, expected in scenarios(O):
        _densify_both(splat, O, name, cloud, raw, options, seed)


def _random_case(O, n, degree, seed):
    rng = np.random.default_rng(seed)
    cloud = O.random_cloud(n, degree, seed)
    cloud.scales[:] = rng.uniform(-5.0, 0.5, n * 3).astype(np.float32)
    cloud.opacities[:] = rng.uniform(-7.0, 4.0, n).astype(np.float32)
    raw = np.zeros((n, 8), np.float32)
    raw[:, 1] = rng.integers(0, 6, n)                        # visits
    raw[:, 0] = rng.exponential(3e-4, n) * raw[:, 1]         # gradient sums
    raw[:, 2] = rng.uniform(0.0, 40.0, n)                    # screen radius
    raw[:, 3] = rng.uniform(0.0, 2.0, n)                     # contribution
    raw[:, 4] = raw[:, 0] * rng.uniform(1.0, 3.0, n)         # absolute gradient sums
    raw[:, 5] = rng.integers(0, 200, n)                      # marked pixels
    raw[:, 6] = rng.uniform(0.0, 5.0, n)                     # marked loss
    raw[:, 7] = rng.uniform(0.0, 1.0, n) * (rng.uniform(size=n) < 0.7)  # edge score
    # Ties for the stable sorts.
    raw[::7, 3] = 0.5
    raw[::5, 0] = raw[::5, 1] * 4e-4
    return cloud, raw


RANDOM_OPTIONS = [
    dict(),
    dict(dense_scale=0.05, max_gaussians=5200),
    dict(dense_scale=0.05, prune_large=True, max_world_scale=1.0, max_screen_radius=30.0),
    dict(dense_scale=0.05, split_threshold=5e-4, transparent_share=0.3),
    dict(dense_scale=0.05, scored_views=10, min_marked_pixels=5.0, transparent_share=0.6),
    dict(dense_scale=0.05, explore_splits=40, explore_seeds=25, max_gaussians=5600),
    dict(dense_scale=0.05, edge_split=True, max_gaussians=6000),
    dict(dense_scale=0.05, max_gaussians=0),
]


@pytest.mark.gpu
@pytest.mark.parametrize("case", range(len(RANDOM_OPTIONS)))
def test_densify_matches_the_reference_on_random_clouds(splat, O, case):
    # 5000 Gaussians of degree 3 with random statistics (ties included) under
    # each option set, F16 and F32 SH: identical results, and the survivors'
    # Adam state gathered through the source table.
    cloud, raw = _random_case(O, 5000, 3, 100 + case)
    options = splat.DensifyOptions(gradient_threshold=2e-4, **RANDOM_OPTIONS[case])
    for storage in (splat.SH_F16, splat.SH_F32):
        trainer, held = _trainer_for(splat, O, cloud, raw, storage)
        view = O.train_camera(72, 56)
        target = O.smooth_target(72, 56, 5)
        trainer.step(to_camera(view), target, splat.LearningRates())
        trainer.set_densify_stats(raw)
        before = trainer.cloud()
        held = O.Cloud(3, before.positions, before.scales, before.rotations, before.opacities, before.sh)
        states = [trainer.debug_download(splat.DEBUG_STATE + g, np.uint32) for g in range(5)]
        seed = 11 + case
        ref = O.ref_densify(held, raw, options._c(), O.RefRng(seed))
        result = trainer.densify(options, splat.Rng(seed))
        assert result.count == ref.counts["count"]
        for key in ("cloned", "split", "seeded", "pruned", "held_back"):
            assert getattr(result, key) == ref.counts[key], key
        np.testing.assert_array_equal(result.source, ref.source)
        _assert_same_cloud(f"random {case}", trainer.cloud(), ref.cloud)
        m = result.count
        kept = result.source >= 0
        for g, width in enumerate((3, 3, 4, 1)):
            new = trainer.debug_download(splat.DEBUG_STATE + g, np.uint32).reshape(m, width)
            old = states[g].reshape(5000, width)
            np.testing.assert_array_equal(new[kept], old[result.source[kept]], f"state group {g}")
            assert np.all(new[~kept] == 0), f"fresh state group {g}"
        assert np.all(trainer.densify_stats().visits == 0.0)
        assert math.isfinite(trainer.step(to_camera(view), target, splat.LearningRates()).loss)


@pytest.mark.gpu
def test_densify_decides_at_the_thresholds_as_the_reference(splat, O):
    # Log-scales and logits on both sides of exp(x) > dense scale, exp(x) >
    # max world scale and sigmoid(x) < opacity limit, one float apart: the
    # device compares against thresholds found with the host's exp, so each
    # decision matches the reference's exactly.
    n = 64
    cloud = line_of(O, n, 0.05)
    dense, world, limit = np.float32(0.1), np.float32(2.0), np.float32(0.005)
    centre = [np.log(dense), np.log(world)]
    logit = np.float32(np.log(limit / (1 - limit)))
    for i in range(n):
        step = (i % 16) - 8
        which = centre[(i // 16) % 2]
        x = np.float32(which)
        for _ in range(abs(step)):
            x = np.nextafter(x, np.float32(np.inf if step > 0 else -np.inf), dtype=np.float32)
        cloud.scales[i * 3] = x
        o = logit
        for _ in range(abs(step)):
            o = np.nextafter(o, np.float32(np.inf if step > 0 else -np.inf), dtype=np.float32)
        cloud.opacities[i] = o if i >= 32 else np.float32(0.0)
    raw = stats_of(n, 2.0)
    options = options_of(dense_scale=float(dense), max_world_scale=float(world), prune_large=True,
                         prune_opacity=float(limit), transparent_share=0.5)
    _densify_both(splat, O, "thresholds", cloud, raw, options, 5)


@pytest.mark.gpu
def test_densify_keeps_the_generator_across_rounds_and_refuses_an_empty_result(splat, O):
    # Two rounds on one generator as the session runs them (the second
    # round's split children come from the advanced generator), and an
    # all-pruned result refused with the trainer unchanged.
    trainer, held = _trainer_for(splat, O, line_of(O, 2, 1.0), stats_of(2, 0.0))
    rng, ref_rng = splat.Rng(7), O.RefRng(7)
    for round_ in range(2):
        current = trainer.cloud()
        held = O.Cloud(0, current.positions, current.scales, current.rotations, current.opacities, current.sh)
        stats = stats_of(held.count, 0.0)
        stats[0, 0] = 2.0
        trainer.set_densify_stats(stats)
        ref = O.ref_densify(held, stats, options_of()._c(), ref_rng)
        result = trainer.densify(options_of(), rng)
        assert result.split == 1
        np.testing.assert_array_equal(result.source, ref.source)
        _assert_same_cloud(f"round {round_}", trainer.cloud(), ref.cloud)
    clear = line_of(O, 3, 0.05, opacity=0.001)
    trainer, held = _trainer_for(splat, O, clear, stats_of(3, 0.0))
    with pytest.raises(splat.SplatError):
        trainer.densify(options_of(), splat.Rng(1))
    assert trainer.cloud().opacities.size == 3


# ----------------------------------------------------------------- relocation


def logit(p):
    return np.float32(np.log(np.float32(p) / (np.float32(1.0) - np.float32(p))))


def relocation_scenarios(O):
    """(name, cloud, RelocateOptions changes, seed, expected) after test_densify.cpp:355-415."""
    splat = splat_module()
    out = []
    c = line_of(O, 2, 0.1)
    c.opacities[:] = [logit(0.9), logit(0.001)]
    out.append(("dead onto live", c, splat.RelocateOptions(max_gaussians=2), 1, dict(count=2, cloned=1, seeded=0)))
    c = line_of(O, 1002, 0.1)
    c.opacities[:] = logit(0.001)
    c.opacities[0], c.opacities[1] = logit(0.9), logit(0.09)
    out.append(("in proportion", c, splat.RelocateOptions(max_gaussians=1002), 1, dict(count=1002)))
    out.append(("growth", line_of(O, 1000, 0.1), splat.RelocateOptions(max_gaussians=1030), 1,
                dict(count=1030, seeded=30, cloned=0)))
    out.append(("growth capped", line_of(O, 1000, 0.1), splat.RelocateOptions(max_gaussians=1000), 1,
                dict(count=1000, seeded=0)))
    out.append(("nothing alive", line_of(O, 5, 0.1, 0.001), splat.RelocateOptions(), 1, dict(count=5, cloned=0)))
    c = line_of(O, 4, 0.1)
    c.positions[3] = np.nan
    c.sh[2 * 3 + 1] = np.inf
    out.append(("non-finite are dead", c, splat.RelocateOptions(max_gaussians=4), 3, dict(count=4, cloned=2)))
    return out


@needs_reference
def test_reference_relocation_matches_its_own_tests(O):
    # relocate_cloud through the oracle wrapper, against the reference's tests:
    # the relocated pair's opacity 1 - sqrt(1 - 0.9) and scale 0.1 * 0.9 / D,
    # targets drawn in proportion to opacity, growth within the cap.
    for name, cloud, options, seed, expected in relocation_scenarios(O):
        r = O.ref_relocate(cloud, options._c(), O.RefRng(seed))
        _check_expected(name, r, expected)
        if name == "dead onto live":
            fresh = 1.0 - math.sqrt(1.0 - 0.9)
            d = sum(math.comb(i - 1, k) * (-1) ** k * fresh ** (k + 1) / math.sqrt(k + 1)
                    for i in range(1, 3) for k in range(i))
            for i in range(2):
                assert abs(1.0 / (1.0 + math.exp(-r.cloud.opacities[i])) - fresh) < 1e-5
                assert abs(math.exp(r.cloud.scales[i * 3]) - 0.1 * 0.9 / d) < 1e-5
                assert r.source[i] == -1
        if name == "in proportion":
            on_first = int(np.sum(r.cloud.positions.reshape(-1, 3)[2:, 0] == 0.0))
            assert 850 < on_first < 950


@pytest.mark.gpu
def test_relocation_matches_the_reference(splat, O):
    # Trainer::relocate on the GPU and host against relocate_cloud: the
    # reference's scenarios, then a random cloud with dead and non-finite
    # Gaussians over two rounds on one generator, F16 and F32 SH: the same
    # counts, source table, new cloud bit for bit, and the untouched
    # Gaussians' Adam state.
    for name, cloud, options, seed, expected in relocation_scenarios(O):
        trainer, held = _trainer_for(splat, O, cloud, stats_of(cloud.count, 0.0))
        ref = O.ref_relocate(held, options._c(), O.RefRng(seed))
        r = trainer.relocate(options, splat.Rng(seed))
        for key in ("count", "cloned", "seeded"):
            assert getattr(r, key) == ref.counts[key], f"{name}: {key}"
        np.testing.assert_array_equal(r.source, ref.source, name)
        _assert_same_cloud(name, trainer.cloud(), ref.cloud)
    for storage in (splat.SH_F16, splat.SH_F32):
        cloud, raw = _random_case(O, 4000, 2, 77)
        trainer, held = _trainer_for(splat, O, cloud, raw, storage)
        view = O.train_camera(72, 56)
        target = O.smooth_target(72, 56, 5)
        trainer.step(to_camera(view), target, splat.LearningRates())
        rng, ref_rng = splat.Rng(21), O.RefRng(21)
        options = splat.RelocateOptions(min_opacity=0.01, growth=0.05, max_gaussians=4300)
        for round_ in range(2):
            before = trainer.cloud()
            held = O.Cloud(2, before.positions, before.scales, before.rotations, before.opacities, before.sh)
            m0 = held.count
            states = [trainer.debug_download(splat.DEBUG_STATE + g, np.uint32) for g in range(4)]
            ref = O.ref_relocate(held, options._c(), ref_rng)
            r = trainer.relocate(options, rng)
            assert (r.count, r.cloned, r.seeded) == (ref.counts["count"], ref.counts["cloned"], ref.counts["seeded"])
            assert r.cloned > 0
            np.testing.assert_array_equal(r.source, ref.source)
            _assert_same_cloud(f"random round {round_}", trainer.cloud(), ref.cloud)
            kept = r.source >= 0
            for g, width in enumerate((3, 3, 4, 1)):
                new = trainer.debug_download(splat.DEBUG_STATE + g, np.uint32).reshape(r.count, width)
                np.testing.assert_array_equal(new[kept], states[g].reshape(m0, width)[r.source[kept]])
                assert np.all(new[~kept] == 0)
        assert math.isfinite(trainer.step(to_camera(view), target, splat.LearningRates()).loss)
