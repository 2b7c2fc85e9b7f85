"""Checks the oracle's FP32 restatement and fixtures against the committed
golden outputs of the reference's FP64 twin (make_golden.py), with the
reference's tolerances (forward rgb < 1e-3, log T < 1e-2, loss terms < 1e-3)."""
from __future__ import annotations

from pathlib import Path

import numpy as np

from tests.golden.make_golden import CASES

GOLDEN = Path(__file__).with_name("reference_cases.npz")


def load():
    return np.load(GOLDEN)


def check_golden(O) -> None:
    data = load()
    for name, (w, h, n, degree, seed, tseed, opacity) in CASES.items():
        view = O.train_camera(w, h)
        cloud = O.random_cloud(n, degree, seed)
        if opacity is not None:
            cloud.opacities[:] = opacity
        target = O.smooth_target(w, h, tseed)
        splats, reach, keys = O.preprocess(cloud, view)
        order = O.stable_order(keys)
        tiles, values = O.bin_entries(splats, reach, keys[order], order, view)
        by_tile = O.stable_order(tiles)
        ranges = O.ranges(tiles[by_tile], ((w + 15) // 16) * ((h + 15) // 16))
        image, stops = O.forward(splats, values[by_tile], ranges, view, degree=degree)
        assert np.abs(image[:, :3] - data[f"{name}/rgb"]).max() < 1e-3, name
        assert np.abs(image[:, 3] - data[f"{name}/logT"]).max() < 1e-2, name
        adj, ssim_sum, l1_sum = O.loss(image, target, view, 0.2)
        loss, l1, ssim = data[f"{name}/totals"]
        P = w * h
        assert abs(l1_sum / (3 * P) - l1) < 1e-3 and abs(ssim_sum / (3 * P) - ssim) < 1e-3, name
