"""Generates tests/golden/reference_cases.npz from the reference's own FP64 CPU
twin (src/train/reference.cpp, compiled unmodified into oracle/_ref by
oracle/Makefile) on the seeded inputs of the reference's tests
(tests/test_train.cpp:218-235, :256-293, :353-403; fixtures of
tests/reference_helpers.hpp). Run where the reference tree is present:

    python tests/golden/make_golden.py

The outputs are stored in float64; the inputs are regenerated from the seeds."""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import oracle as O  # noqa: E402

CASES = {
    # name: (width, height, count, degree, cloud seed, target seed, opacity override)
    "forward_100x75": (100, 75, 300, 1, 7, 11, None),
    "gradients_72x56": (72, 56, 60, 1, 13, 11, None),
    "early_stop_80x60": (80, 60, 400, 1, 17, 19, 5.0),
    "degree3_64x48": (64, 48, 120, 3, 31, 5, None),
}


def main() -> None:
    out = {}
    for name, (w, h, n, degree, seed, tseed, opacity) in CASES.items():
        view = O.train_camera(w, h)
        cloud = O.random_cloud(n, degree, seed)
        if opacity is not None:
            cloud.opacities[:] = opacity
        target = O.smooth_target(w, h, tseed)
        rgb, logT, stop = O.ref_render(cloud, view)
        loss, l1, ssim, adjoint = O.ref_loss(rgb, w, h, target, 0.2)
        g = O.ref_gradients(cloud, view, adjoint)
        out[f"{name}/rgb"] = rgb
        out[f"{name}/logT"] = logT
        out[f"{name}/stop"] = stop.astype(np.uint32)
        out[f"{name}/totals"] = np.array([loss, l1, ssim])
        out[f"{name}/adjoint"] = adjoint
        for k in ("positions", "scales", "rotations", "opacities", "sh", "absolute_centre"):
            out[f"{name}/g_{k}"] = getattr(g, k)
        out[f"{name}/contributions"] = O.ref_contributions(cloud, view)
    np.savez_compressed(Path(__file__).with_name("reference_cases.npz"), **out)
    print(f"wrote {len(out)} arrays")


if __name__ == "__main__":
    main()
