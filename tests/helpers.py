"""Conversions between the oracle's fixtures and the product's types, and the
oracle pipeline run on the device's own projected splats."""
from __future__ import annotations

import numpy as np

from tests.conftest import splat_module


def to_cloud(c):
    s = splat_module()
    return s.GaussianCloud(c.sh_degree, c.positions.copy(), c.scales.copy(), c.rotations.copy(), c.opacities.copy(),
                           c.sh.copy())


def to_camera(v):
    s = splat_module()
    return s.Camera(np.asarray(v.view, np.float32), np.asarray(v.position, np.float32), v.fx, v.fy, v.cx, v.cy, v.width,
                    v.height)


def tile_count(view) -> int:
    return ((view.width + 15) // 16) * ((view.height + 15) // 16)


def device_projection(trainer, n: int):
    """The device's splats [n,12], reach [n] and depth keys [n] of the last step."""
    s = splat_module()
    splats = trainer.debug_download(s.DEBUG_SPLATS, np.float32)[: n * 12].reshape(n, 12)
    reach = trainer.debug_download(s.DEBUG_REACH, np.float32)[:n]
    keys = trainer.debug_download(s.DEBUG_DEPTH_KEYS, np.uint32)[:n]
    return splats, reach, keys


def oracle_entries(oracle, splats, reach, keys, view):
    """Tile entries as the reference orders them: stable depth sort of the keys
    (values = Gaussian index), emission in that order, stable sort by tile.
    Returns (tiles sorted, values sorted, ranges)."""
    order = oracle.stable_order(keys)
    tiles, values = oracle.bin_entries(splats, reach, keys[order], order, view)
    by_tile = oracle.stable_order(tiles)
    tiles, values = tiles[by_tile], values[by_tile]
    return tiles, values, oracle.ranges(tiles, tile_count(view))
