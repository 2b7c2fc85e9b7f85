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


def config1_scene(oracle, seed: int = 1):
    """The plain small case: 4096 Gaussians of SH degree 0 in front of a 128x128
    pinhole camera (fx = fy = 128, principal point at the centre, identity
    pose); means x, y ~ U(-1, 1), z ~ U(2, 6); log-scales ~ N(-3, 0.3); unit
    quaternions from N(0, 1)^4; opacity logits ~ N(0, 1); DC colours U(0, 1)
    stored as (rgb - 0.5) / 0.28209479; target U(0, 1) RGBA8. Seeded numpy."""
    rng = np.random.default_rng(seed)
    n = 4096
    pos = np.stack([rng.uniform(-1, 1, n), rng.uniform(-1, 1, n), rng.uniform(2, 6, n)], 1).astype(np.float32).ravel()
    scales = rng.normal(-3.0, 0.3, (n, 3)).astype(np.float32).ravel()
    q = rng.normal(size=(n, 4))
    rot = (q / np.linalg.norm(q, axis=1, keepdims=True)).astype(np.float32).ravel()
    opac = rng.normal(0.0, 1.0, n).astype(np.float32)
    rgb = rng.uniform(0.0, 1.0, (n, 3))
    sh = ((rgb - 0.5) / 0.28209479177387814).astype(np.float32).ravel()
    cloud = oracle.Cloud(0, pos, scales, rot, opac, sh)
    view = oracle.View(np.eye(4, dtype=np.float32), np.zeros(3, np.float32), 128.0, 128.0, 64.0, 64.0, 128, 128)
    target = np.concatenate([rng.integers(0, 256, (128 * 128, 3)), np.full((128 * 128, 1), 255)], 1).astype(np.uint8).ravel()
    return cloud, view, target
