"""ORACLE (test infrastructure only).

Python access to the two CPU checkers of the training path:
  * the reference's own FP64 twin, src/train/reference.cpp, compiled unmodified
    into oracle/_ref/libsplatref.so (reference_render :238,
    reference_contributions :242, reference_loss :276, reference_gradients
    :343);
  * this repository's FP32 restatement of the GLSL kernels, liboracle.so
    (splat_oracle.c), whose integer results the CUDA kernels must match bit for
    bit given the same projected splats;
plus the seeded fixtures of the reference's tests (tests/reference_helpers.hpp).
Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this.
"""
from __future__ import annotations

import ctypes
import math
import subprocess
from dataclasses import dataclass
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF_LIBRARY = HERE / "_ref" / "libsplatref.so"
ORACLE_LIBRARY = HERE / "liboracle.so"

_D = ctypes.POINTER(ctypes.c_double)
_F = ctypes.POINTER(ctypes.c_float)
_U8 = ctypes.POINTER(ctypes.c_uint8)
_U32 = ctypes.POINTER(ctypes.c_uint32)
_U64 = ctypes.POINTER(ctypes.c_uint64)


def build() -> None:
    """Runs oracle/Makefile (the reference part only where the reference tree exists)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


def _load(path: Path):
    if not path.exists():
        build()
    return ctypes.CDLL(str(path))


_ref = None
_oracle = None


def ref_lib():
    global _ref
    if _ref is None:
        if not REF_LIBRARY.exists():
            build()
        if not REF_LIBRARY.exists():
            raise FileNotFoundError(f"{REF_LIBRARY} is not built (the reference tree was not available)")
        _ref = ctypes.CDLL(str(REF_LIBRARY))
    return _ref


def oracle_lib():
    global _oracle
    if _oracle is None:
        _oracle = _load(ORACLE_LIBRARY)
    return _oracle


def have_reference() -> bool:
    return REF_LIBRARY.exists()


def _fp(a):
    return a.ctypes.data_as(_F)


def _dp(a):
    return a.ctypes.data_as(_D)


# ----------------------------------------------------------------- fixtures


@dataclass
class Cloud:
    """GaussianCloud arrays (float32), the reference's layout."""

    sh_degree: int
    positions: np.ndarray
    scales: np.ndarray
    rotations: np.ndarray
    opacities: np.ndarray
    sh: np.ndarray

    @property
    def count(self) -> int:
        return int(self.opacities.size)

    @property
    def coeffs(self) -> int:
        return (self.sh_degree + 1) ** 2

    def copy(self) -> "Cloud":
        return Cloud(self.sh_degree, *(a.copy() for a in (self.positions, self.scales, self.rotations, self.opacities, self.sh)))


@dataclass
class View:
    """The reference's Camera: view[row, col] world->camera, centre, intrinsics, size."""

    view: np.ndarray
    position: np.ndarray
    fx: float
    fy: float
    cx: float
    cy: float
    width: int
    height: int

    def column_major(self) -> np.ndarray:
        return np.ascontiguousarray(np.asarray(self.view, np.float32).T.ravel())


def random_cloud(count: int, degree: int, seed: int) -> Cloud:
    """tests/reference_helpers.hpp:17-34, from the same mt19937 stream."""
    lib = oracle_lib()
    coeffs = (degree + 1) ** 2
    arrays = [np.zeros(count * k, np.float32) for k in (3, 3, 4, 1, 3 * coeffs)]
    lib.fixture_random_cloud(ctypes.c_int(count), ctypes.c_int(degree), ctypes.c_uint32(seed), *[_fp(a) for a in arrays])
    return Cloud(degree, *arrays)


def train_camera(width: int = 64, height: int = 48) -> View:
    """tests/reference_helpers.hpp:37-45: fx = fy = 60, centred, identity pose."""
    return View(np.eye(4, dtype=np.float32), np.zeros(3, np.float32), 60.0, 60.0, width * 0.5, height * 0.5, width, height)


def smooth_target(width: int, height: int, seed: int) -> np.ndarray:
    """tests/reference_helpers.hpp:48-61 (RGBA8)."""
    out = np.zeros(width * height * 4, np.uint8)
    oracle_lib().fixture_smooth_target(ctypes.c_int(width), ctypes.c_int(height), ctypes.c_uint32(seed),
                                       out.ctypes.data_as(_U8))
    return out


def normal_adjoint(seed: int, pixels: int) -> np.ndarray:
    """Standard-normal adjoint as tests/test_train.cpp:86-90 draws it: 3 doubles per pixel."""
    out = np.zeros(pixels * 3, np.float64)
    oracle_lib().fixture_normal_adjoint(ctypes.c_uint32(seed), ctypes.c_int(pixels), _dp(out))
    return out


def mt19937(seed: int, count: int) -> np.ndarray:
    out = np.zeros(count, np.uint32)
    oracle_lib().fixture_mt19937(ctypes.c_uint32(seed), ctypes.c_int(count), out.ctypes.data_as(_U32))
    return out


# ----------------------------------------------------------------- the reference's FP64 twin


def _cloud_args(cloud: Cloud):
    arrays = [np.ascontiguousarray(a, dtype=np.float32) for a in
              (cloud.positions, cloud.scales, cloud.rotations, cloud.opacities, cloud.sh)]
    return arrays, [_fp(a) for a in arrays]


def _camera_args(view: View):
    v16 = view.column_major()
    pos = np.ascontiguousarray(view.position, np.float32)
    intr = np.array([view.fx, view.fy, view.cx, view.cy], np.float32)
    return (v16, pos, intr), [_fp(v16), _fp(pos), _fp(intr), ctypes.c_int(view.width), ctypes.c_int(view.height)]


def ref_render(cloud: Cloud, view: View, background=(0.0, 0.0, 0.0), near: float = 0.01, no_cutoffs: bool = False):
    """reference_render: (rgb [P,3] float64, logT [P], stop [P] uint64)."""
    lib = ref_lib()
    keep, cargs = _cloud_args(cloud)
    ckeep, camargs = _camera_args(view)
    P = view.width * view.height
    rgb, logT, stop = np.zeros(P * 3), np.zeros(P), np.zeros(P, np.uint64)
    bg = np.array(background, np.float32)
    status = lib.ref_render(ctypes.c_int(cloud.count), ctypes.c_int(cloud.sh_degree), *cargs, *camargs, _fp(bg),
                            ctypes.c_float(near), ctypes.c_int(1 if no_cutoffs else 0), None, _dp(rgb), _dp(logT),
                            stop.ctypes.data_as(_U64))
    assert status == 0
    return rgb.reshape(P, 3), logT, stop


def ref_contributions(cloud: Cloud, view: View, background=(0.0, 0.0, 0.0), near: float = 0.01) -> np.ndarray:
    lib = ref_lib()
    keep, cargs = _cloud_args(cloud)
    ckeep, camargs = _camera_args(view)
    out = np.zeros(cloud.count)
    bg = np.array(background, np.float32)
    assert lib.ref_contributions(ctypes.c_int(cloud.count), ctypes.c_int(cloud.sh_degree), *cargs, *camargs, _fp(bg),
                                 ctypes.c_float(near), ctypes.c_int(0), _dp(out)) == 0
    return out


def ref_prune(kind: int, cloud: Cloud, share: float, contribution=None) -> np.ndarray:
    """The reference's remove_largest (kind 0), remove_least_contributing (1) or
    remove_least_opaque (2), densify.cpp:95-113: the survivors' old indices."""
    keep, cargs = _cloud_args(cloud)
    c = np.ascontiguousarray(contribution if contribution is not None else np.zeros(cloud.count), np.float32)
    source = np.zeros(cloud.count, np.int64)
    count = ctypes.c_int()
    assert ref_lib().ref_prune(ctypes.c_int(kind), ctypes.c_int(cloud.count), ctypes.c_int(cloud.sh_degree), *cargs, _fp(c),
                               ctypes.c_double(share), source.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                               ctypes.byref(count)) == 0
    return source[:count.value]


class RefRng:
    """A std::mt19937 kept by the reference side across ref_densify calls."""

    def __init__(self, seed: int):
        lib = ref_lib()
        lib.ref_rng_create.restype = ctypes.c_void_p
        lib.ref_rng_create.argtypes = [ctypes.c_uint32]
        lib.ref_rng_destroy.argtypes = [ctypes.c_void_p]
        self._h = ctypes.c_void_p(lib.ref_rng_create(ctypes.c_uint32(seed & 0xFFFFFFFF)))

    def __del__(self):
        if getattr(self, "_h", None):
            ref_lib().ref_rng_destroy(self._h)
            self._h = None


def ref_rng_pick(rng: RefRng, count: int) -> int:
    """std::uniform_int_distribution<std::size_t>(0, count - 1) on the reference side."""
    lib = ref_lib()
    lib.ref_rng_pick.restype = ctypes.c_uint64
    lib.ref_rng_pick.argtypes = [ctypes.c_void_p, ctypes.c_uint64]
    return int(lib.ref_rng_pick(rng._h, count))


@dataclass
class RefDensified:
    cloud: Cloud
    source: np.ndarray
    counts: dict


def ref_densify(cloud: Cloud, raw_stats: np.ndarray, options, rng: RefRng) -> RefDensified:
    """The reference's densify_cloud (densify.cpp:115-326) on the trainer's raw
    statistics (8 floats per Gaussian). options: a ctypes structure laid out
    as DensifyOptions in the product's field order. Raises ValueError where
    the reference throws."""
    keep, cargs = _cloud_args(cloud)
    raw = np.ascontiguousarray(raw_stats, np.float32).ravel()
    assert raw.size == cloud.count * 8
    room = 2 * cloud.count + int(options.explore_seeds)
    coeffs = (cloud.sh_degree + 1) ** 2
    out = [np.zeros(room * k, np.float32) for k in (3, 3, 4, 1, 3 * coeffs)]
    source = np.zeros(room, np.int64)
    counts = np.zeros(6, np.uint64)
    status = ref_lib().ref_densify(ctypes.c_int(cloud.count), ctypes.c_int(cloud.sh_degree), *cargs, _fp(raw), ctypes.byref(options),
                                   rng._h, *[_fp(a) for a in out], source.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                                   counts.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)))
    if status != 0:
        raise ValueError("the reference's densify_cloud threw")
    n = int(counts[0])
    result = Cloud(cloud.sh_degree, out[0][: n * 3], out[1][: n * 3], out[2][: n * 4], out[3][:n], out[4][: n * 3 * coeffs])
    names = ("count", "cloned", "split", "seeded", "pruned", "held_back")
    return RefDensified(result, source[:n], {k: int(v) for k, v in zip(names, counts)})


def ref_relocate(cloud: Cloud, options, rng: RefRng) -> RefDensified:
    """The reference's relocate_cloud (densify.cpp:328-420). options: a ctypes
    structure laid out as RelocateOptions in the product's field order."""
    keep, cargs = _cloud_args(cloud)
    room = cloud.count + int(max(0.0, options.growth) * cloud.count) + 1
    coeffs = (cloud.sh_degree + 1) ** 2
    out = [np.zeros(room * k, np.float32) for k in (3, 3, 4, 1, 3 * coeffs)]
    source = np.zeros(room, np.int64)
    counts = np.zeros(6, np.uint64)
    status = ref_lib().ref_relocate(ctypes.c_int(cloud.count), ctypes.c_int(cloud.sh_degree), *cargs, ctypes.byref(options),
                                    rng._h, *[_fp(a) for a in out], source.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                                    counts.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)))
    if status != 0:
        raise ValueError("the reference's relocate_cloud threw")
    n = int(counts[0])
    result = Cloud(cloud.sh_degree, out[0][: n * 3], out[1][: n * 3], out[2][: n * 4], out[3][:n], out[4][: n * 3 * coeffs])
    names = ("count", "cloned", "split", "seeded", "pruned", "held_back")
    return RefDensified(result, source[:n], {k: int(v) for k, v in zip(names, counts)})


# ----------------------------------------------------------------- session schedule


def ref_frequency_energy(rgba: np.ndarray, width: int, height: int, factors=(1, 2, 4)) -> np.ndarray:
    """The reference's frequency_energy (schedule.cpp:41-75)."""
    lib = ref_lib()
    image = np.ascontiguousarray(rgba, np.uint8).ravel()
    f = (ctypes.c_int * len(factors))(*factors)
    out = np.zeros(len(factors), np.float64)
    assert lib.ref_frequency_energy(image.ctypes.data_as(_U8), ctypes.c_int(width), ctypes.c_int(height), f,
                                    ctypes.c_int(len(factors)), _dp(out)) == 0
    return out


def ref_resolution_switches(full: float, half: float, quarter: float) -> tuple:
    """The reference's resolution_switches (schedule.cpp:77-82)."""
    out = np.zeros(2, np.float64)
    lib = ref_lib()
    lib.ref_resolution_switches.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_double, _D]
    lib.ref_resolution_switches(full, half, quarter, _dp(out))
    return float(out[0]), float(out[1])


def ref_growth_limit(initial: float, factor: float, observed, image_factor: float, progress: float) -> tuple:
    """The reference's GrowthBudget (schedule.hpp:26-41): (limit, final count)."""
    lib = ref_lib()
    lib.ref_growth_limit.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.POINTER(ctypes.c_uint64), ctypes.c_int,
                                     ctypes.c_double, ctypes.c_double, ctypes.POINTER(ctypes.c_uint64), _D]
    obs = (ctypes.c_uint64 * max(len(observed), 1))(*observed)
    limit, final = ctypes.c_uint64(), ctypes.c_double()
    lib.ref_growth_limit(initial, factor, obs, len(observed), image_factor, progress, ctypes.byref(limit), ctypes.byref(final))
    return limit.value, final.value


def ref_view_order(seed: int, views: int, steps: int) -> list:
    """TrainSession's view order (train.cpp:560-565, 580-586) over std::mt19937(seed)."""
    out = (ctypes.c_int * steps)()
    ref_lib().ref_view_order(ctypes.c_uint32(seed), ctypes.c_int(views), ctypes.c_int(steps), out)
    return list(out)


def half_size(rgba: np.ndarray, width: int, height: int) -> np.ndarray:
    """half_size (train.cpp:232-255) restated: the rounded mean of each 2x2 block, per channel.
    Pinned on a hand-computed case (train.cpp does not compile on its own)."""
    w, h = width // 2, height // 2
    img = np.asarray(rgba, np.uint32).reshape(height, width, 4)[: 2 * h, : 2 * w]
    s = img[0::2, 0::2] + img[0::2, 1::2] + img[1::2, 0::2] + img[1::2, 1::2]
    return ((s + 2) // 4).astype(np.uint8).ravel()


def neighbour_distances(points: np.ndarray) -> np.ndarray:
    """neighbour_distances (train.cpp:143-189) restated for small clouds: on the
    reference's grid, the mean distance to the 3 nearest other points within
    the cube of cells of radius r, for the first r of 1..4 that holds 3, else
    the cell size; float32 of max(mean, 1e-7). Parity unpinned against the
    reference's own code: train.cpp does not compile without its Vulkan tree,
    so this restatement is pinned only on cases whose answer is known (a
    lattice, tests/test_session.py)."""
    p = np.asarray(points, np.float64).reshape(-1, 3)
    n = p.shape[0]
    low, high = p.min(axis=0), p.max(axis=0)
    size = high - low
    cell = max(np.cbrt(max(size[0] * size[1] * size[2], 1e-30) / n * 8.0), max(size) / 512.0)
    cells = ((p - low) / cell).astype(np.int64)
    out = np.zeros(n, np.float32)
    for i in range(n):
        d = p - p[i]
        dist = (d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2]
        far = np.abs(cells - cells[i]).max(axis=1)
        mean = cell
        for r in range(1, 5):
            mask = far <= r
            mask[i] = False
            if mask.sum() >= 3:
                best = np.sort(dist[mask])[:3]
                mean = (np.sqrt(best[0]) + np.sqrt(best[1]) + np.sqrt(best[2])) / 3.0
                break
        out[i] = np.float32(max(mean, 1e-7))
    return out


def ref_save_ply(cloud: Cloud, path) -> None:
    """The reference's save_ply (gaussian_cloud.cpp:330-365)."""
    keep, cargs = _cloud_args(cloud)
    assert ref_lib().ref_save_ply(str(path).encode(), ctypes.c_int(cloud.count), ctypes.c_int(cloud.sh_degree), *cargs) == 0


def ref_load_ply(path) -> Cloud:
    """The reference's load_ply (gaussian_cloud.cpp:236-328); raises ValueError
    where it throws."""
    lib = ref_lib()
    n, d = ctypes.c_int(), ctypes.c_int()
    if lib.ref_load_ply(str(path).encode(), ctypes.byref(n), ctypes.byref(d), None, None, None, None, None) != 0:
        raise ValueError(f"the reference's load_ply refused {path}")
    arrays = [np.zeros(n.value * k, np.float32) for k in (3, 3, 4, 1, 3 * (d.value + 1) ** 2)]
    assert lib.ref_load_ply(str(path).encode(), ctypes.byref(n), ctypes.byref(d), *[_fp(a) for a in arrays]) == 0
    return Cloud(d.value, *arrays)


def ref_save_cgc(cloud: Cloud, path, preset: int = 0, fast: bool = False) -> dict:
    """The reference's save_cgc (src/splat/cgc.cpp), with the LZMA shim."""
    keep, cargs = _cloud_args(cloud)
    stats = np.zeros(4, np.uint64)
    lib = ref_lib()
    status = lib.ref_save_cgc(str(path).encode(), ctypes.c_int(cloud.count), ctypes.c_int(cloud.sh_degree), *cargs,
                              ctypes.c_int(preset), ctypes.c_int(int(fast)), stats.ctypes.data_as(ctypes.c_void_p))
    if status != 0:
        raise ValueError(f"the reference's save_cgc refused {path}")
    return {"bytes": int(stats[0]), "layer_counts": [int(v) for v in stats[1:]]}


def ref_load_cgc(path) -> Cloud:
    """The reference's load_cgc (src/splat/cgc.cpp); raises ValueError where it throws."""
    lib = ref_lib()
    n, d = ctypes.c_int(), ctypes.c_int()
    if lib.ref_load_cgc(str(path).encode(), ctypes.byref(n), ctypes.byref(d), None, None, None, None, None) != 0:
        raise ValueError(f"the reference's load_cgc refused {path}")
    arrays = [np.zeros(n.value * k, np.float32) for k in (3, 3, 4, 1, 3 * (d.value + 1) ** 2)]
    assert lib.ref_load_cgc(str(path).encode(), ctypes.byref(n), ctypes.byref(d), *[_fp(a) for a in arrays]) == 0
    return Cloud(d.value, *arrays)


def ref_cgc_morton(x: int, y: int, z: int) -> int:
    """cgc_detail::morton_code (src/splat/cgc.hpp:53-55)."""
    lib = ref_lib()
    lib.ref_cgc_morton.restype = ctypes.c_uint64
    return int(lib.ref_cgc_morton(ctypes.c_uint32(x), ctypes.c_uint32(y), ctypes.c_uint32(z)))


def ref_cgc_canonicalize(scales, wxyz):
    """cgc_detail::canonicalize_axes (src/splat/cgc.hpp:57-58): new (scales, quaternion)."""
    s = np.array(scales, np.float32)
    q = np.array(wxyz, np.float32)
    ref_lib().ref_cgc_canonicalize(_fp(s), _fp(q))
    return s, q


def ref_lzma_compress(data: bytes, level: int = 9, extreme: bool = True, lc: int = 3, lp: int = 0, pb: int = 2) -> bytes:
    """lzma_compress (src/splat/lzma.hpp:13) over the shim."""
    lib = ref_lib()
    lib.ref_lzma_compress.restype = ctypes.c_longlong
    buf = np.frombuffer(data, np.uint8) if data else np.zeros(1, np.uint8)
    args = (buf.ctypes.data_as(ctypes.c_void_p), ctypes.c_size_t(len(data)), ctypes.c_int(level), ctypes.c_int(int(extreme)),
            ctypes.c_int(lc), ctypes.c_int(lp), ctypes.c_int(pb))
    size = lib.ref_lzma_compress(*args, None, ctypes.c_size_t(0))
    assert size >= 0
    out = np.zeros(max(size, 1), np.uint8)
    assert lib.ref_lzma_compress(*args, out.ctypes.data_as(ctypes.c_void_p), ctypes.c_size_t(size)) == size
    return out[:size].tobytes()


def ref_marked_pixels(cloud: Cloud, view: View, target: np.ndarray, share: float, background=(0.0, 0.0, 0.0),
                      near: float = 0.01) -> np.ndarray:
    """reference_marked_pixels: per Gaussian, the pixels it reaches whose mean
    error is at least `share` of the worst (target RGBA8)."""
    lib = ref_lib()
    keep, cargs = _cloud_args(cloud)
    ckeep, camargs = _camera_args(view)
    out = np.zeros(cloud.count)
    bg = np.array(background, np.float32)
    t = np.ascontiguousarray(target, np.uint8)
    assert lib.ref_marked_pixels(ctypes.c_int(cloud.count), ctypes.c_int(cloud.sh_degree), *cargs, *camargs,
                                 t.ctypes.data_as(_U8), ctypes.c_double(share), _fp(bg), ctypes.c_float(near),
                                 _dp(out)) == 0
    return out


def ref_loss(rgb: np.ndarray, width: int, height: int, target: np.ndarray, lam: float):
    """reference_loss: (loss, l1, ssim, adjoint [P,3])."""
    lib = ref_lib()
    rgb = np.ascontiguousarray(rgb, np.float64).ravel()
    t = np.ascontiguousarray(target, np.uint8).ravel()
    adj = np.zeros(width * height * 3)
    totals = np.zeros(3)
    assert lib.ref_loss(ctypes.c_int(width), ctypes.c_int(height), _dp(rgb), t.ctypes.data_as(_U8), ctypes.c_double(lam),
                        _dp(adj), _dp(totals)) == 0
    return totals[0], totals[1], totals[2], adj.reshape(-1, 3)


@dataclass
class RefGradients:
    positions: np.ndarray
    scales: np.ndarray
    rotations: np.ndarray
    opacities: np.ndarray
    sh: np.ndarray
    absolute_centre: np.ndarray


def ref_gradients(cloud: Cloud, view: View, adjoint: np.ndarray, background=(0.0, 0.0, 0.0), near: float = 0.01,
                  no_cutoffs: bool = False, opacity_reg: float = 0.0, scale_reg: float = 0.0) -> RefGradients:
    lib = ref_lib()
    keep, cargs = _cloud_args(cloud)
    ckeep, camargs = _camera_args(view)
    a = np.ascontiguousarray(adjoint, np.float64).ravel()
    n = cloud.count
    out = RefGradients(*(np.zeros(k) for k in (n * 3, n * 3, n * 4, n, cloud.sh.size, n * 2)))
    bg = np.array(background, np.float32)
    assert lib.ref_gradients(ctypes.c_int(n), ctypes.c_int(cloud.sh_degree), *cargs, *camargs, _dp(a), _fp(bg),
                             ctypes.c_float(near), ctypes.c_int(1 if no_cutoffs else 0), ctypes.c_float(opacity_reg),
                             ctypes.c_float(scale_reg), None, _dp(out.positions), _dp(out.scales), _dp(out.rotations),
                             _dp(out.opacities), _dp(out.sh), _dp(out.absolute_centre)) == 0
    return out


# ----------------------------------------------------------------- the FP32 restatement


class OView(ctypes.Structure):
    _fields_ = [("R", ctypes.c_float * 9), ("T", ctypes.c_float * 3), ("pos", ctypes.c_float * 3),
                ("nearPlane", ctypes.c_float), ("fx", ctypes.c_float), ("fy", ctypes.c_float), ("cx", ctypes.c_float),
                ("cy", ctypes.c_float), ("widthF", ctypes.c_float), ("heightF", ctypes.c_float), ("tanX", ctypes.c_float),
                ("tanY", ctypes.c_float), ("width", ctypes.c_int), ("height", ctypes.c_int), ("gridW", ctypes.c_int),
                ("gridH", ctypes.c_int), ("activeDegree", ctypes.c_int), ("activeCoeffs", ctypes.c_int),
                ("perPixel", ctypes.c_float), ("fixedScale", ctypes.c_float)]


def oview(view: View, degree: int, near: float = 0.01) -> OView:
    """The per-view constants exactly as the CUDA trainer computes them (float32)."""
    v = OView()
    m = np.asarray(view.view, np.float32)
    for r in range(3):
        for c in range(3):
            v.R[r * 3 + c] = float(m[r, c])
        v.T[r] = float(m[r, 3])
        v.pos[r] = float(np.float32(view.position[r]))
    f32 = np.float32
    v.nearPlane = near
    v.fx, v.fy, v.cx, v.cy = float(f32(view.fx)), float(f32(view.fy)), float(f32(view.cx)), float(f32(view.cy))
    v.widthF, v.heightF = float(view.width), float(view.height)
    v.tanX = float(f32(0.5) * f32(view.width) / f32(view.fx))
    v.tanY = float(f32(0.5) * f32(view.height) / f32(view.fy))
    v.width, v.height = view.width, view.height
    v.gridW, v.gridH = (view.width + 15) // 16, (view.height + 15) // 16
    v.activeDegree, v.activeCoeffs = degree, (degree + 1) ** 2
    v.perPixel = float(f32(1.0) / (f32(3.0) * f32(view.width) * f32(view.height)))
    v.fixedScale = float(f32(3.0) * f32(view.width) * f32(view.height) * f32(64.0))
    return v


def round_sh_like_device(sh: np.ndarray, degree: int, storage: str) -> np.ndarray:
    """SH as the device holds it: DC in FP32, the rest rounded to nearest in f32/f16/bf16."""
    coeffs = (degree + 1) ** 2
    s = np.asarray(sh, np.float32).reshape(-1, coeffs * 3).copy()
    rest = s[:, 3:]
    if storage == "f16":
        rest = rest.astype(np.float16).astype(np.float32)
    elif storage == "bf16":
        bits = rest.view(np.uint32).astype(np.uint64)
        bits = ((bits + 0x7FFF + ((bits >> 16) & 1)) >> 16) << 16
        rest = bits.astype(np.uint32).view(np.float32)
    s[:, 3:] = rest
    return s.ravel()


def preprocess(cloud: Cloud, view: View, degree: int | None = None, sh_storage: str = "f32", near: float = 0.01):
    """oracle_preprocess: (splats [n,12], reach [n], keys [n] uint32)."""
    lib = oracle_lib()
    deg = cloud.sh_degree if degree is None else degree
    n = cloud.count
    splats, reach, keys = np.zeros(n * 12, np.float32), np.zeros(n, np.float32), np.zeros(n, np.uint32)
    sh = round_sh_like_device(cloud.sh, cloud.sh_degree, sh_storage)
    keep, cargs = _cloud_args(Cloud(cloud.sh_degree, cloud.positions, cloud.scales, cloud.rotations, cloud.opacities, sh))
    v = oview(view, deg, near)
    lib.oracle_preprocess(ctypes.c_int(n), ctypes.c_int(cloud.coeffs), *cargs, ctypes.byref(v), _fp(splats), _fp(reach),
                          keys.ctypes.data_as(_U32))
    return splats.reshape(n, 12), reach, keys


def bin_entries(splats: np.ndarray, reach: np.ndarray, item_keys: np.ndarray, order: np.ndarray | None, view: View,
                degree: int = 0):
    """oracle_bin: (entry tiles, entry splat indices) in emission order."""
    lib = oracle_lib()
    v = oview(view, degree)
    s = np.ascontiguousarray(splats, np.float32).ravel()
    r = np.ascontiguousarray(reach, np.float32)
    k = np.ascontiguousarray(item_keys, np.uint32)
    o = None if order is None else np.ascontiguousarray(order, np.uint32)
    lib.oracle_bin.restype = ctypes.c_int64
    total = lib.oracle_bin(ctypes.c_int(k.size), None if o is None else o.ctypes.data_as(_U32), k.ctypes.data_as(_U32),
                           _fp(s), _fp(r), ctypes.byref(v), None, None, ctypes.c_int64(0))
    tiles, values = np.zeros(max(total, 1), np.uint32), np.zeros(max(total, 1), np.uint32)
    lib.oracle_bin(ctypes.c_int(k.size), None if o is None else o.ctypes.data_as(_U32), k.ctypes.data_as(_U32), _fp(s),
                   _fp(r), ctypes.byref(v), tiles.ctypes.data_as(_U32), values.ctypes.data_as(_U32), ctypes.c_int64(total))
    return tiles[:total], values[:total]


def ranges(tiles_sorted: np.ndarray, tile_count: int) -> np.ndarray:
    out = np.zeros(tile_count * 2, np.uint32)
    t = np.ascontiguousarray(tiles_sorted, np.uint32)
    oracle_lib().oracle_ranges(ctypes.c_int64(t.size), t.ctypes.data_as(_U32), out.ctypes.data_as(_U32))
    return out.reshape(tile_count, 2)


def forward(splats, entry_values, tile_ranges, view: View, background=(0.0, 0.0, 0.0), degree: int = 0):
    """oracle_forward: (image [P,4] float32, stops [P] uint32)."""
    lib = oracle_lib()
    v = oview(view, degree)
    P = view.width * view.height
    image, stops = np.zeros(P * 4, np.float32), np.zeros(P, np.uint32)
    s = np.ascontiguousarray(splats, np.float32).ravel()
    e = np.ascontiguousarray(entry_values, np.uint32)
    r = np.ascontiguousarray(tile_ranges, np.uint32).ravel()
    bg = np.array(background, np.float32)
    lib.oracle_forward(_fp(s), e.ctypes.data_as(_U32), r.ctypes.data_as(_U32), ctypes.byref(v), _fp(bg), _fp(image),
                       stops.ctypes.data_as(_U32))
    return image.reshape(P, 4), stops


def loss(image: np.ndarray, target: np.ndarray, view: View, lam: float):
    """oracle_loss: (adjoint [P,4], ssim sum, l1 sum)."""
    lib = oracle_lib()
    v = oview(view, 0)
    P = view.width * view.height
    img = np.ascontiguousarray(image, np.float32).ravel()
    t = np.ascontiguousarray(target, np.uint8).ravel()
    adj = np.zeros(P * 4, np.float32)
    ssim, l1 = ctypes.c_double(), ctypes.c_double()
    lib.oracle_loss(_fp(img), t.ctypes.data_as(_U8), ctypes.byref(v), ctypes.c_float(lam), _fp(adj), ctypes.byref(ssim),
                    ctypes.byref(l1))
    return adj.reshape(P, 4), ssim.value, l1.value


def backward(splats, entry_values, tile_ranges, view: View, image, adjoint, stops, fixed: bool, count: int,
             background=(0.0, 0.0, 0.0)):
    """oracle_backward: raw sums [count, 16] (int32 when fixed, else float32)."""
    lib = oracle_lib()
    v = oview(view, 0)
    raw = np.zeros(count * 16, np.int32 if fixed else np.float32)
    s = np.ascontiguousarray(splats, np.float32).ravel()
    e = np.ascontiguousarray(entry_values, np.uint32)
    r = np.ascontiguousarray(tile_ranges, np.uint32).ravel()
    img = np.ascontiguousarray(image, np.float32).ravel()
    adj = np.ascontiguousarray(adjoint, np.float32).ravel()
    st = np.ascontiguousarray(stops, np.uint32)
    bg = np.array(background, np.float32)
    lib.oracle_backward(_fp(s), e.ctypes.data_as(_U32), r.ctypes.data_as(_U32), ctypes.byref(v), _fp(bg), _fp(img),
                        _fp(adj), st.ctypes.data_as(_U32), ctypes.c_int(1 if fixed else 0), raw.ctypes.data_as(ctypes.c_void_p))
    return raw.reshape(count, 16)


def stable_order(keys: np.ndarray) -> np.ndarray:
    """std::stable_sort order of the keys (the sort test's expectation)."""
    return np.argsort(keys, kind="stable").astype(np.uint32)


# ----------------------------------------------------------------- deterministic math on the host


def detmath(x: np.ndarray):
    """splat_expf and splat_logf of include/splat_detmath.h on the host: (exp, log)."""
    x = np.ascontiguousarray(x, np.float32)
    e, l = np.zeros_like(x), np.zeros_like(x)
    oracle_lib().oracle_detmath(_fp(x), _fp(e), _fp(l), ctypes.c_int(x.size))
    return e, l
