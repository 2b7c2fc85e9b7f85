"""splat_b200: the training step of vibe-splat's tile-based differentiable
Gaussian rasterizer, on one B200, behind the C ABI of include/splat_b200.h.

This module mirrors the reference's C++ trainer interface (splat::Trainer,
src/train/trainer.hpp:89-270; TrainerOptions :24-42, LearningRates :51-61,
StepStats :63-73; GaussianCloud src/splat/gaussian_cloud.hpp:145-162; Camera
src/render/camera.hpp:84-93) with the same names, argument meanings and error
behaviour: the reference throws BudgetExceeded, std::runtime_error and
std::logic_error, and so does this module (BudgetExceeded, RuntimeError,
StateError). The compute runs only in the CUDA library libsplat_b200.so; if it
is missing, importing this module fails.

The package directory name has a hyphen, so import it with
importlib.import_module("vibe-splat_b200").
"""
from __future__ import annotations

import ctypes
import math
import os
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
LIBRARY_PATH = _HERE / "libsplat_b200.so"

if not LIBRARY_PATH.exists():
    raise ImportError(
        f"{LIBRARY_PATH} is missing: build it with `python vibe-splat_b200/_build.py` "
        "(or __graft_entry__.build()); there is no CPU fallback"
    )

_lib = ctypes.CDLL(str(LIBRARY_PATH))

# ----------------------------------------------------------------- C structs

SPLAT_OK = 0
SPLAT_ERR_INVALID = 1
SPLAT_ERR_BUDGET = 2
SPLAT_ERR_UNSUPPORTED = 3
SPLAT_ERR_DEVICE = 4
SPLAT_ERR_NONFINITE = 5
SPLAT_ERR_STATE = 6
SPLAT_ERR_NOMEM = 7

SH_F32, SH_BF16, SH_F16 = 0, 1, 2
STATE_F32, STATE_BF16_PAIR = 0, 1
SORT_DEPTH_THEN_TILE, SORT_TILE_DEPTH_64 = 0, 1


class _Options(ctypes.Structure):
    _fields_ = [
        ("lambda_ssim", ctypes.c_float),
        ("background", ctypes.c_float * 3),
        ("near_plane", ctypes.c_float),
        ("force_fixed_point", ctypes.c_int32),
        ("selective_adam", ctypes.c_int32),
        ("opacity_reg", ctypes.c_float),
        ("scale_reg", ctypes.c_float),
        ("position_noise", ctypes.c_float),
        ("mip_filter_2d", ctypes.c_int32),
        ("pose_gradients", ctypes.c_int32),
        ("memory_budget", ctypes.c_uint64),
        ("sh_storage", ctypes.c_int32),
        ("state_storage", ctypes.c_int32),
        ("sort_form", ctypes.c_int32),
        ("exact_math", ctypes.c_int32),
        ("use_graph", ctypes.c_int32),
        ("digit_bits", ctypes.c_int32),
        ("forward_pixels_per_thread", ctypes.c_int32),
        ("backward_pixels_per_thread", ctypes.c_int32),
        ("split_step", ctypes.c_int32),
        ("blend_lists", ctypes.c_int32),
        ("tile_size", ctypes.c_int32),
        ("batch_depth", ctypes.c_int32),
        ("persistent_raster", ctypes.c_int32),
        ("grouped_backward", ctypes.c_int32),
    ]


class _Rates(ctypes.Structure):
    _fields_ = [(name, ctypes.c_float) for name in
                ("position", "scale", "rotation", "opacity", "sh", "sh_rest_scale", "trust_region")]


class _Stats(ctypes.Structure):
    _fields_ = [
        ("loss", ctypes.c_float),
        ("l1", ctypes.c_float),
        ("ssim", ctypes.c_float),
        ("visible_splats", ctypes.c_uint32),
        ("tile_entries", ctypes.c_uint32),
        ("exposure_gradient", ctypes.c_float * 12),
        ("pose_gradient", ctypes.c_float * 6),
    ]


class _Camera(ctypes.Structure):
    _fields_ = [
        ("view", ctypes.c_float * 16),
        ("position", ctypes.c_float * 3),
        ("fx", ctypes.c_float),
        ("fy", ctypes.c_float),
        ("cx", ctypes.c_float),
        ("cy", ctypes.c_float),
        ("width", ctypes.c_int32),
        ("height", ctypes.c_int32),
    ]


_FP = ctypes.POINTER(ctypes.c_float)


class _Cloud(ctypes.Structure):
    _fields_ = [
        ("count", ctypes.c_int32),
        ("sh_degree", ctypes.c_int32),
        ("positions", _FP),
        ("scales", _FP),
        ("rotations", _FP),
        ("opacities", _FP),
        ("sh", _FP),
    ]


_P = ctypes.c_void_p
_lib.splat_last_error.restype = ctypes.c_char_p
_lib.splat_trainer_options_default.argtypes = [ctypes.POINTER(_Options)]
_lib.splat_learning_rates_default.argtypes = [ctypes.POINTER(_Rates)]
_lib.splat_trainer_create.argtypes = [ctypes.POINTER(_Cloud), ctypes.POINTER(_Options), ctypes.POINTER(_P)]
_lib.splat_trainer_destroy.argtypes = [_P]
_lib.splat_trainer_render.argtypes = [_P, ctypes.POINTER(_Camera), _FP]
_lib.splat_trainer_compute_gradients.argtypes = [_P, ctypes.POINTER(_Camera), _P, ctypes.c_size_t, ctypes.POINTER(_Stats)]
_lib.splat_trainer_collect_statistics.argtypes = [_P, ctypes.POINTER(_Camera), _P, ctypes.c_size_t, ctypes.POINTER(_Stats)]
_lib.splat_trainer_score_view.argtypes = [_P, ctypes.POINTER(_Camera), _P, ctypes.c_size_t, ctypes.c_float,
                                         ctypes.c_float, ctypes.POINTER(_Stats)]
_lib.splat_trainer_apply_gradients.argtypes = [_P, ctypes.POINTER(_Rates)]
_lib.splat_trainer_step.argtypes = [_P, ctypes.POINTER(_Camera), _P, ctypes.c_size_t, ctypes.POINTER(_Rates), _P,
                                    ctypes.c_size_t, ctypes.POINTER(_Stats)]
_lib.splat_trainer_step_batch.argtypes = [_P, ctypes.POINTER(_Camera), ctypes.POINTER(_P), ctypes.c_int32,
                                          ctypes.POINTER(_Rates), ctypes.POINTER(_Stats)]
_lib.splat_trainer_prefetch_target.argtypes = [_P, _P, ctypes.c_size_t]
_lib.splat_trainer_step_device_target.argtypes = [_P, ctypes.POINTER(_Camera), _P, ctypes.c_size_t, ctypes.POINTER(_Rates),
                                                  ctypes.POINTER(_Stats)]
_lib.splat_trainer_stream.argtypes = [_P, ctypes.POINTER(_P)]


class _Autotune(ctypes.Structure):
    _fields_ = [("sort_form", ctypes.c_int32), ("digit_bits", ctypes.c_int32),
                ("forward_pixels_per_thread", ctypes.c_int32), ("backward_pixels_per_thread", ctypes.c_int32),
                ("ms", (ctypes.c_double * 3) * 2), ("layout_ms", (ctypes.c_double * 2) * 2),
                ("tile_size", ctypes.c_int32), ("batch_depth", ctypes.c_int32), ("persistent_raster", ctypes.c_int32),
                ("tile_ms", ((ctypes.c_double * 2) * 2) * 2), ("grouped_backward", ctypes.c_int32),
                ("grouped_ms", ((ctypes.c_double * 2) * 2) * 2)]


_lib.splat_trainer_autotune.argtypes = [_P, ctypes.POINTER(_Camera), _P, ctypes.c_size_t, ctypes.c_int32,
                                        ctypes.POINTER(_Autotune)]
_lib.splat_trainer_get_gradients.argtypes = [_P, _FP, _FP, _FP, _FP, _FP]
_lib.splat_trainer_get_cloud.argtypes = [_P, _FP, _FP, _FP, _FP, _FP]
_lib.splat_trainer_set_active_sh_degree.argtypes = [_P, ctypes.c_int32]
_lib.splat_trainer_get_densify_stats.argtypes = [_P, _FP]
_lib.splat_trainer_reset_densify_stats.argtypes = [_P]
_lib.splat_trainer_set_densify_stats.argtypes = [_P, _FP]
_lib.splat_trainer_reset_opacity.argtypes = [_P, ctypes.c_float]
_lib.splat_trainer_apply_changes.argtypes = [_P, ctypes.POINTER(_Cloud), ctypes.POINTER(ctypes.c_int32)]
_lib.splat_trainer_info.argtypes = [_P, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int32),
                                    ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int32),
                                    ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64)]
_lib.splat_trainer_timings.argtypes = [_P, ctypes.POINTER(ctypes.c_char_p), ctypes.POINTER(ctypes.c_double),
                                       ctypes.c_int32, ctypes.POINTER(ctypes.c_int32)]
_lib.splat_trainer_set_timing.argtypes = [_P, ctypes.c_int32]
_lib.splat_trainer_device_parameters.argtypes = [_P, ctypes.c_int32, ctypes.POINTER(ctypes.c_uint64),
                                                 ctypes.POINTER(ctypes.c_uint64)]
_lib.splat_trainer_debug_download.argtypes = [_P, ctypes.c_int32, _P, ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)]
_lib.splat_radix_sort_u32.argtypes = [_P, _P, _P, _P, ctypes.c_uint32, ctypes.c_int32, ctypes.c_int32, _P]
_lib.splat_radix_sort_u64.argtypes = [_P, _P, _P, _P, ctypes.c_uint32, ctypes.c_int32, ctypes.c_int32, _P]
_lib.splat_debug_detmath.argtypes = [_P, _P, _P, ctypes.c_uint32]


class _SmPeaks(ctypes.Structure):
    _fields_ = [("fp32_flops", ctypes.c_double), ("sfu_ops", ctypes.c_double), ("shared_bytes", ctypes.c_double),
                ("warp_instructions", ctypes.c_double)]


_lib.splat_measure_sm_peaks.argtypes = [ctypes.POINTER(_SmPeaks)]
_lib.splat_cloud_load_ply.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int32),
                                      _FP, _FP, _FP, _FP, _FP]
_lib.splat_cloud_save_ply.argtypes = [ctypes.c_char_p, ctypes.POINTER(_Cloud)]


class _CgcOptions(ctypes.Structure):
    _fields_ = [("preset", ctypes.c_int32), ("fast", ctypes.c_int32)]


class _CgcStats(ctypes.Structure):
    _fields_ = [("bytes", ctypes.c_uint64), ("layer_counts", ctypes.c_uint64 * 3)]


_lib.splat_cloud_save_cgc.argtypes = [ctypes.c_char_p, ctypes.POINTER(_Cloud), ctypes.POINTER(_CgcOptions),
                                      ctypes.POINTER(_CgcStats)]
_lib.splat_cloud_load_cgc.argtypes = _lib.splat_cloud_load_ply.argtypes
_lib.splat_cgc_morton_code.argtypes = [ctypes.c_uint32] * 3
_lib.splat_cgc_morton_code.restype = ctypes.c_uint64
_lib.splat_cgc_canonicalize_axes.argtypes = [_FP, _FP]
_lib.splat_lzma_compress.argtypes = [_P, ctypes.c_size_t] + [ctypes.c_int32] * 5 + [_P, ctypes.c_size_t,
                                                                                     ctypes.POINTER(ctypes.c_size_t)]
_lib.splat_lzma_decompress.argtypes = [_P, ctypes.c_size_t, _P, ctypes.c_size_t]
for _name in ("splat_trainer_remove_largest", "splat_trainer_remove_least_contributing", "splat_trainer_remove_least_opaque"):
    getattr(_lib, _name).argtypes = [_P, ctypes.c_double, ctypes.POINTER(ctypes.c_uint64)]
_lib.splat_trainer_set_exposure.argtypes = [_P, _FP]


class _DensifyOptions(ctypes.Structure):
    _fields_ = [("gradient_threshold", ctypes.c_float), ("dense_scale", ctypes.c_float), ("prune_opacity", ctypes.c_float),
                ("prune_large", ctypes.c_int32), ("max_screen_radius", ctypes.c_float), ("max_world_scale", ctypes.c_float),
                ("max_gaussians", ctypes.c_uint64), ("split_threshold", ctypes.c_float), ("scored_views", ctypes.c_int32),
                ("min_marked_pixels", ctypes.c_float), ("transparent_share", ctypes.c_double),
                ("explore_splits", ctypes.c_uint64), ("explore_seeds", ctypes.c_uint64), ("edge_split", ctypes.c_int32)]


class _DensifyResult(ctypes.Structure):
    _fields_ = [(name, ctypes.c_uint64) for name in ("count", "cloned", "split", "seeded", "pruned", "held_back")]


class _RelocateOptions(ctypes.Structure):
    _fields_ = [("min_opacity", ctypes.c_float), ("growth", ctypes.c_double), ("max_gaussians", ctypes.c_uint64)]


_lib.splat_relocate_options_default.argtypes = [ctypes.POINTER(_RelocateOptions)]
_lib.splat_trainer_relocate.argtypes = [_P, ctypes.POINTER(_RelocateOptions), _P, ctypes.POINTER(_DensifyResult),
                                        ctypes.POINTER(ctypes.c_int64), ctypes.c_uint64]
class _SessionOptions(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int32), ("sh_degree", ctypes.c_int32), ("seed", ctypes.c_uint32),
                ("report_every", ctypes.c_int32), ("densify", ctypes.c_int32), ("densify_mode", ctypes.c_int32),
                ("full_adam", ctypes.c_int32), ("full_resolution", ctypes.c_int32), ("adaptive_schedule", ctypes.c_int32),
                ("gradient_threshold", ctypes.c_float), ("split_threshold", ctypes.c_float), ("dense_fraction", ctypes.c_double),
                ("densify_interval", ctypes.c_int32), ("score_views", ctypes.c_int32), ("score_min_pixels", ctypes.c_float),
                ("explore", ctypes.c_int32), ("significance_prune", ctypes.c_int32), ("edge_split", ctypes.c_int32),
                ("threshold_rise", ctypes.c_double), ("prune_share", ctypes.c_double), ("recovery_prune", ctypes.c_double),
                ("max_growth", ctypes.c_double), ("max_gaussians", ctypes.c_uint64), ("coarse_until", ctypes.c_double * 2),
                ("views_per_step", ctypes.c_int32)]


class _SessionData(ctypes.Structure):
    _fields_ = [("points", ctypes.POINTER(ctypes.c_double)), ("colors", ctypes.POINTER(ctypes.c_uint8)),
                ("point_count", ctypes.c_uint64), ("cameras", ctypes.POINTER(_Camera)), ("images", ctypes.POINTER(_P)),
                ("views", ctypes.c_int32), ("extent", ctypes.c_double), ("typical_depth", ctypes.c_double)]


class _SessionState(ctypes.Structure):
    _fields_ = [("iteration", ctypes.c_int32), ("level", ctypes.c_int32), ("view", ctypes.c_int32),
                ("views_in_step", ctypes.c_int32), ("position_rate", ctypes.c_float), ("gaussians", ctypes.c_uint64), ("first_loss", ctypes.c_float),
                ("last_loss", ctypes.c_float), ("report_iteration", ctypes.c_int32), ("probe_psnr", ctypes.c_double),
                ("mean_loss", ctypes.c_double), ("densify_rounds", ctypes.c_int32), ("densify_seconds", ctypes.c_double),
                ("last_densify", _DensifyResult), ("held_back_total", ctypes.c_uint64), ("pruned_total", ctypes.c_uint64),
                ("coarse_until", ctypes.c_double * 2)]


_lib.splat_session_options_default.argtypes = [ctypes.POINTER(_SessionOptions)]
_lib.splat_session_create.argtypes = [ctypes.POINTER(_SessionData), ctypes.POINTER(_SessionOptions), ctypes.POINTER(_Options),
                                      ctypes.POINTER(_P)]
_lib.splat_session_destroy.argtypes = [_P]
_lib.splat_session_step.argtypes = [_P, ctypes.POINTER(_Stats)]
_lib.splat_session_get_state.argtypes = [_P, ctypes.POINTER(_SessionState)]
_lib.splat_session_trainer.argtypes = [_P, ctypes.POINTER(_P)]
_lib.splat_frequency_energy.argtypes = [_P, ctypes.c_int32, ctypes.c_int32, ctypes.POINTER(ctypes.c_int32), ctypes.c_int32,
                                        ctypes.POINTER(ctypes.c_double)]
_lib.splat_resolution_switches.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.POINTER(ctypes.c_double)]
_lib.splat_growth_limit.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.POINTER(ctypes.c_uint64), ctypes.c_int32,
                                    ctypes.c_double, ctypes.c_double, ctypes.POINTER(ctypes.c_uint64),
                                    ctypes.POINTER(ctypes.c_double)]
_lib.splat_half_size.argtypes = [_P, ctypes.c_int32, ctypes.c_int32, _P]
_lib.splat_initial_cloud.argtypes = [ctypes.POINTER(ctypes.c_double), _P, ctypes.c_uint64, ctypes.c_int32, _FP, _FP, _FP, _FP, _FP]
_lib.splat_trainer_step_batch_device_targets.argtypes = [_P, ctypes.POINTER(_Camera), ctypes.POINTER(_P), ctypes.c_int32,
                                                         ctypes.POINTER(_Rates), ctypes.POINTER(_Stats)]
_lib.splat_trainer_collect_statistics_device_target.argtypes = [_P, ctypes.POINTER(_Camera), _P, ctypes.c_size_t,
                                                                ctypes.POINTER(_Stats)]
_lib.splat_trainer_score_view_device_target.argtypes = [_P, ctypes.POINTER(_Camera), _P, ctypes.c_size_t, ctypes.c_float,
                                                        ctypes.c_float, ctypes.POINTER(_Stats)]
_lib.splat_rng_create.argtypes = [ctypes.c_uint32, ctypes.POINTER(_P)]
_lib.splat_rng_destroy.argtypes = [_P]
_lib.splat_rng_pick.argtypes = [_P, ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint64)]
_lib.splat_densify_options_default.argtypes = [ctypes.POINTER(_DensifyOptions)]
_lib.splat_trainer_densify.argtypes = [_P, ctypes.POINTER(_DensifyOptions), _P, ctypes.POINTER(_DensifyResult),
                                       ctypes.POINTER(ctypes.c_int64), ctypes.c_uint64]
_lib.splat_trainer_set_sh_dropout.argtypes = [_P, ctypes.c_float, ctypes.c_int32, ctypes.c_uint32]
_lib.splat_trainer_set_filter3d.argtypes = [_P, _FP, ctypes.c_size_t]
_lib.splat_trainer_add_position_noise.argtypes = [_P, ctypes.c_float, ctypes.c_uint32]
_lib.splat_trainer_enable_second_order.argtypes = [_P]
_lib.splat_trainer_update_curvature.argtypes = [_P]

# ----------------------------------------------------------------- errors


class SplatError(RuntimeError):
    """A failed call; .status is the splat_status code."""

    def __init__(self, status: int, message: str):
        super().__init__(message)
        self.status = status


class BudgetExceeded(SplatError):
    """A view would need more memory than the budget allows (trainer.hpp:46-49). The
    trainer is still usable: remove Gaussians and try again."""


class UnsupportedOption(SplatError):
    """An option of the reference that this library has no kernel for."""


class DeviceError(SplatError):
    """A CUDA error or a failed device-side check."""


class NonFiniteLoss(SplatError):
    """The loss came out NaN or infinite."""


class StateError(SplatError):
    """Called in the wrong order, as the reference's std::logic_error (trainer.cpp:853)."""


_ERRORS = {
    SPLAT_ERR_BUDGET: BudgetExceeded,
    SPLAT_ERR_UNSUPPORTED: UnsupportedOption,
    SPLAT_ERR_DEVICE: DeviceError,
    SPLAT_ERR_NONFINITE: NonFiniteLoss,
    SPLAT_ERR_STATE: StateError,
    SPLAT_ERR_NOMEM: DeviceError,
}


def _check(status: int) -> None:
    if status != SPLAT_OK:
        message = _lib.splat_last_error().decode()
        raise _ERRORS.get(status, SplatError)(status, message)


# ----------------------------------------------------------------- value types


@dataclass
class GaussianCloud:
    """The reference's GaussianCloud: raw parameters as in a 3DGS .ply."""

    sh_degree: int = 0
    positions: np.ndarray = field(default_factory=lambda: np.zeros(0, np.float32))
    scales: np.ndarray = field(default_factory=lambda: np.zeros(0, np.float32))
    rotations: np.ndarray = field(default_factory=lambda: np.zeros(0, np.float32))
    opacities: np.ndarray = field(default_factory=lambda: np.zeros(0, np.float32))
    sh: np.ndarray = field(default_factory=lambda: np.zeros(0, np.float32))

    def size(self) -> int:
        return int(np.asarray(self.opacities).size)

    def sh_coeffs(self) -> int:
        return (self.sh_degree + 1) ** 2

    def validate(self) -> None:
        n = self.size()
        if not 0 <= self.sh_degree <= 3:
            raise RuntimeError("GaussianCloud: SH degree must be 0..3")
        sizes = (self.positions.size, self.scales.size, self.rotations.size, self.sh.size)
        if sizes != (n * 3, n * 3, n * 4, n * 3 * self.sh_coeffs()):
            raise RuntimeError("GaussianCloud: inconsistent array sizes")

    def _c(self):
        arrays = [np.ascontiguousarray(np.asarray(a, dtype=np.float32).ravel())
                  for a in (self.positions, self.scales, self.rotations, self.opacities, self.sh)]
        c = _Cloud(self.size(), self.sh_degree, *[a.ctypes.data_as(_FP) for a in arrays])
        return c, arrays

    def copy(self) -> "GaussianCloud":
        return GaussianCloud(self.sh_degree, *(np.array(a, dtype=np.float32, copy=True) for a in
                                               (self.positions, self.scales, self.rotations, self.opacities, self.sh)))


@dataclass
class Camera:
    """The reference's Camera: OpenCV pinhole, world->camera view matrix (4x4,
    as a numpy array indexed [row, column])."""

    view: np.ndarray = field(default_factory=lambda: np.eye(4, dtype=np.float32))
    position: np.ndarray = field(default_factory=lambda: np.zeros(3, np.float32))
    fx: float = 1.0
    fy: float = 1.0
    cx: float = 0.0
    cy: float = 0.0
    width: int = 1
    height: int = 1

    def _c(self) -> _Camera:
        # Whole-array assignments: a step spends no more host time here than
        # it must (the GPU waits on the host between synchronous steps).
        c = _Camera()
        c.view[:] = np.asarray(self.view, dtype=np.float32).T.reshape(16).tolist()  # column-major
        c.position[:] = np.asarray(self.position, dtype=np.float32).reshape(-1)[:3].tolist()
        c.fx, c.fy, c.cx, c.cy = float(self.fx), float(self.fy), float(self.cx), float(self.cy)
        c.width, c.height = int(self.width), int(self.height)
        return c

    @staticmethod
    def look_at(eye, target, up, fx: float, width: int, height: int, fy: float | None = None) -> "Camera":
        """A camera at `eye` looking at `target` (x right, y down, z forward)."""
        eye = np.asarray(eye, np.float64)
        forward = np.asarray(target, np.float64) - eye
        forward /= np.linalg.norm(forward)
        right = np.cross(forward, np.asarray(up, np.float64))
        if np.linalg.norm(right) < 1e-9:
            right = np.cross(forward, np.array([1.0, 0.0, 0.0]))
        right /= np.linalg.norm(right)
        down = np.cross(forward, right)
        rot = np.stack([right, down, forward])
        view = np.eye(4)
        view[:3, :3] = rot
        view[:3, 3] = -rot @ eye
        return Camera(view.astype(np.float32), eye.astype(np.float32), fx, fy if fy is not None else fx,
                      width * 0.5, height * 0.5, width, height)


@dataclass
class TrainerOptions:
    """TrainerOptions (trainer.hpp:24-42), plus the B200 knobs: SH and optimiser
    storage, sort form, exact (CPU-reproducible) or SFU exp/log, CUDA graph, and
    the radix digit width. The defaults are the reference's layout and arithmetic."""

    lambda_ssim: float = 0.2
    background: tuple = (0.0, 0.0, 0.0)
    near_plane: float = 0.01
    force_fixed_point: bool = False
    selective_adam: bool = True
    opacity_reg: float = 0.0
    scale_reg: float = 0.0
    position_noise: float = 0.0
    mip_filter_2d: bool = False
    pose_gradients: bool = False
    memory_budget: int = 2**64 - 1
    sh_storage: int = SH_F16
    state_storage: int = STATE_BF16_PAIR
    sort_form: int = SORT_DEPTH_THEN_TILE
    exact_math: bool = True
    use_graph: bool = False
    digit_bits: int = 8
    forward_pixels_per_thread: int = 1
    backward_pixels_per_thread: int = 2
    split_step: bool = False
    blend_lists: bool = False
    tile_size: int = 16
    batch_depth: int = 128
    persistent_raster: bool = False
    grouped_backward: bool = False

    def _c(self) -> _Options:
        o = _Options()
        o.lambda_ssim = self.lambda_ssim
        for c in range(3):
            o.background[c] = float(self.background[c])
        o.near_plane = self.near_plane
        o.force_fixed_point = int(self.force_fixed_point)
        o.selective_adam = int(self.selective_adam)
        o.opacity_reg, o.scale_reg, o.position_noise = self.opacity_reg, self.scale_reg, self.position_noise
        o.mip_filter_2d, o.pose_gradients = int(self.mip_filter_2d), int(self.pose_gradients)
        o.memory_budget = int(self.memory_budget)
        o.sh_storage, o.state_storage, o.sort_form = self.sh_storage, self.state_storage, self.sort_form
        o.exact_math, o.use_graph, o.digit_bits = int(self.exact_math), int(self.use_graph), self.digit_bits
        o.forward_pixels_per_thread = self.forward_pixels_per_thread
        o.backward_pixels_per_thread = self.backward_pixels_per_thread
        o.split_step = int(self.split_step)
        o.blend_lists = int(self.blend_lists)
        o.tile_size, o.batch_depth = self.tile_size, self.batch_depth
        o.persistent_raster = int(self.persistent_raster)
        o.grouped_backward = int(self.grouped_backward)
        return o


@dataclass
class LearningRates:
    """LearningRates (trainer.hpp:51-61)."""

    position: float = 1.6e-4
    scale: float = 0.005
    rotation: float = 0.001
    opacity: float = 0.05
    sh: float = 0.025
    sh_rest_scale: float = 0.05
    trust_region: float = 0.0

    def _c(self) -> _Rates:
        return _Rates(self.position, self.scale, self.rotation, self.opacity, self.sh, self.sh_rest_scale,
                      self.trust_region)


@dataclass
class DensifyOptions:
    """DensifyOptions (densify.hpp:23-50)."""

    gradient_threshold: float = 2e-4
    dense_scale: float = 0.0
    prune_opacity: float = 0.005
    prune_large: bool = False
    max_screen_radius: float = 20.0
    max_world_scale: float = 0.0
    max_gaussians: int = 2**64 - 1
    split_threshold: float = 0.0
    scored_views: int = 0
    min_marked_pixels: float = 5.0
    transparent_share: float = 1.0
    explore_splits: int = 0
    explore_seeds: int = 0
    edge_split: bool = False

    def _c(self) -> _DensifyOptions:
        o = _DensifyOptions()
        for name, _ in _DensifyOptions._fields_:
            value = getattr(self, name)
            setattr(o, name, int(value) if isinstance(value, bool) else value)
        return o


@dataclass
class RelocateOptions:
    """RelocateOptions (densify.hpp:87-91)."""

    min_opacity: float = 0.005
    growth: float = 0.05
    max_gaussians: int = 2**64 - 1

    def _c(self) -> _RelocateOptions:
        return _RelocateOptions(self.min_opacity, self.growth, int(self.max_gaussians))


@dataclass
class DensifyResult:
    """DensifyResult (densify.hpp:52-62): the counts and, per new Gaussian, the
    old index whose optimiser state it keeps (-1 for a new one)."""

    count: int
    cloned: int
    split: int
    seeded: int
    pruned: int
    held_back: int
    source: np.ndarray


class Rng:
    """The std::mt19937 densification draws from; its state carries over from
    round to round, as the reference's session keeps one (train.hpp:254)."""

    def __init__(self, seed: int):
        h = _P()
        _check(_lib.splat_rng_create(ctypes.c_uint32(seed & 0xFFFFFFFF), ctypes.byref(h)))
        self._h = h

    def pick(self, count: int) -> int:
        """std::uniform_int_distribution<std::size_t>(0, count - 1)(rng)."""
        out = ctypes.c_uint64()
        _check(_lib.splat_rng_pick(self._h, int(count), ctypes.byref(out)))
        return out.value

    def close(self) -> None:
        if getattr(self, "_h", None):
            _lib.splat_rng_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()


@dataclass
class StepStats:
    """StepStats (trainer.hpp:63-73)."""

    loss: float = 0.0
    l1: float = 0.0
    ssim: float = 0.0
    visible_splats: int = 0
    tile_entries: int = 0

    @staticmethod
    def _from(c: _Stats) -> "StepStats":
        return StepStats(c.loss, c.l1, c.ssim, c.visible_splats, c.tile_entries)


@dataclass
class Gradients:
    positions: np.ndarray
    scales: np.ndarray
    rotations: np.ndarray
    opacities: np.ndarray
    sh: np.ndarray


@dataclass
class DensifyStats:
    """DensifyStats as Trainer::densify_stats() downloads it (trainer.cpp:686-708)."""

    gradient_sum: np.ndarray
    visits: np.ndarray
    max_radius: np.ndarray
    contribution: np.ndarray
    absolute_gradient_sum: np.ndarray
    marked_pixels: np.ndarray
    marked_loss: np.ndarray
    edge_score: np.ndarray


# Buffers splat_trainer_debug_download knows.
DEBUG_SPLATS, DEBUG_REACH, DEBUG_DEPTH_KEYS, DEBUG_ENTRY_KEYS, DEBUG_ENTRY_VALUES, DEBUG_RANGES = range(6)
DEBUG_IMAGE, DEBUG_STOPS, DEBUG_ADJOINT, DEBUG_RAW, DEBUG_COUNTERS, DEBUG_PARTIALS, DEBUG_ERROR = range(6, 13)
DEBUG_BLEND_COUNTS = 13
DEBUG_STATE = 14  # + parameter group 0..4
DEBUG_TILE_SCHEDULE = 19  # per tile: the backward's walk length, then its tile order


def _target_ptr(target) -> tuple:
    t = np.ascontiguousarray(np.asarray(target, dtype=np.uint8).ravel())
    return t, t.ctypes.data_as(_P), t.nbytes


def _fptr(a: np.ndarray):
    return a.ctypes.data_as(_FP)


class Trainer:
    """Trains Gaussians on one B200: the reference's splat::Trainer, method for method."""

    def __init__(self, initial: GaussianCloud, options: TrainerOptions | None = None):
        initial.validate()
        if initial.size() == 0:
            raise RuntimeError("nothing to train: the cloud is empty")
        self.options = options or TrainerOptions()
        c, self._keep = initial._c()
        handle = _P()
        _check(_lib.splat_trainer_create(ctypes.byref(c), ctypes.byref(self.options._c()), ctypes.byref(handle)))
        self._h = handle
        self._count = initial.size()
        self._degree = initial.sh_degree
        self._prefetch_keep = None

    @classmethod
    def _borrowed(cls, handle) -> "Trainer":
        """A view of a trainer another object owns (a session's)."""
        t = cls.__new__(cls)
        t.options = None
        t._keep = None
        t._h = handle
        t._owner = False
        n, degree = ctypes.c_int64(), ctypes.c_int32()
        _check(_lib.splat_trainer_info(handle, ctypes.byref(n), ctypes.byref(degree), None, None, None, None))
        t._count, t._degree = n.value, degree.value
        t._prefetch_keep = None
        return t

    def close(self) -> None:
        if getattr(self, "_h", None) and getattr(self, "_owner", True):
            _check(_lib.splat_trainer_destroy(self._h))
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- the step

    def render(self, camera: Camera) -> np.ndarray:
        """width * height * 4 floats: rgb and the log transmittance."""
        out = np.empty(camera.width * camera.height * 4, np.float32)
        _check(_lib.splat_trainer_render(self._h, ctypes.byref(camera._c()), _fptr(out)))
        return out

    def compute_gradients(self, camera: Camera, target) -> StepStats:
        t, p, n = _target_ptr(target)
        s = _Stats()
        _check(_lib.splat_trainer_compute_gradients(self._h, ctypes.byref(camera._c()), p, n, ctypes.byref(s)))
        return StepStats._from(s)

    def collect_statistics(self, camera: Camera, target) -> StepStats:
        t, p, n = _target_ptr(target)
        s = _Stats()
        _check(_lib.splat_trainer_collect_statistics(self._h, ctypes.byref(camera._c()), p, n, ctypes.byref(s)))
        return StepStats._from(s)

    def score_view(self, camera: Camera, target, error_share: float, pixel_weight: float = 1.0) -> StepStats:
        """Trainer::score_view: a statistics pass that marks the pixels whose mean
        error is at least error_share of the view's worst and adds, per Gaussian,
        the marked pixels it reaches, that count times the loss and its edge
        score to the densification statistics (in pixels times pixel_weight)."""
        t, p, n = _target_ptr(target)
        s = _Stats()
        _check(_lib.splat_trainer_score_view(self._h, ctypes.byref(camera._c()), p, n, float(error_share),
                                             float(pixel_weight), ctypes.byref(s)))
        return StepStats._from(s)

    def apply_gradients(self, rates: LearningRates) -> None:
        _check(_lib.splat_trainer_apply_gradients(self._h, ctypes.byref(rates._c())))

    def step(self, camera: Camera, target, rates: LearningRates, next_target=None) -> StepStats:
        t, p, n = _target_ptr(target)
        s = _Stats()
        if next_target is not None:
            nt, np_, nn = _target_ptr(next_target)
            self._prefetch_keep = nt
        else:
            np_, nn = None, 0
        _check(_lib.splat_trainer_step(self._h, ctypes.byref(camera._c()), p, n, ctypes.byref(rates._c()), np_, nn,
                                       ctypes.byref(s)))
        return StepStats._from(s)

    def step_device_target(self, camera: Camera, device_target_ptr: int, rates: LearningRates) -> StepStats:
        """Trainer::step with the target already in device memory (a device address
        of width * height * 4 bytes)."""
        s = _Stats()
        _check(_lib.splat_trainer_step_device_target(self._h, ctypes.byref(camera._c()), _P(device_target_ptr),
                                                     camera.width * camera.height * 4, ctypes.byref(rates._c()),
                                                     ctypes.byref(s)))
        return StepStats._from(s)

    def autotune(self, camera: Camera, target, repeats: int = 3) -> dict:
        """Times each tile-sort form and radix digit width, then each forward and
        backward pixel layout, then (two-pixel float layouts) each tile edge,
        batch depth and launch form, on this view with gradient passes (no
        parameter changes) and keeps the fastest."""
        t, p, n = _target_ptr(target)
        r = _Autotune()
        _check(_lib.splat_trainer_autotune(self._h, ctypes.byref(camera._c()), p, n, int(repeats), ctypes.byref(r)))
        return {"sort_form": r.sort_form, "digit_bits": r.digit_bits,
                "forward_pixels_per_thread": r.forward_pixels_per_thread,
                "backward_pixels_per_thread": r.backward_pixels_per_thread,
                "ms": {f"form{f}/digits{d + 6}": r.ms[f][d] for f in range(2) for d in range(3)},
                "layout_ms": {f"fwd{f + 1}/bwd{b + 1}": r.layout_ms[f][b] for f in range(2) for b in range(2)},
                "tile_size": r.tile_size, "batch_depth": r.batch_depth, "persistent_raster": r.persistent_raster,
                "tile_ms": {f"tile{16 * (t + 1)}/batch{128 * (b + 1)}/persistent{q}": r.tile_ms[t][b][q]
                            for t in range(2) for b in range(2) for q in range(2) if r.tile_ms[t][b][q] > 0},
                "grouped_backward": r.grouped_backward,
                "grouped_ms": {f"tile{16 * (t + 1)}/batch{128 * (b + 1)}/persistent{q}": r.grouped_ms[t][b][q]
                               for t in range(2) for b in range(2) for q in range(2) if r.grouped_ms[t][b][q] > 0}}

    def stream(self) -> int:
        """The cudaStream_t the trainer runs on, as an integer handle."""
        out = _P()
        _check(_lib.splat_trainer_stream(self._h, ctypes.byref(out)))
        return out.value or 0

    def collect_statistics_device_target(self, camera: Camera, device_target_ptr: int) -> StepStats:
        """collect_statistics with the target already in device memory."""
        s = _Stats()
        _check(_lib.splat_trainer_collect_statistics_device_target(self._h, ctypes.byref(camera._c()), _P(device_target_ptr),
                                                                   camera.width * camera.height * 4, ctypes.byref(s)))
        return StepStats._from(s)

    def score_view_device_target(self, camera: Camera, device_target_ptr: int, error_share: float,
                                 pixel_weight: float = 1.0) -> StepStats:
        """score_view with the target already in device memory."""
        s = _Stats()
        _check(_lib.splat_trainer_score_view_device_target(self._h, ctypes.byref(camera._c()), _P(device_target_ptr),
                                                           camera.width * camera.height * 4, float(error_share),
                                                           float(pixel_weight), ctypes.byref(s)))
        return StepStats._from(s)

    def step_batch_device_targets(self, cameras: list, device_target_ptrs: list, rates: LearningRates) -> list:
        """step_batch with the targets already in device memory (device addresses)."""
        k = len(cameras)
        cams = (_Camera * k)(*[c._c() for c in cameras])
        ptrs = (_P * k)(*[_P(int(a)) for a in device_target_ptrs])
        stats = (_Stats * k)()
        _check(_lib.splat_trainer_step_batch_device_targets(self._h, cams, ptrs, k, ctypes.byref(rates._c()), stats))
        return [StepStats._from(x) for x in stats]

    def step_batch(self, cameras: list, targets: list, rates: LearningRates) -> list:
        """Several views in one step (new in this library): one Adam step from
        the summed gradients. Needs sort_form SORT_TILE_DEPTH_64."""
        k = len(cameras)
        cams = (_Camera * k)(*[c._c() for c in cameras])
        kept = [np.ascontiguousarray(np.asarray(t, np.uint8).ravel()) for t in targets]
        ptrs = (_P * k)(*[a.ctypes.data_as(_P) for a in kept])
        stats = (_Stats * k)()
        _check(_lib.splat_trainer_step_batch(self._h, cams, ptrs, k, ctypes.byref(rates._c()), stats))
        return [StepStats._from(s) for s in stats]

    def prefetch_target(self, target) -> None:
        t, p, n = _target_ptr(target)
        self._prefetch_keep = t
        _check(_lib.splat_trainer_prefetch_target(self._h, p, n))

    # -- state

    def gradients(self) -> Gradients:
        n, f = self._count, 3 * (self._degree + 1) ** 2
        g = Gradients(*(np.empty(k, np.float32) for k in (n * 3, n * 3, n * 4, n, n * f)))
        _check(_lib.splat_trainer_get_gradients(self._h, _fptr(g.positions), _fptr(g.scales), _fptr(g.rotations),
                                                _fptr(g.opacities), _fptr(g.sh)))
        return g

    def cloud(self) -> GaussianCloud:
        n, f = self._count, 3 * (self._degree + 1) ** 2
        c = GaussianCloud(self._degree, *(np.empty(k, np.float32) for k in (n * 3, n * 3, n * 4, n, n * f)))
        _check(_lib.splat_trainer_get_cloud(self._h, _fptr(c.positions), _fptr(c.scales), _fptr(c.rotations),
                                            _fptr(c.opacities), _fptr(c.sh)))
        return c

    def set_active_sh_degree(self, degree: int) -> None:
        _check(_lib.splat_trainer_set_active_sh_degree(self._h, int(degree)))

    def densify_stats(self) -> DensifyStats:
        raw = np.empty(self._count * 8, np.float32)
        _check(_lib.splat_trainer_get_densify_stats(self._h, _fptr(raw)))
        r = raw.reshape(-1, 8)
        return DensifyStats(*(r[:, k].copy() for k in range(8)))

    def densify_stats_raw(self) -> np.ndarray:
        """The statistics as stored: 8 floats per Gaussian (trainer.cpp:686-708)."""
        raw = np.empty(self._count * 8, np.float32)
        _check(_lib.splat_trainer_get_densify_stats(self._h, _fptr(raw)))
        return raw.reshape(-1, 8)

    def set_densify_stats(self, raw) -> None:
        """Replaces the statistics: 8 floats per Gaussian, the layout densify_stats reads."""
        r = np.ascontiguousarray(np.asarray(raw, np.float32).ravel())
        if r.size != self._count * 8:
            raise ValueError("8 statistics per Gaussian expected")
        _check(_lib.splat_trainer_set_densify_stats(self._h, _fptr(r)))

    def reset_densify_stats(self) -> None:
        _check(_lib.splat_trainer_reset_densify_stats(self._h))

    def _prune(self, fn, share: float) -> int:
        removed = ctypes.c_uint64()
        _check(fn(self._h, float(share), ctypes.byref(removed)))
        self._count -= removed.value
        return removed.value

    def densify(self, options: DensifyOptions, rng: Rng) -> DensifyResult:
        """Trainer::densify (trainer.cpp:710-715): clone, split, prune and seed
        by the densification statistics, on the GPU."""
        capacity = 2 * self._count + int(options.explore_seeds)
        source = np.empty(capacity, np.int64)
        r = _DensifyResult()
        _check(_lib.splat_trainer_densify(self._h, ctypes.byref(options._c()), rng._h, ctypes.byref(r),
                                          source.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), capacity))
        self._count = r.count
        return DensifyResult(r.count, r.cloned, r.split, r.seeded, r.pruned, r.held_back, source[:r.count].copy())

    def relocate(self, options: RelocateOptions, rng: Rng) -> DensifyResult:
        """Trainer::relocate (trainer.cpp:717-722): 3DGS-MCMC relocation of the
        dead onto live Gaussians, then growth."""
        capacity = self._count + int(max(0.0, options.growth) * self._count) + 1
        source = np.empty(capacity, np.int64)
        r = _DensifyResult()
        _check(_lib.splat_trainer_relocate(self._h, ctypes.byref(options._c()), rng._h, ctypes.byref(r),
                                           source.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), capacity))
        self._count = r.count
        return DensifyResult(r.count, r.cloned, r.split, r.seeded, r.pruned, r.held_back, source[:r.count].copy())

    def remove_largest_gaussians(self, share: float) -> int:
        """Trainer::remove_largest_gaussians: the largest first (GPU)."""
        return self._prune(_lib.splat_trainer_remove_largest, share)

    def remove_least_contributing_gaussians(self, share: float) -> int:
        """Trainer::remove_least_contributing_gaussians: by the collected contribution (GPU)."""
        return self._prune(_lib.splat_trainer_remove_least_contributing, share)

    def remove_least_opaque_gaussians(self, share: float) -> int:
        """Trainer::remove_least_opaque_gaussians: the least opaque first (GPU)."""
        return self._prune(_lib.splat_trainer_remove_least_opaque, share)

    def set_exposure(self, exposure) -> None:
        e = np.ascontiguousarray(np.asarray(exposure, np.float32).ravel())
        _check(_lib.splat_trainer_set_exposure(self._h, _fptr(e)))

    def set_sh_dropout(self, probability: float, retained_degree: int = 0, seed: int = 0) -> None:
        _check(_lib.splat_trainer_set_sh_dropout(self._h, float(probability), int(retained_degree), int(seed)))

    def set_filter3d(self, filter_values) -> None:
        f = np.ascontiguousarray(np.asarray(filter_values, np.float32).ravel())
        _check(_lib.splat_trainer_set_filter3d(self._h, _fptr(f) if f.size else None, f.size))

    def add_position_noise(self, scaler: float, iteration: int = 0) -> None:
        _check(_lib.splat_trainer_add_position_noise(self._h, float(scaler), int(iteration)))

    def enable_second_order(self) -> None:
        _check(_lib.splat_trainer_enable_second_order(self._h))

    def update_curvature(self) -> None:
        _check(_lib.splat_trainer_update_curvature(self._h))

    def reset_opacity(self, maximum: float) -> None:
        _check(_lib.splat_trainer_reset_opacity(self._h, float(maximum)))

    def apply_changes(self, cloud: GaussianCloud, source) -> None:
        """Replaces the Gaussians; source[i] is the old index whose optimiser
        state Gaussian i keeps, -1 for new ones (Trainer::apply_changes)."""
        cloud.validate()
        c, keep = cloud._c()
        src = np.ascontiguousarray(np.asarray(source, np.int32))
        _check(_lib.splat_trainer_apply_changes(self._h, ctypes.byref(c), src.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))))
        self._count = cloud.size()

    def _info(self):
        g, d, a, f = ctypes.c_int64(), ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
        gb, bpg = ctypes.c_uint64(), ctypes.c_uint64()
        _check(_lib.splat_trainer_info(self._h, ctypes.byref(g), ctypes.byref(d), ctypes.byref(a), ctypes.byref(f),
                                       ctypes.byref(gb), ctypes.byref(bpg)))
        return g.value, d.value, a.value, bool(f.value), gb.value, bpg.value

    def gaussian_count(self) -> int:
        return self._info()[0]

    def sh_degree(self) -> int:
        return self._info()[1]

    def active_sh_degree(self) -> int:
        return self._info()[2]

    def uses_fixed_point(self) -> bool:
        return self._info()[3]

    def gpu_bytes(self) -> int:
        return self._info()[4]

    def bytes_per_gaussian(self) -> int:
        return self._info()[5]

    def set_timing(self, enabled: bool) -> None:
        _check(_lib.splat_trainer_set_timing(self._h, int(enabled)))

    def timings(self) -> list:
        names = (ctypes.c_char_p * 16)()
        ms = (ctypes.c_double * 16)()
        count = ctypes.c_int32()
        _check(_lib.splat_trainer_timings(self._h, names, ms, 16, ctypes.byref(count)))
        return [(names[i].decode(), ms[i]) for i in range(count.value)]

    def device_parameters(self, group: int) -> tuple:
        addr, size = ctypes.c_uint64(), ctypes.c_uint64()
        _check(_lib.splat_trainer_device_parameters(self._h, group, ctypes.byref(addr), ctypes.byref(size)))
        return addr.value, size.value

    def debug_download(self, which: int, dtype=np.uint8) -> np.ndarray:
        size = ctypes.c_size_t()
        _check(_lib.splat_trainer_debug_download(self._h, which, None, 0, ctypes.byref(size)))
        out = np.empty(size.value, np.uint8)
        if size.value:
            _check(_lib.splat_trainer_debug_download(self._h, which, out.ctypes.data_as(_P), size.value, ctypes.byref(size)))
        return out.view(dtype)


# ----------------------------------------------------------------- stage entry points


def radix_sort_device(keys_ptr: int, values_ptr: int, tmp_keys_ptr: int, tmp_values_ptr: int, count: int,
                      key_bits: int, key_bytes: int = 4, digit_bits: int = 8, stream: int = 0) -> None:
    """RadixSorter::record on device pointers (u32 or u64 keys, u32 values)."""
    fn = _lib.splat_radix_sort_u64 if key_bytes == 8 else _lib.splat_radix_sort_u32
    _check(fn(_P(keys_ptr), _P(values_ptr), _P(tmp_keys_ptr), _P(tmp_values_ptr), count, key_bits, digit_bits,
              _P(stream) if stream else None))


def detmath_device(in_ptr: int, exp_ptr: int, log_ptr: int, count: int) -> None:
    _check(_lib.splat_debug_detmath(_P(in_ptr), _P(exp_ptr), _P(log_ptr), count))


def load_ply(path) -> GaussianCloud:
    """load_ply: a 3DGS .ply (binary little-endian or ASCII) as a GaussianCloud."""
    name = str(path).encode()
    count, degree = ctypes.c_int32(), ctypes.c_int32()
    _check(_lib.splat_cloud_load_ply(name, ctypes.byref(count), ctypes.byref(degree), None, None, None, None, None))
    n, d = count.value, degree.value
    arrays = [np.empty(n * k, np.float32) for k in (3, 3, 4, 1, 3 * (d + 1) ** 2)]
    _check(_lib.splat_cloud_load_ply(name, ctypes.byref(count), ctypes.byref(degree), *[_fptr(a) for a in arrays]))
    return GaussianCloud(d, *arrays)


def save_ply(cloud: GaussianCloud, path) -> None:
    """save_ply: the standard binary little-endian 3DGS layout."""
    c, keep = cloud._c()
    _check(_lib.splat_cloud_save_ply(str(path).encode(), ctypes.byref(c)))


CGC_BALANCED, CGC_SMALL = 0, 1


def save_cgc(cloud: GaussianCloud, path, preset: int = CGC_BALANCED, fast: bool = False) -> dict:
    """save_cgc (src/splat/cgc.hpp:41-43): the layered, LZMA-compressed format;
    needs a CUDA device. Returns the file's size and the splats per layer."""
    c, keep = cloud._c()
    stats = _CgcStats()
    _check(_lib.splat_cloud_save_cgc(str(path).encode(), ctypes.byref(c), ctypes.byref(_CgcOptions(preset, int(fast))),
                                     ctypes.byref(stats)))
    return {"bytes": int(stats.bytes), "layer_counts": [int(v) for v in stats.layer_counts]}


def load_cgc(path) -> GaussianCloud:
    """load_cgc (src/splat/cgc.hpp:45-49): a CGC file of version 1 or 2 (host only)."""
    name = str(path).encode()
    count, degree = ctypes.c_int32(), ctypes.c_int32()
    _check(_lib.splat_cloud_load_cgc(name, ctypes.byref(count), ctypes.byref(degree), None, None, None, None, None))
    n, d = count.value, degree.value
    arrays = [np.empty(n * k, np.float32) for k in (3, 3, 4, 1, 3 * (d + 1) ** 2)]
    _check(_lib.splat_cloud_load_cgc(name, ctypes.byref(count), ctypes.byref(degree), *[_fptr(a) for a in arrays]))
    return GaussianCloud(d, *arrays)


def cgc_morton_code(x: int, y: int, z: int) -> int:
    """cgc_detail::morton_code: the low 21 bits of x, y, z interleaved."""
    return int(_lib.splat_cgc_morton_code(x, y, z))


def cgc_canonicalize_axes(log_scales, wxyz):
    """cgc_detail::canonicalize_axes: (scales descending, quaternion with w largest and not negative)."""
    s = np.array(log_scales, np.float32)
    q = np.array(wxyz, np.float32)
    _check(_lib.splat_cgc_canonicalize_axes(_fptr(s), _fptr(q)))
    return s, q


def lzma_compress(data: bytes, level: int = 9, extreme: bool = True, lc: int = 3, lp: int = 0, pb: int = 2) -> bytes:
    """lzma_compress (src/splat/lzma.hpp:13): an .lzma ("alone") stream."""
    buf = ctypes.create_string_buffer(bytes(data), max(len(data), 1))
    size = ctypes.c_size_t()
    _check(_lib.splat_lzma_compress(buf, len(data), level, int(extreme), lc, lp, pb, None, 0, ctypes.byref(size)))
    out = ctypes.create_string_buffer(max(size.value, 1))
    _check(_lib.splat_lzma_compress(buf, len(data), level, int(extreme), lc, lp, pb, out, size.value, ctypes.byref(size)))
    return out.raw[: size.value]


def lzma_decompress(stream: bytes, expected: int) -> bytes:
    """lzma_decompress (src/splat/lzma.hpp:17): raises SplatError on corrupt,
    truncated or wrongly sized data."""
    src = ctypes.create_string_buffer(bytes(stream), max(len(stream), 1))
    out = ctypes.create_string_buffer(max(expected, 1))
    _check(_lib.splat_lzma_decompress(src, len(stream), out, expected))
    return out.raw[:expected]


def measure_sm_peaks() -> dict:
    """splat_measure_sm_peaks: FP32 FLOP/s, SFU ex2 results/s, shared-memory
    bytes/s and warp instructions issued per second, measured on the current GPU."""
    r = _SmPeaks()
    _check(_lib.splat_measure_sm_peaks(ctypes.byref(r)))
    return {"fp32_flops": r.fp32_flops, "sfu_ops": r.sfu_ops, "shared_bytes": r.shared_bytes,
            "warp_instructions": r.warp_instructions}


def library():
    """The loaded ctypes library, for callers that bind more entry points."""
    return _lib


# ----------------------------------------------------------------- session


@dataclass
class SessionOptions:
    """TrainOptions' training schedule (train.hpp:25-112) as the session takes it."""

    iterations: int = 15000
    sh_degree: int = 2
    seed: int = 1
    report_every: int = 500
    densify: bool = True
    densify_mode: int = 0  # 0 clone/split/prune, 1 relocation
    full_adam: bool = False
    full_resolution: bool = False
    adaptive_schedule: bool = False
    gradient_threshold: float = 2e-4
    split_threshold: float = 1.2e-3
    dense_fraction: float = 0.001
    densify_interval: int = 100
    score_views: int = 10
    score_min_pixels: float = 5.0
    explore: int = 0
    significance_prune: bool = False
    edge_split: bool = False
    threshold_rise: float = 1.0
    prune_share: float = 0.0
    recovery_prune: float = 0.0
    max_growth: float = -1.0
    max_gaussians: int = 0
    coarse_until: tuple = (0.35, 0.15)
    views_per_step: int = 1

    def _c(self) -> _SessionOptions:
        o = _SessionOptions()
        for name, _ in _SessionOptions._fields_:
            value = getattr(self, name)
            if name == "coarse_until":
                o.coarse_until[0], o.coarse_until[1] = float(value[0]), float(value[1])
            else:
                setattr(o, name, int(value) if isinstance(value, bool) else value)
        return o


class Session:
    """TrainSession (train.hpp:193-270): the schedule around a trainer, one
    iteration per step(), with the views resident on the device at three sizes."""

    def __init__(self, points, colors, cameras, images, extent: float, typical_depth: float,
                 options: SessionOptions | None = None, trainer_options: TrainerOptions | None = None):
        self.options = options or SessionOptions()
        self._points = np.ascontiguousarray(np.asarray(points, np.float64).reshape(-1, 3))
        self._colors = np.ascontiguousarray(np.asarray(colors, np.uint8).reshape(-1, 3))
        if self._points.shape[0] != self._colors.shape[0]:
            raise ValueError("one colour per point")
        cams = (_Camera * len(cameras))(*[c._c() for c in cameras])
        self._images = [np.ascontiguousarray(np.asarray(im, np.uint8).ravel()) for im in images]
        ptrs = (_P * len(self._images))(*[im.ctypes.data_as(_P) for im in self._images])
        data = _SessionData(self._points.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                            self._colors.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), self._points.shape[0], cams, ptrs,
                            len(cameras), float(extent), float(typical_depth))
        handle = _P()
        topt = (trainer_options or TrainerOptions())._c()
        _check(_lib.splat_session_create(ctypes.byref(data), ctypes.byref(self.options._c()), ctypes.byref(topt),
                                         ctypes.byref(handle)))
        self._h = handle
        self._images = None

    def step(self) -> StepStats:
        s = _Stats()
        _check(_lib.splat_session_step(self._h, ctypes.byref(s)))
        return StepStats._from(s)

    def finished(self) -> bool:
        return self.state().iteration >= self.options.iterations

    def state(self) -> _SessionState:
        st = _SessionState()
        _check(_lib.splat_session_get_state(self._h, ctypes.byref(st)))
        return st

    def trainer(self) -> Trainer:
        """The session's trainer, borrowed: valid while the session lives."""
        h = _P()
        _check(_lib.splat_session_trainer(self._h, ctypes.byref(h)))
        return Trainer._borrowed(h)

    def close(self) -> None:
        if getattr(self, "_h", None):
            _lib.splat_session_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()


def frequency_energy(rgba, width: int, height: int, factors=(1, 2, 4)) -> np.ndarray:
    """frequency_energy (schedule.cpp:41-75), on the GPU."""
    image = np.ascontiguousarray(np.asarray(rgba, np.uint8).ravel())
    f = (ctypes.c_int32 * len(factors))(*factors)
    out = np.zeros(len(factors), np.float64)
    _check(_lib.splat_frequency_energy(image.ctypes.data_as(_P), width, height, f, len(factors),
                                       out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
    return out


def resolution_switches(full: float, half: float, quarter: float) -> tuple:
    """resolution_switches (schedule.cpp:77-82): until half size ends, until quarter size ends."""
    out = (ctypes.c_double * 2)()
    _check(_lib.splat_resolution_switches(full, half, quarter, out))
    return out[0], out[1]


def growth_limit(initial: float, factor: float, observed, image_factor: float, progress: float) -> tuple:
    """GrowthBudget (schedule.hpp:26-41) after `observed` rounds: (limit, final count)."""
    obs = (ctypes.c_uint64 * max(len(observed), 1))(*observed)
    limit, final = ctypes.c_uint64(), ctypes.c_double()
    _check(_lib.splat_growth_limit(initial, factor, obs, len(observed), image_factor, progress, ctypes.byref(limit),
                                   ctypes.byref(final)))
    return limit.value, final.value


def half_size(rgba, width: int, height: int) -> np.ndarray:
    """half_size (train.cpp:232-255), on the GPU."""
    image = np.ascontiguousarray(np.asarray(rgba, np.uint8).ravel())
    out = np.zeros((height // 2) * (width // 2) * 4, np.uint8)
    _check(_lib.splat_half_size(image.ctypes.data_as(_P), width, height, out.ctypes.data_as(_P)))
    return out


def initial_cloud(points, colors, sh_degree: int) -> GaussianCloud:
    """initial_cloud (train.cpp:194-212), the neighbour search on the GPU."""
    p = np.ascontiguousarray(np.asarray(points, np.float64).reshape(-1, 3))
    c = np.ascontiguousarray(np.asarray(colors, np.uint8).reshape(-1, 3))
    n, f = p.shape[0], 3 * (sh_degree + 1) ** 2
    out = GaussianCloud(sh_degree, *(np.empty(k, np.float32) for k in (n * 3, n * 3, n * 4, n, n * f)))
    _check(_lib.splat_initial_cloud(p.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), c.ctypes.data_as(_P), n, sh_degree,
                                    _fptr(out.positions), _fptr(out.scales), _fptr(out.rotations), _fptr(out.opacities),
                                    _fptr(out.sh)))
    return out
