"""ORACLE (test infrastructure only): the FP64 CUDA restatement of the
reference's FP64 twin (oracle/fp64_oracle.cu, built into oracle/liboracle_fp64.so
by oracle/Makefile), driven from torch on the GPU.

render() follows reference_render (src/train/reference.cpp:238, prepare()
:117-185 and composite() :193-232), loss() follows reference_loss (:276-341)
and gradients() reference_gradients (:343-533, without the penalties and the
Mip and 3D filters, which no test here turns on). The splats' per-tile lists are built here with torch: every splat
is listed in the 16x16 tiles its pixel box [floor(c - r) - 1, ceil(c + r) + 1]
meets (the box the twin walks), in the twin's walk order (depth ascending,
ties by index descending: the reverse of its stable descending-depth sort).
Used as the large-size oracle for central differences (finite_differences)
where the CPU twin would take minutes per render. Only tests/ and bench.py use
this module.
"""
from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIBRARY = HERE / "liboracle_fp64.so"
_lib = None


def lib():
    global _lib
    if _lib is None:
        if not LIBRARY.exists():
            subprocess.run(["make", "-s", "-C", str(HERE), "liboracle_fp64.so"], check=True)
        _lib = ctypes.CDLL(str(LIBRARY))
        p, i, f, d = ctypes.c_void_p, ctypes.c_int, ctypes.c_float, ctypes.c_double
        _lib.fp64_record_words.restype = i
        _lib.fp64_prepare.argtypes = [i, i, p, p, p, p, p, p, p, p, i, i, f, i, p, p]
        _lib.fp64_prepare.restype = i
        _lib.fp64_composite.argtypes = [p, p, p, p, i, i, i, i, d, d, d, p, p, p, p, i, p]
        _lib.fp64_composite.restype = i
        _lib.fp64_gradients.argtypes = [i, i, p, p, p, p, p, p, p, p, i, i, p, p, p, p, i, i, d, d, d, p, p, p, p, p, p, p,
                                        p, p, p]
        _lib.fp64_gradients.restype = i
        _lib.fp64_loss.argtypes = [p, p, i, i, d, p, p, p, p]
        _lib.fp64_loss.restype = i
    return _lib


def _check(status: int, what: str) -> None:
    if status != 0:
        raise RuntimeError(f"{what} failed with CUDA error {status}")


class DeviceCloud:
    """A cloud's float32 arrays on the GPU (the reference's GaussianCloud layout)."""

    def __init__(self, cloud, device: str = "cuda"):
        import torch

        self.sh_degree = cloud.sh_degree
        self.count = int(cloud.opacities.size)
        as_t = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.float32)).to(device)
        self.positions, self.scales, self.rotations = as_t(cloud.positions), as_t(cloud.scales), as_t(cloud.rotations)
        self.opacities, self.sh = as_t(cloud.opacities), as_t(cloud.sh)

    def group(self, name: str):
        return getattr(self, name)


class Render:
    """One FP64 render: the image (rgb [P, 3], logT [P]), the stop of each pixel
    (the walk rank of its stopping splat, -1 without one) and the lists it was
    made from, which gradients() walks again."""

    def __init__(self, **kw):
        self.__dict__.update(kw)


def _camera_arrays(view):
    v16 = np.ascontiguousarray(np.asarray(view.view, np.float32).T.ravel())
    pos = np.ascontiguousarray(view.position, np.float32)
    intr = np.array([view.fx, view.fy, view.cx, view.cy], np.float32)
    return v16, pos, intr


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _records(dc: DeviceCloud, view, near: float, cull: bool):
    import torch

    L = lib()
    dev = dc.positions.device
    stream = torch.cuda.current_stream(dev).cuda_stream
    rec = torch.empty((dc.count, L.fp64_record_words()), dtype=torch.float64, device=dev)
    v16, pos, intr = _camera_arrays(view)
    _check(L.fp64_prepare(dc.count, dc.sh_degree, dc.positions.data_ptr(), dc.scales.data_ptr(), dc.rotations.data_ptr(),
                          dc.opacities.data_ptr(), dc.sh.data_ptr(), _ptr(v16), _ptr(pos), _ptr(intr), view.width,
                          view.height, near, int(cull), rec.data_ptr(), stream), "fp64_prepare")
    return rec


def render_full(dc: DeviceCloud, view, background=(0.0, 0.0, 0.0), near: float = 0.01, record: bool = False) -> Render:
    """reference_render in FP64 on the GPU, keeping its lists; with record, also
    which (entry, pixel) pairs were blended (for frozen_render)."""
    import torch

    L = lib()
    dev = dc.positions.device
    stream = torch.cuda.current_stream(dev).cuda_stream
    rec = _records(dc, view, near, True)
    W, H = int(view.width), int(view.height)
    gw, gh = (W + 15) // 16, (H + 15) // 16
    valid = rec[:, 11] != 0
    idx = torch.nonzero(valid).squeeze(1)
    # Walk order: depth ascending, ties by index descending.
    idx_desc = torch.flip(idx, dims=[0])
    walk = idx_desc[torch.sort(rec[idx_desc, 3], stable=True).indices]
    rank = torch.full((dc.count,), -1, dtype=torch.int64, device=dev)
    rank[walk] = torch.arange(walk.numel(), device=dev)
    cx, cy, r = rec[idx, 0], rec[idx, 1], rec[idx, 2]
    x0 = torch.clamp(torch.floor(cx - r).to(torch.int64) - 1, min=0)
    x1 = torch.clamp(torch.ceil(cx + r).to(torch.int64) + 1, max=W - 1)
    y0 = torch.clamp(torch.floor(cy - r).to(torch.int64) - 1, min=0)
    y1 = torch.clamp(torch.ceil(cy + r).to(torch.int64) + 1, max=H - 1)
    keep = (x0 <= x1) & (y0 <= y1)
    idx, x0, x1, y0, y1 = idx[keep], x0[keep], x1[keep], y0[keep], y1[keep]
    tx0, tx1, ty0, ty1 = x0 // 16, x1 // 16, y0 // 16, y1 // 16
    tw = tx1 - tx0 + 1
    counts = tw * (ty1 - ty0 + 1)
    total = int(counts.sum().item()) if counts.numel() else 0
    if total:
        owner = torch.repeat_interleave(torch.arange(idx.numel(), device=dev), counts)
        first = torch.cumsum(counts, 0) - counts
        local = torch.arange(total, device=dev) - first[owner]
        tx = tx0[owner] + local % tw[owner]
        ty = ty0[owner] + local // tw[owner]
        tile = ty * gw + tx
        splat = idx[owner]
        order = torch.sort(tile * (1 << 32) + rank[splat]).indices
        entries = splat[order].contiguous()
        per_tile = torch.bincount(tile, minlength=gw * gh)
    else:
        entries = torch.zeros(1, dtype=torch.int64, device=dev)
        per_tile = torch.zeros(gw * gh, dtype=torch.int64, device=dev)
    tile_start = torch.zeros(gw * gh + 1, dtype=torch.int64, device=dev)
    tile_start[1:] = torch.cumsum(per_tile, 0)
    rgb = torch.empty((W * H, 3), dtype=torch.float64, device=dev)
    logT = torch.empty(W * H, dtype=torch.float64, device=dev)
    stop = torch.empty(W * H, dtype=torch.int64, device=dev)
    bits = torch.zeros(max(total, 1) * 8, dtype=torch.int32, device=dev) if record else None
    _check(L.fp64_composite(rec.data_ptr(), entries.data_ptr(), tile_start.data_ptr(), rank.data_ptr(), gw, gh, W, H,
                            float(background[0]), float(background[1]), float(background[2]), rgb.data_ptr(),
                            logT.data_ptr(), stop.data_ptr(), bits.data_ptr() if record else None, 1 if record else 0,
                            stream), "fp64_composite")
    return Render(rec=rec, entries=entries, tile_start=tile_start, rank=rank, rgb=rgb, logT=logT, stop=stop, grid=(gw, gh),
                  background=tuple(float(b) for b in background), entry_count=total, bits=bits, near=near)


def frozen_render(dc: DeviceCloud, view, base: Render):
    """The render of the current parameters with the (entry, pixel) pairs the
    base render blended, in its order, held fixed: no cutoff test, no
    transmittance floor, no culling. rgb [P, 3] float64."""
    import torch

    L = lib()
    dev = dc.positions.device
    stream = torch.cuda.current_stream(dev).cuda_stream
    rec = _records(dc, view, base.near, False)
    W, H = int(view.width), int(view.height)
    gw, gh = base.grid
    rgb = torch.empty((W * H, 3), dtype=torch.float64, device=dev)
    logT = torch.empty(W * H, dtype=torch.float64, device=dev)
    stop = torch.empty(W * H, dtype=torch.int64, device=dev)
    bg = base.background
    _check(L.fp64_composite(rec.data_ptr(), base.entries.data_ptr(), base.tile_start.data_ptr(), base.rank.data_ptr(), gw, gh,
                            W, H, bg[0], bg[1], bg[2], rgb.data_ptr(), logT.data_ptr(), stop.data_ptr(), base.bits.data_ptr(),
                            2, stream), "fp64_composite")
    return rgb


def render(dc: DeviceCloud, view, background=(0.0, 0.0, 0.0), near: float = 0.01):
    """reference_render in FP64 on the GPU: (rgb [P, 3] float64, logT [P]) as torch tensors."""
    r = render_full(dc, view, background, near)
    return r.rgb, r.logT


def gradients(dc: DeviceCloud, view, rendered: Render, adjoint) -> dict:
    """reference_gradients in FP64 on the GPU for the adjoint (a [P, 3] float64
    tensor): the ParameterGradients arrays as numpy float64, keyed by group."""
    import torch

    L = lib()
    dev = dc.positions.device
    stream = torch.cuda.current_stream(dev).cuda_stream
    n = dc.count
    coeffs = (dc.sh_degree + 1) ** 2
    raw = torch.empty(n * 11, dtype=torch.float64, device=dev)
    out = {k: torch.empty(n * m, dtype=torch.float64, device=dev)
           for k, m in (("positions", 3), ("scales", 3), ("rotations", 4), ("opacities", 1), ("sh", 3 * coeffs))}
    a = adjoint.contiguous().to(dev, torch.float64)
    v16, pos, intr = _camera_arrays(view)
    gw, gh = rendered.grid
    bg = rendered.background
    _check(L.fp64_gradients(n, dc.sh_degree, dc.positions.data_ptr(), dc.scales.data_ptr(), dc.rotations.data_ptr(),
                            dc.opacities.data_ptr(), dc.sh.data_ptr(), _ptr(v16), _ptr(pos), _ptr(intr), view.width,
                            view.height, rendered.rec.data_ptr(), rendered.entries.data_ptr(), rendered.tile_start.data_ptr(),
                            rendered.rank.data_ptr(), gw, gh, bg[0], bg[1], bg[2], rendered.logT.data_ptr(),
                            rendered.stop.data_ptr(), a.data_ptr(), raw.data_ptr(), out["positions"].data_ptr(),
                            out["scales"].data_ptr(), out["rotations"].data_ptr(), out["opacities"].data_ptr(),
                            out["sh"].data_ptr(), stream), "fp64_gradients")
    return {k: v.cpu().numpy() for k, v in out.items()}


def loss(rgb, target, width: int, height: int, lam: float):
    """reference_loss in FP64 on the GPU: (loss, l1, ssim, adjoint [P, 3] float64 tensor).
    target: RGBA8 (numpy or a uint8 tensor on the GPU)."""
    import torch

    L = lib()
    dev = rgb.device
    stream = torch.cuda.current_stream(dev).cuda_stream
    t = target if isinstance(target, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(target, np.uint8)).to(dev)
    pixels = width * height
    blocks = ((width + 15) // 16) * ((height + 15) // 16)
    fields = torch.empty(pixels * 9, dtype=torch.float64, device=dev)
    adjoint = torch.empty((pixels, 3), dtype=torch.float64, device=dev)
    partials = torch.empty(2 * blocks, dtype=torch.float64, device=dev)
    _check(L.fp64_loss(rgb.data_ptr(), t.data_ptr(), width, height, float(lam), fields.data_ptr(), adjoint.data_ptr(),
                       partials.data_ptr(), stream), "fp64_loss")
    sums = partials.view(2, blocks).sum(dim=1).cpu().numpy()
    per_value = 1.0 / (3.0 * pixels)
    ssim, l1 = float(sums[0]) * per_value, float(sums[1]) * per_value
    return (1.0 - lam) * l1 + lam * (1.0 - ssim), l1, ssim, adjoint


def loss_of(dc: DeviceCloud, view, target, lam: float, background=(0.0, 0.0, 0.0), near: float = 0.01) -> float:
    rgb, _ = render(dc, view, background, near)
    return loss(rgb, target, view.width, view.height, lam)[0]


def finite_differences(dc: DeviceCloud, view, target, lam: float, picks, step: float = 1e-4, frozen: bool = True,
                       background=(0.0, 0.0, 0.0), near: float = 0.01) -> np.ndarray:
    """Central differences of the FP64 loss for each (group, flat index) in
    picks, as the reference's finite_differences (tests/test_train.cpp:66-84)
    takes them: the float parameter moved up and down by `step`, the
    difference divided by the two float values' actual difference.

    frozen (the default): the renders keep the base point's blended (splat,
    pixel) pairs and order (frozen_render). With the cutoffs live, a pair whose
    alpha crosses 1/255 under the nudge jumps the image by T/255 of a colour,
    and at thousands of Gaussians those jumps over 2 step outweigh the true
    derivative; the adjoint differentiates the render with its active pairs
    fixed, and so do these differences. frozen=False differences the live
    render, as the reference's own test does with every cutoff switched off."""
    base = render_full(dc, view, background, near, record=True) if frozen else None

    def value():
        if frozen:
            rgb = frozen_render(dc, view, base)
        else:
            rgb, _ = render(dc, view, background, near)
        return loss(rgb, target, view.width, view.height, lam)[0]

    out = np.zeros(len(picks), np.float64)
    for k, (group, index) in enumerate(picks):
        values = dc.group(group)
        original = float(values[index].item())
        up = np.float32(original + step)
        down = np.float32(original - step)
        values[index] = float(up)
        high = value()
        values[index] = float(down)
        low = value()
        values[index] = original
        out[k] = (high - low) / (float(up) - float(down))
    return out
