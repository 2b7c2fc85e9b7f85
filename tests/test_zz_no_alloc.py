"""The radix sort entry point that allocates nothing (splat_radix_sort_u32_noalloc).

It exists for callers that cannot allocate device memory: an application that
owns a fixed device-memory budget, or a latency-critical loop in which
cudaMalloc/cudaFree would synchronise the device. Its scratch is a fixed
file-scope device array shared by every call, so this test checks, through the
C ABI, that two calls in a row (the second one on a different input, so a
stale histogram or look-back word from the first would show) give exactly the
pairs the allocating entry point gives, at the exact maximum count as well,
and that a count beyond its maximum is refused with a clear error. One case
runs in a child process of its own, so that the call there is the first one
in its CUDA context and its address lookup starts cold; the others run in
this process, after the other tests.
"""
from __future__ import annotations

import ctypes
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_KEYS = 1 << 22


def _bind(lib):
    fn = lib.splat_radix_sort_u32_noalloc
    fn.argtypes = [ctypes.c_void_p] * 4 + [ctypes.c_uint32, ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p]
    fn.restype = ctypes.c_int
    ref = lib.splat_radix_sort_u32
    ref.argtypes = fn.argtypes
    ref.restype = ctypes.c_int
    return fn, ref


def _sort(fn, keys: np.ndarray, key_bits: int, digit_bits: int):
    import torch

    k = torch.from_numpy(keys.view(np.int32).copy()).cuda()
    v = torch.arange(keys.size, dtype=torch.int32, device="cuda")
    tk, tv = torch.empty_like(k), torch.empty_like(v)
    torch.cuda.synchronize()
    status = fn(k.data_ptr(), v.data_ptr(), tk.data_ptr(), tv.data_ptr(), keys.size, key_bits, digit_bits, None)
    torch.cuda.synchronize()
    return status, k.cpu().numpy().view(np.uint32), v.cpu().numpy().view(np.uint32)


@pytest.mark.parametrize("digit_bits", [8, 7, 6])
def test_no_alloc_sort_matches_the_allocating_sort_twice(splat, digit_bits):
    lib = splat.library()
    fn, ref = _bind(lib)
    rng = np.random.default_rng(7 + digit_bits)
    cases = [(rng.integers(0, 1 << 32, 1_000_003, dtype=np.uint64).astype(np.uint32), 32),
             ((rng.integers(0, 1 << 32, 300_001, dtype=np.uint64) & 0x0F).astype(np.uint32), 8)]
    for keys, bits in cases:  # two calls in a row on the shared scratch
        s0, k0, v0 = _sort(fn, keys, bits, digit_bits)
        assert s0 == 0, lib.splat_last_error()
        s1, k1, v1 = _sort(ref, keys, bits, digit_bits)
        assert s1 == 0
        np.testing.assert_array_equal(k0, k1)
        np.testing.assert_array_equal(v0, v1)
        order = np.argsort(keys, kind="stable").astype(np.uint32)
        np.testing.assert_array_equal(v0, order)


def test_no_alloc_sort_refuses_counts_beyond_its_maximum(splat):
    lib = splat.library()
    fn, _ = _bind(lib)
    lib.splat_last_error.restype = ctypes.c_char_p
    status = fn(None, None, None, None, MAX_KEYS + 1, 32, 8, None)
    assert status == splat.SPLAT_ERR_INVALID
    assert b"maximum" in lib.splat_last_error()


def test_no_alloc_sort_at_its_maximum_count(splat):
    """4,194,304 keys of 32 bits with 8-bit digits: the look-back words fill
    the whole array; twice in a row, against the allocating sort and numpy."""
    lib = splat.library()
    fn, ref = _bind(lib)
    rng = np.random.default_rng(31)
    for _ in range(2):
        keys = rng.integers(0, 1 << 32, MAX_KEYS, dtype=np.uint64).astype(np.uint32)
        s0, k0, v0 = _sort(fn, keys, 32, 8)
        assert s0 == 0, lib.splat_last_error()
        s1, k1, v1 = _sort(ref, keys, 32, 8)
        assert s1 == 0
        np.testing.assert_array_equal(k0, k1)
        np.testing.assert_array_equal(v0, v1)
        np.testing.assert_array_equal(v0, np.argsort(keys, kind="stable").astype(np.uint32))


_CHILD = r"""
import ctypes, importlib, sys
import numpy as np
import torch
sys.path.insert(0, sys.argv[1])
lib = importlib.import_module("vibe-splat_b200").library()
fn = lib.splat_radix_sort_u32_noalloc
fn.argtypes = [ctypes.c_void_p] * 4 + [ctypes.c_uint32, ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p]
fn.restype = ctypes.c_int
keys = np.random.default_rng(5).integers(0, 1 << 32, 777_777, dtype=np.uint64).astype(np.uint32)
k = torch.from_numpy(keys.view(np.int32).copy()).cuda()
v = torch.arange(keys.size, dtype=torch.int32, device="cuda")
tk, tv = torch.empty_like(k), torch.empty_like(v)
torch.cuda.synchronize()
status = fn(k.data_ptr(), v.data_ptr(), tk.data_ptr(), tv.data_ptr(), keys.size, 32, 8, None)
assert status == 0, status
order = np.argsort(keys, kind="stable").astype(np.uint32)
assert np.array_equal(v.cpu().numpy().view(np.uint32), order)
assert np.array_equal(k.cpu().numpy().view(np.uint32), keys[order])
print("ok")
"""


def test_no_alloc_sort_first_call_in_a_fresh_process(splat):
    root = Path(__file__).resolve().parent.parent
    out = subprocess.run([sys.executable, "-c", _CHILD, str(root)], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.strip().endswith("ok")
