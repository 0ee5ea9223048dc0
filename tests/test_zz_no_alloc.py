"""dsmc_stage_sort_static (the stage sort on the library's static scratch,
allocating nothing) against dsmc_stage_sort on the same inputs, two calls in a
row with different sizes so that state left by the first call would show in
the second, and allocating nothing on the second call (free device memory and
the default stream-ordered pool unchanged).  Collected last so that it also
runs after every other GPU test."""
import ctypes

import numpy as np
import pytest
import torch

from cudadsmc_b200 import stages
from cudadsmc_b200._capi import DsmcError

pytestmark = pytest.mark.gpu


def _u32(a, dev):
    return torch.from_numpy(a.view(np.int32)).to(dev)


def _np(t):
    return t.cpu().numpy().view(np.uint32)


def _case(seed, n, nkeys):
    rng = np.random.default_rng(seed)
    keys = rng.integers(0, nkeys, n).astype(np.uint32)
    keys[: n // 10] = nkeys - 1  # one crowded key
    vals = rng.permutation(n).astype(np.uint32)
    return keys, vals


class _DeviceMemory:
    """Free device memory (cudaMemGetInfo) and the default stream-ordered
    pool's used bytes (cudaMemPoolAttrUsedMemCurrent / High) of the current
    device, read through the CUDA runtime the library itself loads."""

    def __init__(self):
        self.rt = ctypes.CDLL("libcudart.so.12")

    def read(self):
        free, total = ctypes.c_size_t(), ctypes.c_size_t()
        assert self.rt.cudaMemGetInfo(ctypes.byref(free), ctypes.byref(total)) == 0
        dev = ctypes.c_int()
        assert self.rt.cudaGetDevice(ctypes.byref(dev)) == 0
        pool = ctypes.c_void_p()
        assert self.rt.cudaDeviceGetDefaultMemPool(ctypes.byref(pool), dev) == 0
        used, high = ctypes.c_uint64(), ctypes.c_uint64()
        assert self.rt.cudaMemPoolGetAttribute(pool, 7, ctypes.byref(used)) == 0  # UsedMemCurrent
        assert self.rt.cudaMemPoolGetAttribute(pool, 8, ctypes.byref(high)) == 0  # UsedMemHigh
        return free.value, used.value, high.value


def test_static_sort_matches_stage_sort_twice_in_a_row(cuda):
    cases = [(11, 300000, 100000), (12, 70000, 5000)]
    inputs = [(seed, nkeys) + _case(seed, n, nkeys) for seed, n, nkeys in cases]
    # every device buffer of the two calls exists before they run, and the
    # memory readings around the second call see only what it allocates
    # (the first call on a device may load the library's module, which
    # reserves the static scratch)
    dev_in = [(_u32(keys, cuda), _u32(vals, cuda),
               torch.full((nkeys + 1,), -1, dtype=torch.int32, device=cuda))
              for _, nkeys, keys, vals in inputs]
    torch.cuda.synchronize()
    mem = _DeviceMemory()
    outs = []
    before = None
    for (seed, nkeys, keys, vals), (kt, vt, st) in zip(inputs, dev_in):
        if outs:
            torch.cuda.synchronize()
            before = mem.read()
        stages.sort_static(kt, vt, nkeys, cell_start=st)
        outs.append((keys, vals, nkeys, kt, vt, st))
    torch.cuda.synchronize()
    after = mem.read()
    # the call allocated nothing: neither device memory nor pool memory
    assert after == before, (before, after)
    for keys, vals, nkeys, kt, vt, st in outs:
        kr, vr = _u32(keys, cuda), _u32(vals, cuda)
        sr = torch.zeros(nkeys + 1, dtype=torch.int32, device=cuda)
        stages.sort(kr, vr, nkeys, cell_start=sr)
        torch.cuda.synchronize()
        assert np.array_equal(_np(kt), _np(kr))
        assert np.array_equal(_np(vt), _np(vr))
        assert np.array_equal(_np(st), _np(sr))
        order = np.argsort(keys, kind="stable")
        assert np.array_equal(_np(vt), vals[order])


def test_static_sort_limits(cuda):
    keys, vals = _case(13, 1000, 100)
    kt, vt = _u32(keys, cuda), _u32(vals, cuda)
    # sizes above the static scratch are refused before any device work
    with pytest.raises(DsmcError) as e:
        stages.check(stages.lib().dsmc_stage_sort_static(
            stages._p(kt), stages._p(vt), stages.SORT_STATIC_MAX_N + 1, 100, None, None), "sort")
    assert e.value.status == 6
    with pytest.raises(DsmcError) as e:
        stages.check(stages.lib().dsmc_stage_sort_static(
            stages._p(kt), stages._p(vt), 1000, stages.SORT_STATIC_MAX_KEYS + 1, None, None), "sort")
    assert e.value.status == 6
    # the largest key range is accepted
    stages.sort_static(kt, vt, stages.SORT_STATIC_MAX_KEYS)
    torch.cuda.synchronize()
    assert np.array_equal(_np(vt), vals[np.argsort(keys, kind="stable")])
