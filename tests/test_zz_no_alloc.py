"""psb_dft_corr3_noalloc: dft_corr3 for callers that cannot allocate.

Such a caller (for example one whose device memory is all owned by its own
allocator, or one that must not call cudaMalloc because it synchronises the
device) hands the engine device buffers it already has; the engine's scratch
is a fixed array compiled into the library.  This test plays that caller: it
takes device buffers from torch, calls the entry point through the C ABI on
torch's current stream several times in a row with different inputs, and checks
each output against the allocating entry point psb_dft_corr3 and against the
oracle (exact integers, so the tolerance is zero), including the largest grid
the fixed array takes (32^3), and that the calls leave the device's free
memory unchanged.  This file sorts last so that a run stopping at the first
failure has already run every other test.
"""
import ctypes
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

LIB = Path(__file__).resolve().parent.parent / "psacking_b200" / "libpsb200.so"


def _lib():
    lib = ctypes.CDLL(str(LIB))
    lib.psb_dft_corr3_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                          ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    lib.psb_dft_corr3.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                  ctypes.c_void_p]
    lib.psb_last_error.argtypes = [ctypes.c_char_p, ctypes.c_size_t]
    return lib


def _err(lib):
    buf = ctypes.create_string_buffer(1024)
    lib.psb_last_error(buf, 1024)
    return buf.value.decode()


def _reference(lib, a, b):
    out = np.zeros_like(a)
    st = lib.psb_dft_corr3(a.ctypes.data, b.ctypes.data, *a.shape, out.ctypes.data)
    assert st == 0, _err(lib)
    return out


def _noalloc(lib, stream, a, b, dev):
    import torch
    da = torch.from_numpy(a).to(dev)
    db = torch.from_numpy(b).to(dev)
    dout = torch.full(a.shape, -7, dtype=torch.int32, device=dev)
    torch.cuda.synchronize()
    st = lib.psb_dft_corr3_noalloc(da.data_ptr(), db.data_ptr(), *a.shape, dout.data_ptr(), stream.cuda_stream)
    assert st == 0, _err(lib)
    stream.synchronize()
    return dout.cpu().numpy()


def test_noalloc_matches_allocating_entry_point_twice():
    import torch
    from oracle import psb_oracle as O
    assert torch.cuda.is_available()
    lib = _lib()
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream(dev)
    rng = np.random.default_rng(5)
    # the second shape is the largest grid the fixed array takes
    shapes = [(32, 17, 9), (32, 32, 32), (12, 32, 32)]
    for call, shape in enumerate(shapes):
        a = rng.integers(0, 7, shape).astype(np.int32)
        b = rng.integers(0, 3, shape).astype(np.int32)
        want = _reference(lib, a, b)
        got = _noalloc(lib, stream, a, b, dev)
        np.testing.assert_array_equal(got, want, err_msg=f"call {call}")
        if call != 1:   # the oracle's direct sums take a while at 32^3
            np.testing.assert_array_equal(got, O.dft_corr3(a, b), err_msg=f"call {call} vs oracle")


def test_noalloc_leaves_device_memory_unchanged():
    """Two calls in a row after a first one (which loads the kernels): the
    device's free memory is the same before and after them."""
    import torch
    lib = _lib()
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream(dev)
    shape = (20, 24, 28)
    rng = np.random.default_rng(9)
    a = torch.from_numpy(rng.integers(0, 5, shape).astype(np.int32)).to(dev)
    b = torch.from_numpy(rng.integers(0, 2, shape).astype(np.int32)).to(dev)
    out = torch.empty(shape, dtype=torch.int32, device=dev)
    outs = []
    for i in range(3):
        if i == 1:
            torch.cuda.synchronize()
            free0 = torch.cuda.mem_get_info(dev)[0]
        st = lib.psb_dft_corr3_noalloc(a.data_ptr(), b.data_ptr(), *shape, out.data_ptr(), stream.cuda_stream)
        assert st == 0, _err(lib)
        stream.synchronize()
        outs.append(out.cpu().numpy())
    free1 = torch.cuda.mem_get_info(dev)[0]
    assert free1 == free0
    want = _reference(lib, a.cpu().numpy(), b.cpu().numpy())
    for o in outs:
        np.testing.assert_array_equal(o, want)


def test_noalloc_rejects_oversized_grid():
    import torch
    lib = _lib()
    dev = torch.device("cuda", 0)
    shape = (33, 4, 4)
    da = torch.zeros(shape, dtype=torch.int32, device=dev)
    st = lib.psb_dft_corr3_noalloc(da.data_ptr(), da.data_ptr(), *shape, da.data_ptr(), None)
    assert st == 5  # PSB_ERR_LIMIT
    assert "32 voxels per axis" in _err(lib)
