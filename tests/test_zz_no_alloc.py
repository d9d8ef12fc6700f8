"""psb_dft_corr3_noalloc: dft_corr3 for callers that cannot allocate.

Such a caller (for example one whose device memory is all owned by its own
allocator, or one that must not call cudaMalloc because it synchronises the
device) hands the engine device buffers it already has; the engine's scratch
is a fixed array compiled into the library.  This test plays that caller: it
takes device buffers from torch, calls the entry point through the C ABI on
torch's current stream twice in a row with different inputs, and checks each
output against the allocating entry point psb_dft_corr3 (exact integers, so the
tolerance is zero).  This file sorts last so that a run stopping at the first
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


def test_noalloc_matches_allocating_entry_point_twice():
    import torch
    assert torch.cuda.is_available()
    lib = _lib()
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream(dev)
    rng = np.random.default_rng(5)
    shapes = [(32, 17, 9), (12, 32, 32)]
    for call, shape in enumerate(shapes):
        a = rng.integers(0, 7, shape).astype(np.int32)
        b = rng.integers(0, 3, shape).astype(np.int32)
        want = _reference(lib, a, b)
        da = torch.from_numpy(a).to(dev)
        db = torch.from_numpy(b).to(dev)
        dout = torch.full(shape, -7, dtype=torch.int32, device=dev)
        torch.cuda.synchronize()
        st = lib.psb_dft_corr3_noalloc(da.data_ptr(), db.data_ptr(), *shape, dout.data_ptr(), stream.cuda_stream)
        assert st == 0, _err(lib)
        stream.synchronize()
        got = dout.cpu().numpy()
        np.testing.assert_array_equal(got, want, err_msg=f"call {call}")


def test_noalloc_rejects_oversized_grid():
    import torch
    lib = _lib()
    dev = torch.device("cuda", 0)
    shape = (33, 4, 4)
    da = torch.zeros(shape, dtype=torch.int32, device=dev)
    st = lib.psb_dft_corr3_noalloc(da.data_ptr(), da.data_ptr(), *shape, da.data_ptr(), None)
    assert st == 5  # PSB_ERR_LIMIT
    assert "32 voxels per axis" in _err(lib)
