"""The allocation-free preconditioner entry point, called through the C ABI.

nsr_precondition_noalloc exists for callers that cannot allocate device memory
where they need the preconditioner (inside another framework's CUDA graph
capture, under a latency budget that rules out cudaMalloc's device-wide
synchronisation, or in a host application that owns all device memory).  Its
scratch space is a fixed file-scope device array, so its results must match
the workspace-based nsr_precondition exactly, call after call, even though
every call reuses the same array.

This file is collected last so that a run stopping at the first failure has
already run every other test.
"""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

NSR_ERR_CAPACITY = 1005


def _grid(nz, nx):
    from nsrno_b200 import _lib
    return _lib.NsrGrid(nz, nx, 8, 10, 5e-5, 1500.0, 1000.0, 12.0, 1.1, 0.0)


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _with_workspace(lib, grid, freqs, x, shift, adjoint, stream):
    n_sys = x.shape[0]
    nbytes = lib.nsr_precondition_workspace_size(ctypes.byref(grid), n_sys)
    ws = torch.empty(nbytes, dtype=torch.uint8, device=x.device)
    y = torch.empty_like(x)
    code = lib.nsr_precondition(ctypes.byref(grid), _ptr(freqs), n_sys, shift, adjoint, _ptr(x), _ptr(y),
                                _ptr(ws), nbytes, stream)
    assert code == 0, lib.nsr_error_string(code)
    return y


def test_no_alloc_preconditioner_matches_workspace_version_twice(cuda):
    from nsrno_b200 import _lib
    lib = _lib.load()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rng = np.random.default_rng(11)
    # two calls in a row with different grids, sizes and inputs: the second
    # call must not see anything left in the shared array by the first
    cases = [((768, 1024), [4.2e6, 7.9e6], 0.15, 0), ((256, 256), [1.0e6, 1.5e6, 2.0e6], 0.3, 1)]
    for (nz, nx), freqs, shift, adjoint in cases:
        grid = _grid(nz, nx)
        f = torch.tensor(freqs, dtype=torch.float64, device=cuda)
        x = torch.as_tensor((rng.standard_normal((len(freqs), nz, nx)) +
                             1j * rng.standard_normal((len(freqs), nz, nx))).astype(np.complex64), device=cuda)
        got = torch.empty_like(x)
        torch.cuda.synchronize()
        before = torch.cuda.memory_allocated(cuda)
        code = lib.nsr_precondition_noalloc(ctypes.byref(grid), _ptr(f), x.shape[0], shift, adjoint,
                                            _ptr(x), _ptr(got), stream)
        torch.cuda.synchronize()
        assert code == 0, lib.nsr_error_string(code)
        # the call itself takes no memory from the caller's allocator
        assert torch.cuda.memory_allocated(cuda) == before
        want = _with_workspace(lib, grid, f, x, shift, adjoint, stream)
        torch.cuda.synchronize()
        err = float((got - want).abs().norm() / want.abs().norm())
        assert err < 3e-6, err


def test_no_alloc_rejects_requests_beyond_its_capacity(cuda):
    from nsrno_b200 import _lib
    lib = _lib.load()
    grid = _grid(768, 1024)
    f = torch.full((3,), 5e6, dtype=torch.float64, device=cuda)
    x = torch.zeros((3, 768, 1024), dtype=torch.complex64, device=cuda)
    y = torch.empty_like(x)
    code = lib.nsr_precondition_noalloc(ctypes.byref(grid), _ptr(f), 3, 0.15, 0, _ptr(x), _ptr(y),
                                        ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert code == NSR_ERR_CAPACITY
