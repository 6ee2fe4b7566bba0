"""ssam_stencil2d_noalloc, the entry point for callers that cannot allocate
device memory (a fixed memory budget owned by an embedding runtime, or a
host that forbids allocation after start-up).  It keeps the multi-step
scratch grid in a fixed library-owned device array instead of a memory pool.

Checked through the C ABI against ssam_stencil2d on two calls in a row, with
a different input each time, so that the second call cannot pass on what the
first left in the shared array.  This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest
import torch

import oracle
import ssam_b200 as S
from ssam_cases import star_matrix

pytestmark = pytest.mark.gpu

SCRATCH_LIMIT = 16 * 1024 * 1024  # SSAM_NOALLOC_SCRATCH_BYTES in include/ssam.h


def _noalloc(lib, src, dst, coeffs, radius, shape, steps, boundary):
    h, w = src.shape
    c = (ctypes.c_double * len(coeffs))(*coeffs)
    fn = lib.ssam_stencil2d_noalloc
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64,
                   ctypes.c_int64, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                   ctypes.POINTER(ctypes.c_double), ctypes.c_int, ctypes.c_int,
                   ctypes.c_void_p]
    stream = torch.cuda.current_stream(src.device).cuda_stream
    return fn(src.data_ptr(), dst.data_ptr(), w, h, src.stride(0), S.F32, shape, radius, c,
              steps, S.BOUNDARY[boundary], stream)


@pytest.mark.parametrize("shape,radius,steps,boundary", [
    (S.BOX, 1, 9, "copy"),    # chain 4 + 4 + 1: the scratch array is used twice
    (S.STAR, 2, 5, "zero"),   # chain 2 + 2 + 1
    (S.BOX, 3, 3, "copy"),    # three single-step launches
])
def test_noalloc_matches_stencil2d_on_two_calls(cuda, shape, radius, steps, boundary):
    lib = S.lib()
    h, w = 1000, 700  # 2.8 MB of scratch, inside the 16 MiB array
    f = 2 * radius + 1
    g = np.random.Generator(np.random.PCG64(radius * 10 + steps))
    ncoef = 4 * radius + 1 if shape == S.STAR else f * f
    coeffs = list(g.random(ncoef) / ncoef)
    for call in range(2):
        src = torch.rand(h, w, device=cuda, generator=torch.Generator(cuda).manual_seed(call))
        want = S.stencil2d(src, coeffs, radius, shape, steps=steps, boundary=boundary)
        got = torch.full_like(src, float("nan"))
        st = _noalloc(lib, src, got, coeffs, radius, shape, steps, boundary)
        assert st == S.OK, lib.ssam_last_error().decode()
        torch.cuda.synchronize()
        # same kernels on the same inputs: within the FP32 tolerance of the
        # parity tests (they agree exactly in practice)
        err = (got - want).abs().max().item()
        assert err <= 1e-5 * steps, f"call {call}: max |noalloc - stencil2d| = {err}"
        # and directly against the oracle's chain of single steps
        m = star_matrix(coeffs, radius) if shape == S.STAR else np.array(coeffs).reshape(f, f)
        ref = oracle.conv2d(src.cpu().numpy(), m.astype(np.float32), boundary, steps=steps)
        err = np.abs(got.cpu().numpy() - ref).max()
        assert err <= 1e-5 * steps, f"call {call}: max |noalloc - oracle| = {err}"


def test_noalloc_rejects_grids_beyond_the_array(cuda):
    lib = S.lib()
    n = 2100  # 2100 x 2100 x 4 bytes > 16 MiB
    assert n * n * 4 > SCRATCH_LIMIT
    src = torch.rand(n, n, device=cuda)
    dst = torch.empty_like(src)
    st = _noalloc(lib, src, dst, [0.2] * 5, 1, S.STAR, 8, "zero")
    assert st == S.ERR_INVALID
    assert "at most" in lib.ssam_last_error().decode()
    # a single step needs no scratch, so any size is accepted
    assert _noalloc(lib, src, dst, [0.2] * 5, 1, S.STAR, 1, "zero") == S.OK
    torch.cuda.synchronize()
