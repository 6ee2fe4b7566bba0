"""ssam_b200 -- B200-native register-cache systolic stencils and convolutions.

Python front end over the C ABI of ``libssam_b200.so`` (``include/ssam.h``).
It exists for tests, benchmarks and Python users; C/C++ callers link the
shared library directly.  torch is used only to hold device memory and to
name the CUDA stream -- every byte of compute runs in this package's own
sm_100a kernels.  There is no CPU fallback: if the library is missing or no
B200 is visible, calls raise.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libssam_b200.so")

OK, ERR_INVALID, ERR_UNSUPPORTED, ERR_CUDA, ERR_NOMEM, ERR_TIMEOUT = range(6)
F32, F64, BF16, F16 = range(4)
BOUNDARY = {"zero": 0, "clamp": 1, "copy": 2}
STAR, BOX = 0, 1

_STATUS_NAMES = {0: "SSAM_OK", 1: "SSAM_ERR_INVALID", 2: "SSAM_ERR_UNSUPPORTED",
                 3: "SSAM_ERR_CUDA", 4: "SSAM_ERR_NOMEM", 5: "SSAM_ERR_TIMEOUT"}


class SsamError(RuntimeError):
    """A non-OK status from the C ABI; ``status`` holds the code."""

    def __init__(self, status: int, msg: str):
        super().__init__(f"{_STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


_lib = None


class Grid2D(ctypes.Structure):
    """``ssam_grid2d``: one grid of a batch (device pointers)."""
    _fields_ = [("src", ctypes.c_void_p), ("dst", ctypes.c_void_p), ("width", ctypes.c_int64),
                ("height", ctypes.c_int64), ("pitch", ctypes.c_int64)]


BATCH_PERSISTENT, BATCH_PER_GRID = 0, 1


class PoissonOptions(ctypes.Structure):
    """``ssam_poisson_options``."""
    _fields_ = [("tol", ctypes.c_double), ("sweep_dtype", ctypes.c_int),
                ("sweeps_per_correction", ctypes.c_int), ("max_sweeps", ctypes.c_int),
                ("omega", ctypes.c_double), ("cnn_smoothing", ctypes.c_int)]


class PoissonStats(ctypes.Structure):
    """``ssam_poisson_stats``."""
    _fields_ = [("converged", ctypes.c_int), ("sweeps", ctypes.c_int),
                ("corrections", ctypes.c_int), ("initial_rel_residual", ctypes.c_double),
                ("rel_residual", ctypes.c_double), ("cnn_corrections", ctypes.c_int),
                ("fell_back", ctypes.c_int)]

_i64 = ctypes.c_int64
_int = ctypes.c_int
_vp = ctypes.c_void_p
_dp = ctypes.POINTER(ctypes.c_double)


def _declare(lib):
    lib.ssam_last_error.restype = ctypes.c_char_p
    lib.ssam_last_error.argtypes = []
    lib.ssam_abi_version.restype = _int
    lib.ssam_kernel_launches.restype = ctypes.c_uint64
    lib.ssam_kernel_launches.argtypes = []
    lib.ssam_stencil2d.restype = _int
    lib.ssam_stencil2d.argtypes = [_vp, _vp, _i64, _i64, _i64, _int, _int, _int, _dp,
                                   _int, _int, _vp]
    lib.ssam_stencil2d_host.restype = _int
    lib.ssam_stencil2d_host.argtypes = lib.ssam_stencil2d.argtypes
    lib.ssam_stencil3d.restype = _int
    lib.ssam_stencil3d.argtypes = [_vp, _vp, _i64, _i64, _i64, _int, _int, _int, _dp, _int,
                                   _int, _vp]
    lib.ssam_stencil3d_host.restype = _int
    lib.ssam_stencil3d_host.argtypes = lib.ssam_stencil3d.argtypes
    lib.ssam_device_status.restype = _int
    lib.ssam_device_status.argtypes = [_vp]
    lib.ssam_trim_scratch.restype = _int
    lib.ssam_debug_batched_barrier.restype = _int
    lib.ssam_debug_batched_barrier.argtypes = [ctypes.c_uint, ctypes.c_ulonglong]
    lib.ssam_stencil2d_noalloc.restype = _int
    lib.ssam_stencil2d_noalloc.argtypes = lib.ssam_stencil2d.argtypes
    lib.ssam_stencil2d_batched.restype = _int
    lib.ssam_stencil2d_batched.argtypes = [ctypes.POINTER(Grid2D), _int, _int, _int, _int, _dp,
                                           _int, _int, _int, _vp]
    lib.ssam_poisson_solve.restype = _int
    lib.ssam_poisson_solve.argtypes = [_vp, _vp, _int, _int, ctypes.POINTER(PoissonOptions),
                                       ctypes.POINTER(PoissonStats), _vp]
    lib.ssam_poisson_solve_learned.restype = _int
    lib.ssam_poisson_solve_learned.argtypes = [_vp, _vp, _int, _int,
                                               ctypes.POINTER(PoissonOptions), _vp,
                                               ctypes.POINTER(PoissonStats), _vp]
    lib.ssam_poisson_residual.restype = _int
    lib.ssam_poisson_residual.argtypes = [_vp, _vp, _int, _int, _dp, _vp]
    lib.ssam_poisson_jacobi.restype = _int
    lib.ssam_poisson_jacobi.argtypes = [_vp, _vp, _vp, _int, _int, _int, _int, _vp]
    lib.ssam_cnn_conv3d.restype = _int
    lib.ssam_cnn_conv3d.argtypes = [_vp, _vp, _vp, _vp, _int, _int, _int, ctypes.c_float, _vp]
    lib.ssam_cnn_conv3d_wgrad.restype = _int
    lib.ssam_cnn_conv3d_wgrad.argtypes = [_vp, _vp, _vp, _vp, _int, _int, _int, _vp]
    for name, args in (("ssam_cnn_create", [_int, _int, ctypes.c_ulonglong,
                                             ctypes.POINTER(ctypes.c_void_p)]),
                       ("ssam_cnn_destroy", [_vp]),
                       ("ssam_cnn_num_params", [_vp, ctypes.POINTER(ctypes.c_int64)]),
                       ("ssam_cnn_get_params", [_vp, _vp, _vp]),
                       ("ssam_cnn_set_params", [_vp, _vp]),
                       ("ssam_cnn_forward", [_vp, _vp, _vp, _int, _vp]),
                       ("ssam_cnn_gradient", [_vp, _vp, _vp, _int, _dp, _vp]),
                       ("ssam_cnn_adam_step", [_vp, ctypes.c_float, _vp]),
                       ("ssam_cnn_save", [_vp, ctypes.c_char_p]),
                       ("ssam_cnn_load", [_vp, ctypes.c_char_p])):
        getattr(lib, name).restype = _int
        getattr(lib, name).argtypes = args
    lib.ssam_autotune_stencil2d.restype = _int
    lib.ssam_autotune_stencil2d.argtypes = lib.ssam_stencil2d.argtypes + [_vp]
    for name in ("ssam_autotune_save", "ssam_autotune_load"):
        getattr(lib, name).restype = _int
        getattr(lib, name).argtypes = [ctypes.c_char_p]
    lib.ssam_autotune_clear.restype = _int
    lib.ssam_autotune_stencil3d.restype = _int
    lib.ssam_autotune_stencil3d.argtypes = [_vp, _vp, _i64, _i64, _i64, _int, _int, _int, _dp,
                                            _int, _vp, _vp]
    lib.ssam_autotune_jacobi3d.restype = _int
    lib.ssam_autotune_jacobi3d.argtypes = [_i64, _int, _int, _vp, _vp]
    lib.ssam_conv2d.restype = _int
    lib.ssam_conv2d.argtypes = [_vp, _vp, _i64, _i64, _i64, _int, _dp, _int, _int,
                                _int, _vp]


def lib():
    """The loaded ``libssam_b200.so`` (ctypes)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"{LIB_PATH} is not built; run `python -m ssam_b200.build` "
                "(there is no CPU fallback)")
        _lib = ctypes.CDLL(LIB_PATH)
        _declare(_lib)
    return _lib


def _check(status: int) -> None:
    if status != OK:
        raise SsamError(status, lib().ssam_last_error().decode())


def _dtype_code(t) -> int:
    import torch
    m = {torch.float32: F32, torch.float64: F64, torch.bfloat16: BF16, torch.float16: F16}
    if t.dtype not in m:
        raise TypeError(f"unsupported grid dtype {t.dtype}")
    return m[t.dtype]


def _doubles(vals):
    vals = [float(v) for v in vals]
    return (ctypes.c_double * len(vals))(*vals)


def _stream_ptr(t, stream):
    import torch
    if stream is None:
        stream = torch.cuda.current_stream(t.device)
    return ctypes.c_void_p(stream.cuda_stream)


def _grid2d(src, dst):
    import torch
    if not src.is_cuda:
        raise ValueError("src must be a CUDA tensor (use the *_host entry points for host buffers)")
    if src.dim() != 2 or src.stride(1) != 1:
        raise ValueError("2D grids must be row-major with unit x stride")
    if dst is None:
        dst = torch.empty_strided(src.shape, src.stride(), dtype=src.dtype, device=src.device)
    if dst.shape != src.shape or dst.stride() != src.stride() or dst.dtype != src.dtype:
        raise ValueError("dst must match src in shape, strides and dtype")
    return dst


def stencil2d(src, coeffs, radius: int, shape: int = STAR, steps: int = 1,
              boundary: str = "zero", dst=None, stream=None):
    """``steps`` steps of a square radius-``radius`` stencil (``ssam_stencil2d``).

    ``coeffs``: STAR -> [c, n1, s1, w1, e1, n2, ...]; BOX -> (2r+1)^2 row-major.
    """
    dst = _grid2d(src, dst)
    h, w = src.shape
    c = _doubles(coeffs)
    _check(lib().ssam_stencil2d(src.data_ptr(), dst.data_ptr(), w, h, src.stride(0),
                                _dtype_code(src), shape, radius, c, steps,
                                BOUNDARY[boundary], _stream_ptr(src, stream)))
    return dst


def stencil2d_host(src, dst, coeffs, radius: int, shape: int = STAR, steps: int = 1,
                   boundary: str = "zero", device=None, stream=None):
    """``ssam_stencil2d_host``: ``src``/``dst`` are CPU tensors (pinned for
    full bandwidth); copies in, steps, copies out.  Queued on ``stream``;
    synchronise before reading ``dst``."""
    import torch
    if src.is_cuda or dst.is_cuda:
        raise ValueError("stencil2d_host takes host tensors")
    if src.dim() != 2 or src.stride(1) != 1 or dst.shape != src.shape or \
            dst.stride() != src.stride() or dst.dtype != src.dtype:
        raise ValueError("src/dst must be matching row-major 2D host tensors")
    dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    if stream is None:
        stream = torch.cuda.current_stream(dev)
    h, w = src.shape
    c = _doubles(coeffs)
    with torch.cuda.device(dev):
        _check(lib().ssam_stencil2d_host(src.data_ptr(), dst.data_ptr(), w, h, src.stride(0),
                                         _dtype_code(src), shape, radius, c, steps,
                                         BOUNDARY[boundary], ctypes.c_void_p(stream.cuda_stream)))
    return dst


def conv2d(src, weight, boundary: str = "zero", dst=None, stream=None):
    """Correlation with an (fh, fw) weight matrix (``ssam_conv2d``)."""
    dst = _grid2d(src, dst)
    h, w = src.shape
    rows = [list(map(float, r)) for r in (weight.tolist() if hasattr(weight, "tolist") else weight)]
    fh, fw = len(rows), len(rows[0])
    c = _doubles([v for r in rows for v in r])
    _check(lib().ssam_conv2d(src.data_ptr(), dst.data_ptr(), w, src.stride(0), h,
                             _dtype_code(src), c, fw, fh, BOUNDARY[boundary],
                             _stream_ptr(src, stream)))
    return dst


STAR3D, POISSON19 = 0, 2


def _grid3d(src, dst):
    import torch
    if not src.is_cuda:
        raise ValueError("src must be a CUDA tensor")
    if src.dim() != 3 or not src.is_contiguous():
        raise ValueError("3D grids must be contiguous (nz, ny, nx) tensors")
    if dst is None:
        dst = torch.empty_like(src)
    if dst.shape != src.shape or dst.dtype != src.dtype or not dst.is_contiguous():
        raise ValueError("dst must match src")
    return dst


def stencil3d(src, coeffs, radius: int = 1, shape: int = STAR3D, steps: int = 1,
              boundary: str = "zero", dst=None, stream=None):
    """``steps`` steps of a 3D stencil (``ssam_stencil3d``); ``coeffs`` is the
    dense (2r+1)^3 cube indexed [dz+r][dy+r][dx+r] (any array-like)."""
    dst = _grid3d(src, dst)
    nz, ny, nx = src.shape
    flat = coeffs.ravel().tolist() if hasattr(coeffs, "ravel") else list(coeffs)
    c = _doubles(flat)
    _check(lib().ssam_stencil3d(src.data_ptr(), dst.data_ptr(), nx, ny, nz, _dtype_code(src),
                                shape, radius, c, steps, BOUNDARY[boundary],
                                _stream_ptr(src, stream)))
    return dst


def stencil3d_host(src, dst, coeffs, radius: int = 1, shape: int = STAR3D, steps: int = 1,
                   boundary: str = "zero", device=None, stream=None):
    """``ssam_stencil3d_host`` on (pinned) CPU tensors; synchronise before
    reading ``dst``."""
    import torch
    if src.is_cuda or dst.is_cuda or src.shape != dst.shape or src.dim() != 3:
        raise ValueError("stencil3d_host takes matching 3D host tensors")
    dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    if stream is None:
        stream = torch.cuda.current_stream(dev)
    nz, ny, nx = src.shape
    flat = coeffs.ravel().tolist() if hasattr(coeffs, "ravel") else list(coeffs)
    with torch.cuda.device(dev):
        _check(lib().ssam_stencil3d_host(src.data_ptr(), dst.data_ptr(), nx, ny, nz,
                                         _dtype_code(src), shape, radius, _doubles(flat),
                                         steps, BOUNDARY[boundary],
                                         ctypes.c_void_p(stream.cuda_stream)))
    return dst


def device_status(stream=None) -> None:
    """Raise SsamError(SSAM_ERR_TIMEOUT) if a bounded device wait gave up."""
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    _check(lib().ssam_device_status(ctypes.c_void_p(s.cuda_stream)))


def stencil2d_batched(srcs, coeffs, radius: int, shape: int = STAR, steps: int = 1,
                      boundary: str = "zero", dsts=None, persistent: bool = True, stream=None):
    """``ssam_stencil2d_batched`` over a list of 2D CUDA tensors of one dtype."""
    if dsts is None:
        dsts = [_grid2d(s_, None) for s_ in srcs]
    arr = (Grid2D * len(srcs))()
    for i, (a, b) in enumerate(zip(srcs, dsts)):
        _grid2d(a, b)
        arr[i] = Grid2D(a.data_ptr(), b.data_ptr(), a.shape[1], a.shape[0], a.stride(0))
    _check(lib().ssam_stencil2d_batched(arr, len(srcs), _dtype_code(srcs[0]), shape, radius,
                                        _doubles(coeffs), steps, BOUNDARY[boundary],
                                        BATCH_PERSISTENT if persistent else BATCH_PER_GRID,
                                        _stream_ptr(srcs[0], stream)))
    return dsts


def _poisson_grid(t):
    if not t.is_cuda or t.dim() != 4 or t.shape[1] != t.shape[2] or t.shape[2] != t.shape[3] \
            or not t.is_contiguous():
        raise ValueError("Poisson grids are contiguous CUDA tensors of shape (nbatch, n, n, n)")
    return t.shape[0], t.shape[1]


def poisson_solve(f, u, tol: float = 1e-5, sweep_dtype=None, sweeps_per_correction: int = 1000,
                  max_sweeps: int = 200000, cnn=None, omega: float = 1.0,
                  cnn_smoothing: int = 4, stream=None) -> dict:
    """``ssam_poisson_solve``: f, u are float64 (nbatch, n, n, n); u holds the
    initial guess and receives the solution.  With ``cnn`` (a WarmStartCNN)
    this is ``ssam_poisson_solve_learned``: the network's correction comes
    before the sweeps of every defect-correction step."""
    import torch
    nb, n = _poisson_grid(f)
    if u.shape != f.shape or f.dtype != torch.float64 or u.dtype != torch.float64:
        raise ValueError("f and u must be float64 tensors of the same shape")
    dt = F32 if sweep_dtype in (None, "f32", torch.float32) else BF16
    opt = PoissonOptions(tol, dt, sweeps_per_correction, max_sweeps, omega, cnn_smoothing)
    st = PoissonStats()
    if cnn is None:
        _check(lib().ssam_poisson_solve(f.data_ptr(), u.data_ptr(), n, nb, ctypes.byref(opt),
                                        ctypes.byref(st), _stream_ptr(f, stream)))
    else:
        _check(lib().ssam_poisson_solve_learned(f.data_ptr(), u.data_ptr(), n, nb,
                                                ctypes.byref(opt), cnn._h, ctypes.byref(st),
                                                _stream_ptr(f, stream)))
    return {k: getattr(st, k) for k, _ in st._fields_}


def poisson_residual(f, u, stream=None) -> list:
    """FP64 ||f - A u|| / ||f|| per right-hand side."""
    nb, n = _poisson_grid(f)
    rel = (ctypes.c_double * nb)()
    _check(lib().ssam_poisson_residual(f.data_ptr(), u.data_ptr(), n, nb, rel,
                                       _stream_ptr(f, stream)))
    return list(rel)


def poisson_jacobi(rhs, u_in, sweeps: int, u_out=None, stream=None):
    """``sweeps`` Jacobi sweeps in the storage type of the tensors."""
    import torch
    nb, n = _poisson_grid(rhs)
    if u_out is None:
        u_out = torch.empty_like(u_in)
    _check(lib().ssam_poisson_jacobi(rhs.data_ptr(), u_in.data_ptr(), u_out.data_ptr(), n, nb,
                                     _dtype_code(rhs), sweeps, _stream_ptr(rhs, stream)))
    return u_out


class TuneReport(ctypes.Structure):
    """``ssam_tune_report``."""
    _fields_ = [("rows_per_thread", ctypes.c_int), ("warps_per_block", ctypes.c_int),
                ("columns_per_thread", ctypes.c_int), ("fused_steps", ctypes.c_int),
                ("candidates", ctypes.c_int), ("ms_per_step", ctypes.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


def autotune_stencil2d(src, coeffs, radius: int, shape: int = STAR, steps: int = 1,
                       boundary: str = "zero", dst=None, stream=None) -> dict:
    """Measure every compiled configuration on ``src`` (``dst`` is scratch)
    and keep the fastest for this grid size class (``ssam_autotune_stencil2d``)."""
    dst = _grid2d(src, dst)
    h, w = src.shape
    rep = TuneReport()
    _check(lib().ssam_autotune_stencil2d(src.data_ptr(), dst.data_ptr(), w, h, src.stride(0),
                                         _dtype_code(src), shape, radius, _doubles(coeffs),
                                         steps, BOUNDARY[boundary], _stream_ptr(src, stream),
                                         ctypes.byref(rep)))
    return rep.as_dict()


class Tune3DReport(ctypes.Structure):
    """``ssam_tune3d_report``."""
    _fields_ = [("rows_per_warp", ctypes.c_int), ("consumer_warps", ctypes.c_int),
                ("ring_slots", ctypes.c_int), ("registers_z", ctypes.c_int),
                ("columns_per_thread", ctypes.c_int), ("candidates", ctypes.c_int),
                ("ms_per_step", ctypes.c_double), ("fused_steps", ctypes.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


def autotune_stencil3d(src, coeffs, radius: int = 1, shape: int = STAR3D,
                       boundary: str = "zero", dst=None, stream=None) -> dict:
    """Measure every compiled 3D configuration for one step on ``src``
    (``dst`` is scratch) and keep the fastest for this grid size class
    (``ssam_autotune_stencil3d``)."""
    dst = _grid3d(src, dst)
    nz, ny, nx = src.shape
    flat = coeffs.ravel().tolist() if hasattr(coeffs, "ravel") else list(coeffs)
    rep = Tune3DReport()
    _check(lib().ssam_autotune_stencil3d(src.data_ptr(), dst.data_ptr(), nx, ny, nz,
                                         _dtype_code(src), shape, radius, _doubles(flat),
                                         BOUNDARY[boundary], _stream_ptr(src, stream),
                                         ctypes.byref(rep)))
    return rep.as_dict()


def autotune_jacobi3d(n: int, nbatch: int, sweep_dtype: str = "f32", device=None,
                      stream=None) -> dict:
    """Measure the Poisson solver's Jacobi-sweep configurations for `nbatch`
    stacked n^3 grids (``ssam_autotune_jacobi3d``; scratch buffers of its
    own); later solves of that size use the fastest."""
    import torch
    dev = torch.device(device) if device is not None else torch.device(
        "cuda", torch.cuda.current_device())
    if stream is None:
        stream = torch.cuda.current_stream(dev)
    code = {"f32": F32, "bf16": BF16}[sweep_dtype]
    rep = Tune3DReport()
    with torch.cuda.device(dev):
        _check(lib().ssam_autotune_jacobi3d(n, nbatch, code, ctypes.c_void_p(stream.cuda_stream),
                                            ctypes.byref(rep)))
    return rep.as_dict()


def autotune_save(path: str) -> None:
    _check(lib().ssam_autotune_save(path.encode()))


def autotune_load(path: str) -> None:
    _check(lib().ssam_autotune_load(path.encode()))


def autotune_clear() -> None:
    _check(lib().ssam_autotune_clear())


def star_coeffs_from_matrix(m) -> list[float]:
    """Reference kernel-argument order (stencil2D_25pt.cu:10-16) from a
    (2r+1)x(2r+1) star matrix: c, then n_k, s_k, w_k, e_k for k = 1..r."""
    rows = m.tolist() if hasattr(m, "tolist") else m
    r = len(rows) // 2
    out = [rows[r][r]]
    for k in range(1, r + 1):
        out += [rows[r - k][r], rows[r + k][r], rows[r][r - k], rows[r][r + k]]
    return out


def to_planar(x):
    """Channels-last (nb, n, n, n, 16) -> the library's planar halves
    (2, nb, n, n, n, 8), contiguous."""
    return x.reshape(*x.shape[:-1], 2, 8).movedim(-2, 0).contiguous()


def from_planar(p):
    """Planar halves (2, nb, n, n, n, 8) -> channels-last (nb, n, n, n, 16)."""
    return p.movedim(0, -2).reshape(*p.shape[1:-1], 16)


def cnn_conv3d(x0, weight, x1=None, dilation: int = 1, scale: float = 1.0, stream=None):
    """3x3x3 convolution of channels-last BF16 activations (nb, n, n, n, 16)
    (x1: optional second 16-channel source) with weights (16, 27, 16 * nsrc)
    on the tensor cores (``ssam_cnn_conv3d``, which works on planar halves;
    the layouts are converted here)."""
    import torch
    nb, n = x0.shape[0], x0.shape[1]
    p0 = to_planar(x0)
    p1 = to_planar(x1) if x1 is not None else None
    out = torch.empty_like(p0)
    _check(lib().ssam_cnn_conv3d(p0.data_ptr(), p1.data_ptr() if p1 is not None else None,
                                 weight.data_ptr(), out.data_ptr(), nb, n, dilation, scale,
                                 _stream_ptr(x0, stream)))
    return from_planar(out)


def cnn_conv3d_wgrad(x0, grad_out, x1=None, dilation: int = 1, stream=None):
    """fp32 weight gradient (16, 27, 16 * nsrc) of ``cnn_conv3d``
    (``ssam_cnn_conv3d_wgrad``)."""
    import torch
    nb, n = x0.shape[0], x0.shape[1]
    nsrc = 2 if x1 is not None else 1
    dw = torch.empty(16, 27, 16 * nsrc, dtype=torch.float32, device=x0.device)
    p0, g = to_planar(x0), to_planar(grad_out)
    p1 = to_planar(x1) if x1 is not None else None
    _check(lib().ssam_cnn_conv3d_wgrad(p0.data_ptr(), p1.data_ptr() if p1 is not None else None,
                                       g.data_ptr(), dw.data_ptr(), nb, n, dilation,
                                       _stream_ptr(x0, stream)))
    return dw


class WarmStartCNN:
    """The Poisson warm-start network (``ssam_cnn_*``): a 3-level, 16-channel
    linear U-Net on the tensor cores.  f and u are float64 CUDA tensors of
    shape (nbatch, n, n, n)."""

    def __init__(self, n: int, nbatch_max: int, seed: int = 0):
        self.n, self.nbatch_max = n, nbatch_max
        h = ctypes.c_void_p()
        _check(lib().ssam_cnn_create(n, nbatch_max, seed, ctypes.byref(h)))
        self._h = h
        cnt = ctypes.c_int64()
        _check(lib().ssam_cnn_num_params(self._h, ctypes.byref(cnt)))
        self.num_params = cnt.value

    def close(self):
        if self._h:
            lib().ssam_cnn_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def forward(self, f, out=None, stream=None):
        import torch
        if out is None:
            out = torch.empty_like(f)
        _check(lib().ssam_cnn_forward(self._h, f.data_ptr(), out.data_ptr(), f.shape[0],
                                      _stream_ptr(f, stream)))
        return out

    def gradient(self, f, target, stream=None) -> float:
        loss = ctypes.c_double()
        _check(lib().ssam_cnn_gradient(self._h, f.data_ptr(), target.data_ptr(), f.shape[0],
                                       ctypes.byref(loss), _stream_ptr(f, stream)))
        return loss.value

    def adam_step(self, lr: float, stream=None):
        import torch
        s = stream if stream is not None else torch.cuda.current_stream()
        _check(lib().ssam_cnn_adam_step(self._h, lr, ctypes.c_void_p(s.cuda_stream)))

    def params(self):
        import numpy as np
        w = np.empty(self.num_params, np.float32)
        g = np.empty(self.num_params, np.float32)
        _check(lib().ssam_cnn_get_params(self._h, w.ctypes.data_as(_vp), g.ctypes.data_as(_vp)))
        return w, g

    def set_params(self, w):
        import numpy as np
        w = np.ascontiguousarray(w, np.float32)
        assert w.size == self.num_params
        _check(lib().ssam_cnn_set_params(self._h, w.ctypes.data_as(_vp)))

    def save(self, path: str):
        _check(lib().ssam_cnn_save(self._h, path.encode()))

    def load(self, path: str):
        _check(lib().ssam_cnn_load(self._h, path.encode()))
