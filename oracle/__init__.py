"""ORACLE -- test infrastructure only.

numpy front end for the two CPU checkers of the SSAM stencil path:

* ``libssam_oracle.so`` -- the plain-C restatement of the reference's CPU
  golds (``oracle/ssam_oracle.c``), always built;
* ``_ref/libssam_ref.so`` -- the reference's own golds compiled in place from
  its sources (``make -C oracle ref``).  It exists only where the reference
  tree was present at build time; :func:`have_ref` says whether it loaded.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg import this package.  The CUDA library never calls it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "libssam_oracle.so")
_REF = os.path.join(_HERE, "_ref", "libssam_ref.so")

BND = {"zero": 0, "clamp": 1, "copy": 2, "gold": 3}

_i64 = ctypes.c_int64
_vp = ctypes.c_void_p


def reference_dir() -> str:
    """The reference checkout: $SSAM_REFERENCE_DIR, else a directory named
    ``reference`` beside this repository's checkout."""
    return os.environ.get("SSAM_REFERENCE_DIR",
                          os.path.join(os.path.dirname(os.path.dirname(_HERE)), "reference"))


def build(ref: bool | None = None) -> None:
    """Compile the restatement, and the reference golds when the reference
    tree is present (``ref=None``) or when asked (``ref=True``)."""
    targets = ["all"]
    refdir = reference_dir()
    if ref or (ref is None and os.path.isdir(refdir)):
        targets.append("ref")
    subprocess.run(["make", "-s", "-C", _HERE, f"REF={refdir}", *targets],
                   check=True)


def _load(path):
    return ctypes.CDLL(path) if os.path.exists(path) else None


_lib = None
_ref = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            build(ref=False)
        _lib = ctypes.CDLL(_LIB)
    return _lib


def ref():
    global _ref
    if _ref is None:
        _ref = _load(_REF)
    return _ref


def have_ref() -> bool:
    return ref() is not None


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_vp)


def _sfx(dtype) -> str:
    dtype = np.dtype(dtype)
    if dtype == np.float32:
        return "f32"
    if dtype == np.float64:
        return "f64"
    raise TypeError(f"oracle computes in float32 or float64, not {dtype}")


# --------------------------------------------------------------------- 2D --

def conv2d(src: np.ndarray, filt: np.ndarray, boundary: str = "zero",
           steps: int = 1) -> np.ndarray:
    """``Convolution<T>`` (ssai-2dconv/common.h:186-216) applied ``steps``
    times; ``filt`` is the (fh, fw) weight matrix, row = y offset."""
    src = np.ascontiguousarray(src)
    h, w = src.shape
    filt = np.ascontiguousarray(filt, dtype=src.dtype)
    fh, fw = filt.shape
    dst = np.empty_like(src)
    work = np.empty_like(src)
    fn = getattr(lib(), "ssam_oracle_steps2d_" + _sfx(src.dtype))
    fn(_ptr(src), _ptr(dst), _ptr(work), _i64(w), _i64(h), _i64(w),
       _ptr(filt), ctypes.c_int(fw), ctypes.c_int(fh),
       ctypes.c_int(BND[boundary]), ctypes.c_int(steps))
    return dst


def ref_convolution(src: np.ndarray, filt: np.ndarray) -> np.ndarray:
    """The reference's compiled ``Convolution<T>`` itself (zero padding)."""
    r = ref()
    if r is None:
        raise RuntimeError("oracle/_ref is not built")
    src = np.ascontiguousarray(src)
    h, w = src.shape
    filt = np.ascontiguousarray(filt, dtype=src.dtype)
    fh, fw = filt.shape
    dst = np.empty_like(src)
    fn = getattr(r, "ssam_ref_convolution_" + _sfx(src.dtype))
    fn(_ptr(src), _ptr(dst), ctypes.c_int(w), ctypes.c_int(h), _ptr(filt),
       ctypes.c_int(fw), ctypes.c_int(fh))
    return dst


# --------------------------------------------------------------------- 3D --

def taps3d(src: np.ndarray, taps, boundary: str = "gold",
           out: np.ndarray | None = None) -> np.ndarray:
    """Ordered tap list ``[(dz, dy, dx, coef), ...]`` evaluated like the
    reference golds (tmp3d7pt-v2.cu:278-298, tmp3d13pt.cu:301-327)."""
    src = np.ascontiguousarray(src)
    nz, ny, nx = src.shape
    if out is None:
        out = np.zeros_like(src)
    dz = np.array([t[0] for t in taps], np.int32)
    dy = np.array([t[1] for t in taps], np.int32)
    dx = np.array([t[2] for t in taps], np.int32)
    cf = np.array([t[3] for t in taps], src.dtype)
    reach = int(max(max(abs(dz).max(), abs(dy).max()), abs(dx).max()))
    fn = getattr(lib(), "ssam_oracle_taps3d_" + _sfx(src.dtype))
    fn(_ptr(src), _ptr(out), _i64(nx), _i64(ny), _i64(nz), ctypes.c_int(len(taps)),
       _ptr(dz), _ptr(dy), _ptr(dx), _ptr(cf), ctypes.c_int(reach),
       ctypes.c_int(BND[boundary]))
    return out


def poisson19(src: np.ndarray, boundary: str = "gold",
              out: np.ndarray | None = None) -> np.ndarray:
    """``poisson_gold`` (tmpPoisson.cu:369-386), evaluated in double."""
    src = np.ascontiguousarray(src)
    nz, ny, nx = src.shape
    if out is None:
        out = np.zeros_like(src)
    fn = getattr(lib(), "ssam_oracle_poisson19_" + _sfx(src.dtype))
    fn(_ptr(src), _ptr(out), _i64(nx), _i64(ny), _i64(nz),
       ctypes.c_int(BND[boundary]))
    return out


def steps3d(src: np.ndarray, one_step, steps: int) -> np.ndarray:
    """Iterate a 3D gold the way the reference checks IT fused steps
    (tmp3d7pt-v2.cu:312-317): run, copy back, run again."""
    cur = np.ascontiguousarray(src)
    for _ in range(steps):
        cur = one_step(cur)
    return cur


def ref_gold3d(name: str, src: np.ndarray) -> np.ndarray:
    """One call of the reference's compiled ``v2::j3d7pt_gold``,
    ``j3d13pt_gold`` or ``poisson_gold`` on a cube (output starts at 0, ring
    stays 0, as in the reference's tests)."""
    r = ref()
    if r is None:
        raise RuntimeError("oracle/_ref is not built")
    src = np.ascontiguousarray(src)
    n = src.shape[0]
    assert src.shape == (n, n, n)
    out = np.zeros_like(src)
    fn = getattr(r, f"ssam_ref_{name}_" + _sfx(src.dtype))
    if fn(_ptr(src), _ptr(out), ctypes.c_int(n)) != 0:
        raise ValueError(f"reference gold not instantiated for N={n}")
    return out


def rms_max_error(out: np.ndarray, ref_: np.ndarray, lo: int, hi_off: int):
    """``checkError3D`` (common.hpp:84-127) over [lo, n-hi_off) per axis."""
    out = np.ascontiguousarray(out, np.float64)
    ref_ = np.ascontiguousarray(ref_, np.float64)
    nz, ny, nx = out.shape
    rms = ctypes.c_double()
    mx = ctypes.c_double()
    lib().ssam_oracle_check_error3d_f64(
        _ptr(out), _ptr(ref_), _i64(nx), _i64(ny), _i64(lo), _i64(nz - hi_off),
        _i64(lo), _i64(ny - hi_off), _i64(lo), _i64(nx - hi_off),
        ctypes.byref(rms), ctypes.byref(mx))
    return rms.value, mx.value


# ---------------------------------------------------------------- Poisson --

def jacobi7(rhs: np.ndarray, u: np.ndarray, sweeps: int) -> np.ndarray:
    """FP64 Jacobi sweeps of -lap(u) = rhs, Dirichlet 0, shape (nb, n, n, n)."""
    rhs = np.ascontiguousarray(rhs, np.float64)
    u = np.ascontiguousarray(u, np.float64)
    nb, n = rhs.shape[0], rhs.shape[1]
    out = np.empty_like(u)
    work = np.empty_like(u)
    if sweeps == 0:
        return u.copy()
    lib().ssam_oracle_jacobi7_f64(_ptr(rhs), _ptr(u), _ptr(out), _i64(n), _i64(nb),
                                  ctypes.c_int(sweeps), _ptr(work))
    return out


def residual7(f: np.ndarray, u: np.ndarray):
    """(r, rel) with r = f - A u and rel = ||r|| / ||f|| per right-hand side
    (||r|| itself where f = 0, as the library's ssam_poisson_residual)."""
    f = np.ascontiguousarray(f, np.float64)
    u = np.ascontiguousarray(u, np.float64)
    nb, n = f.shape[0], f.shape[1]
    r = np.empty_like(f)
    norms = np.zeros(2 * nb)
    lib().ssam_oracle_residual7_f64(_ptr(f), _ptr(u), _ptr(r), _i64(n), _i64(nb), _ptr(norms))
    rr, ff = norms[0::2], norms[1::2]
    return r, np.sqrt(np.where(ff > 0, rr / np.where(ff > 0, ff, 1.0), rr))

