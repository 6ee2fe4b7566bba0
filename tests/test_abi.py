"""The C ABI library loads on a machine without a GPU, exports every entry
point that include/ssam.h declares, and rejects bad arguments before it
touches CUDA (no compute is launched here)."""
import ctypes
import os
import re

import pytest

import ssam_b200 as S

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                      "include", "ssam.h")


def declared_functions():
    with open(HEADER) as f:
        text = f.read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return re.findall(r"SSAM_API\s+[\w\s\*]+?\b(ssam_\w+)\s*\(", text)


def test_header_declares_entry_points():
    names = declared_functions()
    assert "ssam_stencil2d" in names and "ssam_conv2d" in names
    assert len(names) == len(set(names))


@pytest.mark.parametrize("name", declared_functions())
def test_library_exports_declared_symbol(name):
    lib = ctypes.CDLL(S.LIB_PATH)
    assert hasattr(lib, name), f"{name} declared in include/ssam.h but not exported"


def test_abi_version():
    assert S.lib().ssam_abi_version() == 2


FAKE_SRC = 0x7f0000000000
FAKE_DST = 0x7f1000000000


def _st2d(**kw):
    a = dict(src=FAKE_SRC, dst=FAKE_DST, w=64, h=64, pitch=64, dtype=S.F32, shape=S.STAR,
             r=1, coeffs=[0.2] * 5, steps=1, bnd=0)
    a.update(kw)
    c = (ctypes.c_double * max(1, len(a["coeffs"])))(*a["coeffs"]) if a["coeffs"] is not None else None
    return S.lib().ssam_stencil2d(a["src"], a["dst"], a["w"], a["h"], a["pitch"], a["dtype"],
                                  a["shape"], a["r"], c, a["steps"], a["bnd"], None)


@pytest.mark.parametrize("kw", [
    dict(src=0), dict(dst=0), dict(w=0), dict(h=-1), dict(pitch=10), dict(dtype=9),
    dict(shape=7), dict(r=0), dict(r=7), dict(shape=S.BOX, r=11), dict(coeffs=None),
    dict(steps=0), dict(bnd=5), dict(bnd=1, steps=2), dict(dst=FAKE_SRC + 128),
    dict(pitch=1 << 62), dict(pitch=(1 << 61) + 1, h=5),  # pitch * height * 4 overflows
])
def test_stencil2d_rejects_bad_arguments(kw):
    assert _st2d(**kw) == S.ERR_INVALID
    assert S.lib().ssam_last_error().decode()


def test_noalloc_rejects_overflowing_pitch():
    """A pitch whose pitch * height * element size wraps around 64 bits is
    rejected before the no-allocation entry compares it with its array (it
    would otherwise pass the size check and write outside the array)."""
    lib = S.lib()
    fn = lib.ssam_stencil2d_noalloc
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64,
                   ctypes.c_int64, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                   ctypes.POINTER(ctypes.c_double), ctypes.c_int, ctypes.c_int,
                   ctypes.c_void_p]
    c = (ctypes.c_double * 9)(*([0.1] * 9))
    pitch = (1 << 62) + 16  # * 64 rows * 4 bytes wraps to a small number
    st = fn(FAKE_SRC, FAKE_DST, 64, 64, pitch, S.F32, S.BOX, 1, c, 4, 0, None)
    assert st == S.ERR_INVALID
    assert "overflow" in lib.ssam_last_error().decode()


@pytest.mark.parametrize("fw,fh", [(0, 3), (3, 0), (29, 3), (3, 29)])
def test_conv2d_rejects_bad_filter(fw, fh):
    w = (ctypes.c_double * 9)(*([1.0] * 9))
    st = S.lib().ssam_conv2d(FAKE_SRC, FAKE_DST, 64, 64, 64, S.F32, w, fw, fh, 0, None)
    assert st == S.ERR_INVALID


def test_python_front_end_refuses_host_tensors():
    import torch
    with pytest.raises(ValueError):
        S.stencil2d(torch.zeros(8, 8), [0.2] * 5, 1)


def test_autotune_cache_file_roundtrip(tmp_path):
    """The tuning cache persists as text and rejects malformed files (no GPU)."""
    lib = S.lib()
    S.autotune_clear()
    p = tmp_path / "tune.txt"
    S.autotune_save(str(p))
    assert p.read_text().startswith("# ssam_b200 autotune cache")
    p.write_text("# ssam_b200 autotune cache v1\n"
                 "choice 0 1 1 1 1 0 1 13 13 8 4 4\n"
                 "depth 0 1 1 1 1 0 13 13 4\n")
    S.autotune_load(str(p))
    q = tmp_path / "again.txt"
    S.autotune_save(str(q))
    assert "choice 0 1 1 1 1 0 1 13 13 8 4 4" in q.read_text()
    assert "depth 0 1 1 1 1 0 13 13 4" in q.read_text()
    bad = tmp_path / "bad.txt"
    bad.write_text("choice 1 2 3\n")
    with pytest.raises(S.SsamError):
        S.autotune_load(str(bad))
    with pytest.raises(S.SsamError):
        S.autotune_load(str(tmp_path / "missing.txt"))
    S.autotune_clear()
    assert lib.ssam_autotune_clear() == 0


def test_autotune_3d_choices_roundtrip(tmp_path):
    """The 3D autotuner's choices (choice3d lines: dtype, shape, radius, rhs,
    size class, PY, NW, S, z-register flag, V) persist beside the 2D ones; bad
    lines are rejected; clearing forgets both kinds (no GPU)."""
    S.autotune_clear()
    p = tmp_path / "tune3d.txt"
    p.write_text("# ssam_b200 autotune cache v1\n"
                 "choice 0 2 2 2 2 0 1 13 13 32 2 4\n"
                 "choice3d 0 0 2 0 9 9 9 2 16 8 1 4\n"
                 "choice3d 2 0 1 1 7 7 10 4 8 6 0 8\n")
    S.autotune_load(str(p))
    q = tmp_path / "again.txt"
    S.autotune_save(str(q))
    text = q.read_text()
    assert "choice3d 0 0 2 0 9 9 9 2 16 8 1 4 1" in text
    assert "choice3d 2 0 1 1 7 7 10 4 8 6 0 8 1" in text
    assert "choice 0 2 2 2 2 0 1 13 13 32 2 4" in text
    for bad_line in ("choice3d 0 0 2 0 9 9 9 2 16 8 2 4\n",   # z flag must be 0 or 1
                     "choice3d 0 0 2 0 9 9 9 0 16 8 1 4\n",   # PY >= 1
                     "choice3d 0 0 2 0 9 9 9 2 16 8 1 0\n",   # V >= 1
                     "choice3d 0 0 2 0 9 9 9 2 16 8 0 4 3\n",  # 1 or 2 steps a launch
                     "depth3d 0 0 1 9 9 9 0\n",               # depth 1 or 2
                     "depth3d 0 0 1 9 9\n",
                     "choice3d 0 0 2 0 9 9\n"):
        bad = tmp_path / "bad3d.txt"
        bad.write_text(bad_line)
        with pytest.raises(S.SsamError):
            S.autotune_load(str(bad))
    # a line saved before the columns-a-thread field reads as V = 4
    old = tmp_path / "old3d.txt"
    old.write_text("choice3d 1 1 1 0 8 8 8 4 4 5 0\n")
    S.autotune_load(str(old))
    S.autotune_save(str(q))
    assert "choice3d 1 1 1 0 8 8 8 4 4 5 0 4 1" in q.read_text()
    # two-step configurations (last field t = 2) and the temporal depth of a
    # size class are kept apart from the single-step choice of that class
    two = tmp_path / "two3d.txt"
    two.write_text("choice3d 0 0 1 0 9 9 9 4 8 6 0 4 2\n"
                   "choice3d 0 0 1 0 9 9 9 2 8 8 1 8\n"
                   "depth3d 0 0 1 9 9 9 2\n")
    S.autotune_load(str(two))
    S.autotune_save(str(q))
    text = q.read_text()
    assert "choice3d 0 0 1 0 9 9 9 4 8 6 0 4 2" in text
    assert "choice3d 0 0 1 0 9 9 9 2 8 8 1 8 1" in text
    assert "depth3d 0 0 1 9 9 9 2" in text
    S.autotune_clear()
    S.autotune_save(str(q))
    assert "choice3d" not in q.read_text() and "depth3d" not in q.read_text()


def test_debug_hook_rejects_out_of_range_settings():
    """The bounded-wait test hook validates its settings (no GPU)."""
    lib = S.lib()
    assert lib.ssam_debug_batched_barrier(5000, 0) == S.ERR_INVALID
    assert lib.ssam_debug_batched_barrier(0, 10**12) == S.ERR_INVALID
    assert lib.ssam_debug_batched_barrier(0, 0) == S.OK
