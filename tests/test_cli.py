"""The reference-spelling command-line drop-ins (ssai-2dstencil, ssai-2dconv,
ssai-3dstencil): argument handling on the CPU; on a GPU, every stencil name
runs and passes its own sampled check against a host evaluation."""
import os
import subprocess

import pytest

BIN = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "ssam_b200",
                   "bin")


def run(exe, *args, timeout=300, cwd=None):
    return subprocess.run([os.path.join(BIN, exe), *map(str, args)], capture_output=True,
                          text=True, timeout=timeout, cwd=cwd)


@pytest.mark.parametrize("exe", ["ssai-2dstencil", "ssai-2dconv", "ssai-3dstencil"])
def test_programs_are_built_and_print_usage(exe):
    assert os.path.exists(os.path.join(BIN, exe)), "run the build first"
    r = run(exe)
    assert r.returncode == 1
    assert exe in r.stdout


def test_unknown_stencil_name_is_refused():
    r = run("ssai-2dstencil", 64, "7", "float")
    assert r.returncode == 1 and "do not call" in r.stdout
    r = run("ssai-3dstencil", "box", "float")
    assert r.returncode == 1 and "invalid function name" in r.stdout


@pytest.mark.gpu
@pytest.mark.parametrize("pts", ["5", "9", "13", "17", "21", "25", "64", "81", "121", "tmp_5",
                                 "tmp_9"])
@pytest.mark.parametrize("dtype", ["float", "double"])
def test_2dstencil_names(cuda, pts, dtype):
    """Every stencil name runs the reference test's computation (its table,
    input recipe and step count) and passes the band check against the
    reference's Convolution applied on the host, printing its "verify dif"."""
    r = run("ssai-2dstencil", 1000, pts, dtype)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "max relative error" in r.stdout and "verify dif =" in r.stdout
    if pts.startswith("tmp"):
        assert f"Iterative={5 if pts == 'tmp_5' else 3}" in r.stdout


@pytest.mark.gpu
def test_2dstencil_runs_repeat_with_a_fixed_seed(cuda):
    """The reference's rand()-drawn inputs and taps come from srand(SSAM_SEED)
    (default 1), so two runs print the same verify line."""
    a = run("ssai-2dstencil", 512, "5", "float")
    b = run("ssai-2dstencil", 512, "5", "float")
    la = [l for l in a.stdout.splitlines() if l.startswith("verify dif")]
    lb = [l for l in b.stdout.splitlines() if l.startswith("verify dif")]
    assert a.returncode == 0 and la == lb


@pytest.mark.gpu
@pytest.mark.parametrize("fsize", [2, 3, 7, 21, 28])
@pytest.mark.parametrize("dtype", ["float", "double"])
def test_2dconv_sizes(cuda, fsize, dtype):
    r = run("ssai-2dconv", dtype, 777, fsize)
    assert r.returncode == 0, r.stdout + r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["7pt", "13pt", "poisson"])
@pytest.mark.parametrize("dtype", ["float", "double"])
@pytest.mark.parametrize("n,it", [(64, 1), (48, 2)])
def test_3dstencil_names(cuda, name, dtype, n, it):
    r = run("ssai-3dstencil", name, dtype, n, it)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "RMS Error" in r.stdout


@pytest.mark.gpu
@pytest.mark.parametrize("name,its", [("7pt", [2, 3, 3, 4]), ("13pt", [2]), ("poisson", [2, 3, 3])])
def test_3dstencil_runs_the_reference_sequence(cuda, name, its):
    """Without an IT argument the program runs the reference's sequence of
    ITERATIVE_COUNT tests, each on a fresh rand() grid, each passing
    checkError3D's RMS tolerance."""
    r = run("ssai-3dstencil", name, "float", 64)
    assert r.returncode == 0, r.stdout + r.stderr
    got = [int(l.split("ITERATIVE_COUNT=")[1].split(":")[0]) for l in r.stdout.splitlines()
           if "ITERATIVE_COUNT=" in l]
    assert got == its
    assert r.stdout.count("[Test] RMS Error") == len(its)


@pytest.mark.gpu
def test_2dconv_reads_the_reference_raw_image(cuda, tmp_path):
    """With ../data/Lena<N>x<N>.raw beside the working directory (the
    reference driver's input, 8-bit pixels) the program convolves that image
    and its sampled check still holds; without it, seeded data."""
    import numpy as np
    n = 256
    (tmp_path / "data").mkdir()
    (tmp_path / "run").mkdir()
    img = (np.arange(n * n) * 37 % 251).astype(np.uint8)
    (tmp_path / "data" / f"Lena{n}x{n}.raw").write_bytes(img.tobytes())
    r = run("ssai-2dconv", "float", n, 5, cwd=str(tmp_path / "run"))
    assert r.returncode == 0, r.stdout + r.stderr
    assert f"Load success : ../data/Lena{n}x{n}.raw" in r.stdout
    r = run("ssai-2dconv", "float", 128, 5, cwd=str(tmp_path / "run"))
    assert r.returncode == 0 and "Load failed" in r.stdout
