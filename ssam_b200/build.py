"""In-tree build of libssam_b200.so for sm_100a.

    python -m ssam_b200.build [-j N] [--ptxas-verbose]

The kernel instantiation list below is the single source of truth for which
(dtype, reach, shape, P, fused steps) kernels exist; the C ABI reports
SSAM_ERR_UNSUPPORTED for anything else.  Generated instantiation units and
objects go to ssam_b200/_build/ (not committed); the shared library lands
next to this file so that it travels with the source tree.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import hashlib
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libssam_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC",
           "-Xcompiler", "-fvisibility=hidden", "--expt-relaxed-constexpr",
           "-Wno-deprecated-gpu-targets"]

# Hand-written (non-generated) translation units.
SOURCES = ["api.cu", "autotune.cu", "stencil3d.cu", "noalloc.cu", "batched.cu",
           "poisson.cu", "cnn.cu", "cnn_conv_ring.cu", "cnn_net.cu"]

DTYPES = {"f32": "float", "f64": "double", "bf16": "__nv_bfloat16", "f16": "__half"}


def instances():
    """(dtype, star, rl, rr, P, T, V) of every compiled 2D kernel.

    V is the number of columns a thread owns (the warp strip is 32*V
    columns): 4 (16 bytes) for FP32, 4 (32 bytes) for FP64, 8 (16 bytes) for
    the 16-bit types by default; FP32/FP64 also get V = 8 for the single-step
    stencils, which halves the halo lanes of the wide (r > 4) stencils and
    gives the autotuner a second strip width.
    """
    out = []
    for dt in DTYPES:
        wide = dt in ("f32", "f64")
        v0 = 4 if wide else 8
        vs = (v0, 8) if wide else (v0,)
        # star r = 1..6 (5/9/13/17/21/25-pt) and box r = 1..5
        # (9/25/49/81/121-pt; conv F = 3..11)
        for star, rmax in ((1, 6), (0, 5)):
            for r in range(1, rmax + 1):
                for v in vs:
                    for p in ((4, 8, 16) if v == v0 else (4, 8)):
                        out.append((dt, star, r, r, p, 1, v))
        # temporal blocking for the bandwidth-bound radii
        for star in (1, 0):
            for r, ts in ((1, (2, 4, 8)), (2, (2, 4))):
                for t in ts:
                    out.append((dt, star, r, r, 8, t, v0))
        # every other square conv size up to 28 (even F has rl = rr + 1)
        if wide:
            for f in range(1, 29):
                rl, rr = f // 2, f - 1 - f // 2
                if f % 2 == 1 and 1 <= rl <= 5:
                    continue
                out.append((dt, 0, rl, rr, 4, 1, v0))
                if rl > 4:
                    out.append((dt, 0, rl, rr, 4, 1, 8))
    return out


def instances_3d():
    """(dtype, shape, r, PY, NW, S, rhs, default, zreg, V) of every compiled
    3D configuration: shape 0 = star (r = 1: 7-pt, r = 2: 13-pt), 1 = the
    19-point Poisson operator; rhs = the Jacobi-sweep form with a
    right-hand-side term; zreg = the kernel that keeps each thread's own
    cells in a register ring along z (stencil3d_zreg.cuh; "z" below); V =
    columns a thread ("z8" / "c8" below: V = 8, a 256-column tile staged as
    two TMA boxes; else 4).  The first of each group is the default; the 3D
    autotuner times them all."""
    cfg = {
        "f32": {(0, 1): [(4, 8, 6), (4, 4, 8), (2, 16, 6), (4, 16, 5), (8, 8, 5),
                         (2, 16, 4, "z"), (2, 8, 4, "z"), (2, 16, 8, "z"), (2, 8, 8, "z"),
                         (2, 8, 4, "z8"), (2, 8, 8, "z8"), (4, 8, 6, "c8")],
                (0, 2): [(4, 4, 8), (4, 8, 6), (2, 8, 6), (2, 16, 6), (4, 12, 6), (4, 12, 8),
                         (2, 12, 4, "z"), (2, 16, 4, "z"), (2, 16, 8, "z"), (2, 12, 8, "z"),
                         (2, 8, 4, "z8"), (2, 8, 8, "z8"), (4, 4, 8, "c8")],
                (1, 1): [(4, 8, 6), (4, 4, 8), (2, 16, 6), (4, 16, 5), (4, 8, 8),
                         (2, 16, 4, "z"), (2, 8, 4, "z"), (2, 16, 8, "z"), (4, 8, 8, "z")],
                "rhs": [(4, 8, 6), (4, 4, 8), (2, 16, 6), (4, 16, 5),
                        (2, 16, 4, "z"), (2, 8, 4, "z"), (2, 16, 8, "z"), (2, 8, 8, "z"),
                        (4, 12, 8, "z")]},
        "bf16": {(0, 1): [(4, 8, 6), (2, 16, 6), (4, 16, 6), (8, 8, 6), (2, 16, 4, "z"),
                          (2, 16, 8, "z"), (4, 12, 8, "z"), (2, 8, 4, "z8"), (4, 8, 6, "c8")],
                 (0, 2): [(4, 4, 8), (4, 8, 6), (2, 16, 6), (2, 12, 4, "z"), (2, 16, 8, "z"),
                          (2, 8, 4, "z8"), (2, 8, 8, "z8"), (4, 4, 8, "c8"), (2, 12, 8, "z")],
                 (1, 1): [(4, 8, 6), (2, 16, 6), (4, 16, 6), (2, 16, 4, "z"), (2, 16, 8, "z")],
                 "rhs": [(4, 8, 6), (2, 16, 6), (4, 16, 6), (2, 16, 4, "z"), (2, 8, 4, "z"),
                         (2, 16, 8, "z"), (4, 12, 8, "z")]},
        "f64": {(0, 1): [(4, 4, 5), (4, 8, 5), (2, 8, 5), (2, 4, 4, "z"), (2, 8, 8, "z")],
                (0, 2): [(4, 4, 6), (2, 8, 6), (2, 4, 4, "z"), (2, 8, 8, "z")],
                (1, 1): [(4, 4, 5), (2, 8, 5), (2, 4, 4, "z"), (2, 8, 8, "z")],
                "rhs": [(4, 4, 5), (2, 8, 5), (2, 4, 4, "z"), (2, 8, 8, "z")]},
        "f16": {(0, 1): [(4, 8, 6)], (0, 2): [(4, 4, 8)], (1, 1): [(4, 8, 6)]},
    }
    out = []
    for dt, groups in cfg.items():
        for key, lst in groups.items():
            shape, r, rhs = (0, 1, True) if key == "rhs" else (key[0], key[1], False)
            for i, c in enumerate(lst):
                tag = c[3] if len(c) > 3 else ""
                out.append((dt, shape, r, c[0], c[1], c[2], rhs, i == 0, tag.startswith("z"),
                            8 if tag.endswith("8") else 4))
    return out


def instances_3d_t2():
    """(dtype, shape, r, PY, NW, S, V, default) of every compiled 3D
    configuration that applies two time steps per launch (stencil3d_t2.cuh):
    shape 0 = star (r = 1: 7-pt, r = 2: 13-pt), 1 = the 19-point operator.
    The first of each group is the default.  Limits (static_asserts of the
    kernel): 2*R*(PY + 2*EY) <= 32 x-halo values a warp (EY = 1 for the
    19-point operator, else 0), 2R staged halo columns (FP64 holds 2: r = 1
    only), PY >= R, ring slots S >= 2R + 2."""
    cfg = {
        "f32": {(0, 1): [(4, 8, 6, 4), (2, 8, 6, 8), (4, 7, 6, 4), (6, 7, 6, 4), (2, 8, 4, 8)],
                (0, 2): [(2, 8, 8, 4), (4, 7, 8, 4)],
                (1, 1): [(2, 8, 6, 4), (4, 7, 6, 4)]},
        "bf16": {(0, 1): [(2, 8, 6, 8), (4, 7, 6, 8), (4, 8, 6, 4)],
                 (0, 2): [(2, 8, 8, 4), (4, 7, 8, 4)],
                 (1, 1): [(2, 8, 6, 8), (4, 7, 6, 4)]},
        "f64": {(0, 1): [(2, 8, 6, 4), (4, 7, 6, 4)],
                (1, 1): [(2, 8, 6, 4)]},
    }
    out = []
    for dt, groups in cfg.items():
        for (shape, r), lst in groups.items():
            for i, (py, nw, s_, v) in enumerate(lst):
                out.append((dt, shape, r, py, nw, s_, v, i == 0))
    return out


def rowloop_instances():
    """(dtype, rl, rr, V) of every compiled row-loop 2D kernel (square filters
    of width FW = rl + rr + 1 >= 7: box r = 3..5 and the wider correlations;
    registered with P = 1)."""
    out = []
    for dt, vs in (("f32", (4, 8)), ("f64", (4,))):
        for f in range(7, 29):
            rl, rr = f // 2, f - 1 - f // 2
            for v in vs:
                if (rl + v - 1) // v + (rr + v - 1) // v <= 30:
                    out.append((dt, rl, rr, v))
    return out


def stream_t_instances():
    """(dtype, star, r, SEG, V, T) of every compiled row-streaming kernel with
    T fused steps (r = 1: T = 2, 4; r = 2: T = 2), registered with P = SEG."""
    out = []
    for dt in ("f32", "f64", "bf16"):
        v = 8 if dt == "bf16" else 4
        for star in (1, 0):
            for r, ts in ((1, (2, 4)), (2, (2,))):
                for t in ts:
                    out.append((dt, star, r, 64, v, t))
    return out


def stream_instances():
    """(dtype, star, r, SEG, V) of every compiled row-streaming 2D kernel
    (one step per launch; a warp walks SEG output rows), registered with
    P = SEG: star r = 1..5 and box r = 1..5 at the default strip width.  (Not
    star r = 6: its 14-row ring measured 321 GCells/s on 8192^2 FP32 against
    388 for the windowed tile.  FP32 with V = 8 measured 10-20 % slower than
    V = 4: more registers, fewer warps.)"""
    out = []
    for dt in DTYPES:
        v = 4 if dt in ("f32", "f64") else 8
        for star, rmax in ((1, 5), (0, 5)):
            for r in range(1, rmax + 1):
                for seg in (32, 128):
                    out.append((dt, star, r, seg, v))
    return out


def _gen_units(chunk: int = 6):
    os.makedirs(os.path.join(BUILD, "gen"), exist_ok=True)
    by_dt: dict[str, list] = {}
    for inst in instances():
        by_dt.setdefault(inst[0], []).append(inst)
    units = []
    for dt, lst in by_dt.items():
        for c in range(0, len(lst), chunk):
            part = lst[c:c + chunk]
            name = f"inst2d_{dt}_{c // chunk:02d}.cu"
            lines = ["// generated by ssam_b200/build.py -- do not edit",
                     '#include "../../csrc/stencil2d.cuh"', "namespace ssam {"]
            for (_, star, rl, rr, p, t, v) in part:
                tag = f"{'s' if star else 'b'}_{rl}_{rr}_{p}_{t}_{v}"
                lines.append(
                    f"static Register2D<{DTYPES[dt]}, {rl}, {rr}, {rl}, {rr}, "
                    f"{'true' if star else 'false'}, {p}, {t}, {v}> reg_{tag};")
            lines.append("}  // namespace ssam")
            text = "\n".join(lines) + "\n"
            path = os.path.join(BUILD, "gen", name)
            if not os.path.exists(path) or open(path).read() != text:
                with open(path, "w") as f:
                    f.write(text)
            units.append(path)
    by_dt = {}
    for inst in instances_3d():
        by_dt.setdefault(inst[0], []).append(inst)
    for dt, lst in by_dt.items():
        for c in range(0, len(lst), 3):
            part = lst[c:c + 3]
            name = f"inst3d_{dt}_{c // 3:02d}.cu"
            lines = ["// generated by ssam_b200/build.py -- do not edit",
                     '#include "../../csrc/stencil3d_launch.cuh"', "namespace ssam {"]
            for (_, shape, r, py, nw, s, rhs, dflt, zreg, v) in part:
                sh = "SH3_POISSON19" if shape else "SH3_STAR"
                tag = f"{shape}_{r}_{py}_{nw}_{s}_{int(rhs)}_{int(zreg)}_{v}"
                lines.append(
                    f"static Register3D<{DTYPES[dt]}, {sh}, {r}, {py}, {nw}, {s}, "
                    f"{'true' if rhs else 'false'}, {'true' if dflt else 'false'}, "
                    f"{'true' if zreg else 'false'}, {v}> reg3_{tag};")
            lines.append("}  // namespace ssam")
            text = "\n".join(lines) + "\n"
            path = os.path.join(BUILD, "gen", name)
            if not os.path.exists(path) or open(path).read() != text:
                with open(path, "w") as f:
                    f.write(text)
            units.append(path)
    by_dt = {}
    for inst in instances_3d_t2():
        by_dt.setdefault(inst[0], []).append(inst)
    for dt, lst in by_dt.items():
        for c in range(0, len(lst), 2):
            part = lst[c:c + 2]
            name = f"inst3dt_{dt}_{c // 2:02d}.cu"
            lines = ["// generated by ssam_b200/build.py -- do not edit",
                     '#include "../../csrc/stencil3d_launch.cuh"', "namespace ssam {"]
            for (_, shape, r, py, nw, s_, v, dflt) in part:
                sh = "SH3_POISSON19" if shape else "SH3_STAR"
                lines.append(
                    f"static Register3D<{DTYPES[dt]}, {sh}, {r}, {py}, {nw}, {s_}, false, "
                    f"{'true' if dflt else 'false'}, false, {v}, 2> "
                    f"reg3t_{shape}_{r}_{py}_{nw}_{s_}_{v};")
            lines.append("}  // namespace ssam")
            text = "\n".join(lines) + "\n"
            path = os.path.join(BUILD, "gen", name)
            if not os.path.exists(path) or open(path).read() != text:
                with open(path, "w") as f:
                    f.write(text)
            units.append(path)
    by_dt = {}
    for inst in rowloop_instances():
        by_dt.setdefault(inst[0], []).append(inst)
    for dt, lst in by_dt.items():
        for c in range(0, len(lst), chunk):
            part = lst[c:c + chunk]
            name = f"inst2dr_{dt}_{c // chunk:02d}.cu"
            lines = ["// generated by ssam_b200/build.py -- do not edit",
                     '#include "../../csrc/stencil2d_rowloop.cuh"', "namespace ssam {"]
            for (_, rl, rr, v) in part:
                lines.append(f"static RegisterRowLoop2D<{DTYPES[dt]}, {rl}, {rr}, {rl}, {rr}, {v}> "
                             f"regr_{rl}_{rr}_{v};")
            lines.append("}  // namespace ssam")
            text = "\n".join(lines) + "\n"
            path = os.path.join(BUILD, "gen", name)
            if not os.path.exists(path) or open(path).read() != text:
                with open(path, "w") as f:
                    f.write(text)
            units.append(path)
    by_dt = {}
    for inst in stream_t_instances():
        by_dt.setdefault(inst[0], []).append(inst)
    for dt, lst in by_dt.items():
        for c in range(0, len(lst), 3):
            part = lst[c:c + 3]
            name = f"inst2dt_{dt}_{c // 3:02d}.cu"
            lines = ["// generated by ssam_b200/build.py -- do not edit",
                     '#include "../../csrc/stencil2d_stream_t.cuh"', "namespace ssam {"]
            for (_, star, r, seg, v, t) in part:
                lines.append(
                    f"static RegisterStreamT2D<{DTYPES[dt]}, {r}, {r}, {r}, {r}, "
                    f"{'true' if star else 'false'}, {seg}, {v}, {t}> "
                    f"regt_{'s' if star else 'b'}_{r}_{t};")
            lines.append("}  // namespace ssam")
            text = "\n".join(lines) + "\n"
            path = os.path.join(BUILD, "gen", name)
            if not os.path.exists(path) or open(path).read() != text:
                with open(path, "w") as f:
                    f.write(text)
            units.append(path)
    by_dt = {}
    for inst in stream_instances():
        by_dt.setdefault(inst[0], []).append(inst)
    for dt, lst in by_dt.items():
        for c in range(0, len(lst), chunk):
            part = lst[c:c + chunk]
            name = f"inst2ds_{dt}_{c // chunk:02d}.cu"
            lines = ["// generated by ssam_b200/build.py -- do not edit",
                     '#include "../../csrc/stencil2d_stream.cuh"', "namespace ssam {"]
            for (_, star, r, seg, v) in part:
                tag = f"{'s' if star else 'b'}_{r}_{seg}_{v}"
                lines.append(
                    f"static RegisterStream2D<{DTYPES[dt]}, {r}, {r}, {r}, {r}, "
                    f"{'true' if star else 'false'}, {seg}, {v}> regs_{tag};")
            lines.append("}  // namespace ssam")
            text = "\n".join(lines) + "\n"
            path = os.path.join(BUILD, "gen", name)
            if not os.path.exists(path) or open(path).read() != text:
                with open(path, "w") as f:
                    f.write(text)
            units.append(path)
    return units


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _local_headers(path: str, seen: set[str] | None = None) -> list[str]:
    """The quoted #include files that `path` pulls in, recursively."""
    seen = set() if seen is None else seen
    with open(path) as f:
        for line in f:
            line = line.strip()
            if line.startswith("#include") and '"' in line:
                inc = os.path.normpath(os.path.join(os.path.dirname(path),
                                                    line.split('"')[1]))
                if inc not in seen and os.path.exists(inc):
                    seen.add(inc)
                    _local_headers(inc, seen)
    return sorted(seen)


def _unit_digest(src: str) -> str:
    """Compiler flags plus the contents of the headers this unit includes."""
    h = hashlib.sha1()
    for hdr in _local_headers(src):
        with open(hdr, "rb") as f:
            h.update(f.read())
    h.update(" ".join(NVFLAGS + ARCH).encode())
    return h.hexdigest()


def _compile(src: str, obj: str, extra: list[str], stamp: str) -> str:
    stamp_path = obj + ".stamp"
    if (os.path.exists(obj) and os.path.exists(stamp_path)
            and open(stamp_path).read() == stamp
            and os.path.getmtime(obj) >= os.path.getmtime(src)):
        return obj
    cmd = [_nvcc(), *ARCH, *NVFLAGS, *extra, "-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
    if r.stderr.strip() and "-Xptxas" in " ".join(extra):
        with open(obj + ".ptxas.txt", "w") as f:
            f.write(r.stderr)
    with open(stamp_path, "w") as f:
        f.write(stamp)
    return obj


def build(jobs: int | None = None, ptxas_verbose: bool = False, quiet: bool = True) -> str:
    os.makedirs(BUILD, exist_ok=True)
    units = [os.path.join(CSRC, s) for s in SOURCES] + _gen_units()
    extra = ["-Xptxas", "-v"] if ptxas_verbose else []
    jobs = jobs or max(1, os.cpu_count() or 1)
    objs = []
    with cf.ThreadPoolExecutor(jobs) as ex:
        futs = []
        for u in units:
            obj = os.path.join(BUILD, os.path.basename(u).replace(".cu", ".o"))
            stamp = _unit_digest(u) + ("v" if ptxas_verbose else "")
            futs.append(ex.submit(_compile, u, obj, extra, stamp))
        for f in futs:
            objs.append(f.result())
    tmp = LIB + ".tmp"
    cmd = [_nvcc(), *ARCH, "-shared", "-o", tmp, *objs, "-cudart", "static",
           "-Xlinker", "--exclude-libs,ALL"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, LIB)
    build_cli()
    if not quiet:
        print(f"built {LIB} from {len(objs)} units, and the ssai-* programs in {BIN}")
    return LIB


BIN = os.path.join(HERE, "bin")
CLI = {"ssai-2dstencil": "ssai_2dstencil.cpp", "ssai-2dconv": "ssai_2dconv.cpp",
       "ssai-3dstencil": "ssai_3dstencil.cpp"}


def build_cli() -> None:
    """The reference-spelling command-line drop-ins (host C++ over the C ABI),
    linked against the library with an rpath to it."""
    os.makedirs(BIN, exist_ok=True)
    inc = os.path.join(os.path.dirname(HERE), "include")
    for exe, src in CLI.items():
        src = os.path.join(HERE, "cli", src)
        out = os.path.join(BIN, exe)
        if (os.path.exists(out) and os.path.getmtime(out) >= os.path.getmtime(src)
                and os.path.getmtime(out) >= os.path.getmtime(LIB)
                and all(os.path.getmtime(out) >= os.path.getmtime(os.path.join(HERE, "cli", h))
                        for h in ("ssai_cli.h", "ref_tables.h"))):
            continue
        cmd = [_nvcc(), "-O2", "-std=c++17", "-Xcompiler", "-fopenmp", "-I", inc, src, "-o",
               out, "-L", HERE, "-lssam_b200", "-lgomp", "-Xlinker", "-rpath,$ORIGIN/.."]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"building {exe} failed:\n{r.stdout}\n{r.stderr}")


def main(argv=None) -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("-j", "--jobs", type=int, default=None)
    ap.add_argument("--ptxas-verbose", action="store_true")
    a = ap.parse_args(argv)
    build(a.jobs, a.ptxas_verbose, quiet=False)


if __name__ == "__main__":
    sys.exit(main())
