"""The benchmark's reference arm and CPU baseline, on the CPU: the JSON line
the reference arm prints, its silence on ranks other than 0, its
`unavailable` lines for paths the reference does not have, and the timed
CPU implementation -- the reference's compiled Convolution<T> / 3D golds
(oracle/_ref) when built, else the oracle's C restatement ("port")."""
import json
import os
import subprocess
import sys

import pytest

import bench
import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def run_bench(*args, env=None, timeout=300):
    e = dict(os.environ)
    e.update(env or {})
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args], cwd=ROOT,
                          env=e, capture_output=True, text=True, timeout=timeout)


def test_reference_arm_line():
    p = run_bench("--impl", "reference", "--steps", "1", "--warmup", "0",
                  "--workload", "star1_f32_4096_copy")
    assert p.returncode == 0, p.stderr[-2000:]
    d = json.loads(p.stdout.strip().splitlines()[-1])
    assert d["impl"] == "reference" and d["metric"] == "GCells/s" and d["unit"] == "GCells/s"
    assert d["value"] > 0 and d["higher_is_better"] is True and d["steps"] == 1
    assert d["config"]["workload"] == "star1_f32_4096_copy"
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["cores"] >= 1 and cb["sample"] and cb["cpu_model"]
    assert cb["kind"] == ("reference" if oracle.have_ref() else "port")
    assert d["e2e"] == {"value": d["value"], "unit": "GCells/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}


def test_reference_arm_is_silent_off_rank_0():
    p = run_bench("--impl", "reference", "--steps", "1", "--warmup", "0",
                  env={"RANK": "1", "WORLD_SIZE": "2"})
    assert p.returncode == 0 and p.stdout.strip() == ""


@pytest.mark.parametrize("workload", ["jacobi128x8_f32_100sweeps", "cnn128x8_forward"])
def test_reference_arm_unavailable_lines(workload):
    p = run_bench("--impl", "reference", "--steps", "1", "--warmup", "0", "--workload", workload)
    assert p.returncode == 0
    d = json.loads(p.stdout.strip().splitlines()[-1])
    assert d["impl"] == "reference" and d["unavailable"]


def test_unknown_workload_is_refused():
    p = run_bench("--workload", "no_such_workload")
    assert p.returncode != 0 and "unknown workload" in p.stderr


SMALL_2D = {"kind": "star", "r": 1, "dtype": "f32", "n": 512, "steps": 1, "boundary": "zero"}
SMALL_3D = {"kind": "3d", "gold": "j3d13pt", "r": 2, "dtype": "f32", "n": 48, "steps": 2,
            "boundary": "copy"}
SMALL_P19 = {"kind": "3d", "gold": "poisson", "r": 1, "dtype": "f32", "n": 48, "steps": 2,
             "boundary": "copy"}


@pytest.mark.parametrize("spec", [SMALL_2D, SMALL_3D, SMALL_P19], ids=["2d", "3d13", "p19"])
@pytest.mark.parametrize("built", [True, False], ids=["ref", "port"])
def test_cpu_rate_reference_or_port(monkeypatch, spec, built):
    if built and not oracle.have_ref():
        pytest.skip("oracle/_ref is not built (no reference tree at build time)")
    monkeypatch.setattr(oracle, "have_ref", lambda: built)
    bench._CPU_PROBE.clear()
    rate, sample, cores, kind = bench.cpu_reference_rate(dict(spec), budget_s=0.2)
    assert rate > 0 and cores >= 1 and sample
    assert kind == ("reference" if built else "port")


def test_host_threads_follows_omp_num_threads(monkeypatch):
    monkeypatch.setenv("OMP_NUM_THREADS", "3")
    assert bench.host_threads() == 3
    monkeypatch.delenv("OMP_NUM_THREADS")
    assert bench.host_threads() >= 1


def test_poisson_cpu_baseline_small():
    from ssam_b200.workloads import gaussian_rhs
    cb = bench.poisson_cpu_baseline(gaussian_rhs(1, 16, 5), 1000, budget_s=0.2)
    assert cb["value"] > 0 and cb["unit"] == "s" and cb["kind"] == "port"
    assert cb["cores"] == bench.host_threads() and cb["cpu_model"] and "sweeps" in cb["sample"]
