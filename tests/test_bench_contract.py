"""bench.py keeps its one-JSON-line contract in every mode, at small sizes:
the reference arm on the host cores (CPU), and on the GPU the headline line,
the MATVEC-only and bounded-solve modes and the batch line."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BASE = {"metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
        "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config"}


def _run(*args, timeout=900):
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args],
                         capture_output=True, text=True, timeout=timeout, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.strip().splitlines() if ln.strip()]
    assert len(lines) == 1, out.stdout[-2000:]          # one JSON line, nothing else
    return json.loads(lines[0])


def test_reference_arm_contract():
    d = _run("--impl", "reference", "--n", "41", "--steps", "1", "--warmup", "0")
    assert BASE <= set(d) and d["impl"] == "reference"
    assert d["value"] > 0 and d["unit"] == "solves/s"
    assert d["cpu_baseline"]["cores"] >= 1 and d["cpu_baseline"]["kind"] in ("port", "reference")
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["value"] == d["value"]


@pytest.mark.gpu
def test_headline_contract_small():
    d = _run("--n", "101", "--steps", "2", "--warmup", "3", "--no-cpu-baseline",
             "--no-large-matvec", "--no-extras")
    assert BASE <= set(d)
    for k in ("roofline", "e2e", "gpu_launches", "clocks", "error", "matvec", "matvec32",
              "cg_iterations_per_s", "time_to_solution_ms"):
        assert k in d, k
    r = d["roofline"]
    assert r["bound"] == "hbm" and r["achieved"] > 0 and r["peak"] > 0 and r["unit"] == "GB/s"
    assert d["e2e"]["h2d_bytes_per_step"] > 0 and d["e2e"]["d2h_bytes_per_step"] > 0
    assert d["gpu_launches"] > 0 and d["relres"]["mixed"] <= 1e-8
    assert d["e2e_fp64"]["value"] > 0 and d["config2"] is None and d["batch256"] is None
    t = d["error"]["vs_tight_fp64"]
    assert t["tight_relres"] <= 1e-13 and t["mixed"] > 0 and t["fp64"] > 0


@pytest.mark.gpu
def test_matvec_and_mixedcap_contracts():
    d = _run("--workload", "matvec", "--n", "201", "--steps", "3", "--warmup", "2")
    assert BASE <= set(d) and d["unit"] == "GB/s" and d["matvec32"]["gbs"] > 0
    d = _run("--workload", "mixedcap", "--n", "201", "--max-inner", "40", "--steps", "1",
             "--warmup", "1")
    assert BASE <= set(d) and d["inner_iterations"] == 40 and d["higher_is_better"] is False


@pytest.mark.gpu
def test_batch_contract_shape():
    d = _run("--workload", "batch256", "--batch-shape", "8,1024", "--steps", "1", "--warmup", "1",
             timeout=1800)
    assert BASE <= set(d) and d["converged"] == 256
    assert d["roofline"]["frac"] > 0 and d["config"]["nodes_per_thread"] == 8


@pytest.mark.gpu
def test_fp64_and_capped_batch_contracts():
    """The binary64-only line (with a NITMAX cap, the profiling form) and the
    batch line stopped after a few inner iterations."""
    d = _run("--workload", "fp64", "--n", "101", "--steps", "2", "--warmup", "1")
    assert BASE <= set(d) and d["unit"] == "ms" and d["higher_is_better"] is False
    assert d["relres"] <= 1e-8 and d["roofline"]["kernel"] == "k_cg64"
    d = _run("--workload", "fp64", "--n", "101", "--nitmax", "20", "--steps", "1", "--warmup", "1")
    assert d["iterations"] == 20 and d["relres"] > 1e-8
    d = _run("--workload", "batch256", "--batch-shape", "4,1024", "--batch-max-inner", "40",
             "--steps", "1", "--warmup", "1", timeout=1800)
    assert d["max_inner"] == 40 and d["iterations_rank0"]["max"] == 40
    assert d["converged"] < 256
