"""bench.py output contract: one JSON line per run with the keys the
measurement harness reads (metric, value, unit, ..., roofline, cpu_baseline,
e2e, gpu_launches, clocks), for both arms."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BASE_KEYS = {"metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
             "scaling", "vs_baseline", "dtype", "data", "config"}


def _run(args, env=None, timeout=900):
    e = dict(os.environ)
    e.update(env or {})
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py")] + args, cwd=ROOT, env=e,
                       capture_output=True, text=True, timeout=timeout)
    assert r.returncode == 0, r.stderr[-2000:]
    return [ln for ln in r.stdout.splitlines() if ln.strip()]


def _one_json(lines):
    js = [ln for ln in lines if ln.lstrip().startswith("{")]
    assert len(js) == 1, lines
    return json.loads(js[0])


def test_reference_arm_line():
    d = _one_json(_run(["--impl", "reference", "--steps", "1", "--warmup", "0"]))
    assert BASE_KEYS <= set(d), set(d) ^ BASE_KEYS
    assert d["impl"] == "reference"
    assert d["value"] > 0 and d["higher_is_better"] is True and d["n_gpus"] == 1
    assert d["warmup"] >= 3  # the contract's minimum warm-up is enforced
    cb = d["cpu_baseline"]
    assert cb["kind"] in ("reference", "port") and cb["cores"] >= 1 and cb["sample"]
    assert cb["value"] == d["value"]
    e2e = d["e2e"]
    assert e2e["value"] == d["value"] and e2e["unit"] == d["unit"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0
    assert d["config"]["workload"].startswith("512^3 ComplexF32")


def test_reference_arm_other_ranks_exit_quietly():
    # under torchrun only rank 0 runs the CPU arm; the others exit 0 with no output
    lines = _run(["--impl", "reference", "--steps", "1", "--warmup", "0"],
                 env={"RANK": "1", "LOCAL_RANK": "1", "WORLD_SIZE": "2"})
    assert not [ln for ln in lines if ln.lstrip().startswith("{")], lines


@pytest.mark.gpu
def test_gpu_arm_line():
    d = _one_json(_run(["--steps", "3", "--warmup", "3"], timeout=1200))
    assert BASE_KEYS <= set(d)
    assert d["unit"] == "GB/s" and d["value"] > 0 and d["scaling"] == "weak"
    rf = d["roofline"]
    assert rf["bound"] == "hbm" and rf["unit"] == "GB/s"
    assert abs(rf["frac"] - rf["achieved"] / rf["peak"]) < 1e-3
    assert rf["traffic"] is None or rf["traffic"] > 0
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["value"] > 0
    e2e = d["e2e"]
    assert e2e["value"] > 0 and e2e["h2d_bytes_per_step"] == e2e["d2h_bytes_per_step"] == 8 * 512 ** 3
    assert e2e["results_consistent"] is True
    assert d["gpu_launches"] == 4 * d["steps"]  # fused slab + dim-3 pass, forward and inverse
    assert "sm_mhz" in d["clocks"] and "reasons" in d["clocks"]
    er = d["errors"]
    assert er["fwd_rel_l2_vs_host_fp64"] <= 1e-5 and er["inv_rel_l2_vs_host_fp64"] <= 1e-5
    assert er["roundtrip_rel_l2"] <= 1e-5
    cf = d["configs"]
    for k in ("c1", "c2", "c4", "c5"):
        assert "error" not in cf[k], cf[k]
    assert cf["c1"]["fwd_rel_l2_vs_host_fp64"] <= 1e-12 and cf["c1"]["roundtrip_rel_l2"] <= 1e-12
    for r in cf["c2"]["results"]:
        tol = 1e-12 if r["precision"] == "Float64" else 1e-5
        assert r["fwd_rel_l2_vs_host_fp64"] <= tol and r["inv_rel_l2_vs_host_fp64"] <= tol
    assert cf["c4"]["grids_worst_fwd_rel_l2_vs_host_fp64"] <= 1e-5
    assert cf["c4"]["dct2_rel_l2_vs_host_fp64"] <= 1e-12 and cf["c4"]["dct3_rel_l2_vs_host_fp64"] <= 1e-12
    assert all(r["completed"] > 0 and r["p99_ms"] > 0 for r in cf["c5"]["rates"])
