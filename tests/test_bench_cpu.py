"""bench.py's contract on CPU: the reference arm's JSON line, the warm-up
rule, and the algorithmic byte model the roofline divides by."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def _run(*args, env=None):
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args], capture_output=True, text=True,
                          timeout=600, env=env)


def test_reference_arm_line_on_a_small_problem():
    r = _run("--impl", "reference", "--n", "16", "--nt", "20", "--steps", "1", "--warmup", "3",
             "--ref-sample-steps", "4")
    assert r.returncode == 0, r.stderr
    lines = [ln for ln in r.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["unit"] == "shots/h" and d["higher_is_better"] is True
    assert d["value"] > 0 and d["cpu_baseline"]["value"] == d["value"]
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"] == {"value": d["value"], "unit": "shots/h", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert d["config"]["grid_phy"] == [16, 16, 16] and d["config"]["nt"] == 20


def test_reference_arm_is_rank_zero_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2")
    r = _run("--impl", "reference", "--gpus", "2", "--n", "16", "--nt", "20", "--steps", "1", "--warmup", "3",
             env=env)
    assert r.returncode == 0 and r.stdout.strip() == ""


def test_fewer_than_three_warmups_refused():
    r = _run("--impl", "reference", "--warmup", "2")
    assert r.returncode != 0 and "--warmup" in r.stderr


@pytest.mark.parametrize("n,pml", [(200, 20), (44, 10)])
def test_byte_model(synth, n, pml):
    s = synth.scaled_cfg2(n, 10, pml=pml)
    # interior kernels: bytes per gridphy cell
    assert bench.kernel_bytes(s, "vel_phy_bwd_image") == 144 * s.n_phy
    assert bench.kernel_bytes(s, "stress_phy_bwd") == 76 * s.n_phy
    # the absorbing-layer kernels touch every updated cell outside gridphy
    N = n + 2 * pml
    shell = (N - 4) ** 3 - n ** 3
    vp = bench.kernel_bytes(s, "vel_pml")
    assert 56 * shell + 24 * shell <= vp <= 56 * shell + 3 * 24 * shell
    # a full-gridext kernel does the work of its interior and absorbing-layer pair
    assert bench.kernel_bytes(s, "stress_fz_rev") == (bench.kernel_bytes(s, "stress_phy_rev")
                                                      + bench.kernel_bytes(s, "stress_pml_sau"))
    assert bench.kernel_bytes(s, "vowr_pack") is None


def test_traffic_read_from_the_committed_profile():
    t = bench.traffic_from_profiles("vel_phy_bwd_image")
    assert t is not None and 1.0e9 < t < 1.5e9
    assert bench.traffic_from_profiles("no_such_kernel") is None


def test_reference_arm_on_a_non_cubic_grid():
    r = _run("--impl", "reference", "--grid", "24", "16", "12", "--nt", "20", "--steps", "1", "--warmup", "3",
             "--ref-sample-steps", "4")
    assert r.returncode == 0, r.stderr
    d = json.loads([ln for ln in r.stdout.splitlines() if ln.strip()][0])
    assert d["config"]["grid_phy"] == [24, 16, 12] and d["config"]["pml"] == 20 and d["value"] > 0


def test_gpus_n_starts_n_ranks_that_shard_the_shots():
    """--gpus 2 without a launcher starts two ranks itself (gloo on CPU with
    --dry-run); each takes its round-robin share of the job's shots and
    rank 0 alone prints one line with the real world size."""
    env = {k: v for k, v in os.environ.items() if k not in ("WORLD_SIZE", "RANK", "LOCAL_RANK")}
    r = _run("--gpus", "2", "--dry-run", "--steps", "3", "--warmup", "3", env=env)
    assert r.returncode == 0, r.stderr
    lines = [ln for ln in r.stdout.splitlines() if ln.strip().startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["n_gpus"] == 2 and d["shots"] == 6
    assert d["shards"] == [[0, 2, 4], [1, 3, 5]]


def test_gpus_and_launcher_world_size_must_agree():
    env = dict(os.environ, WORLD_SIZE="2", RANK="0")
    r = _run("--gpus", "1", "--dry-run", "--steps", "1", "--warmup", "3", env=env)
    assert r.returncode == 2 and "WORLD_SIZE=2" in r.stderr
