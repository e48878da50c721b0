"""bench.py's reference arm on the CPU: the JSON line the contract asks for, on a small sample.

The reference arm times the exact CPU Dijkstra (the oracle port, with the device solve's early exit) on the host
cores and prints one line with the GPU arm's metric, unit and workload configuration. Run here on the first 8
searches of the workload, as one process and as two ranks under torchrun (rank 0 alone prints; the other rank exits
0 without work). CPU only.
"""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _lines(out):
    return [json.loads(x) for x in out.splitlines() if x.startswith("{")]


def _check(line, steps, warmup):
    assert line["impl"] == "reference"
    assert line["unit"] == "Gcell-relax/s" and line["higher_is_better"] is True
    assert line["value"] > 0 and line["ms_per_step"] > 0
    assert line["steps"] == steps and line["warmup"] == warmup
    assert line["config"]["searches"] == 8 and line["config"]["seed"] and line["config"]["workload"]
    cb = line["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == line["value"] and "8 searches" in cb["sample"]
    e2e = line["e2e"]
    assert e2e["value"] == line["value"] and e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0
    rs = line["reported_states"]
    assert 0 < rs["value"] <= line["value"] and rs["states_per_step"] > 0


def _env():
    e = dict(os.environ)
    e["CUDA_VISIBLE_DEVICES"] = ""
    return e


def test_reference_arm_prints_the_contract_line():
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "2", "--warmup", "1",
                        "--searches", "8"], cwd=ROOT, capture_output=True, text=True, timeout=600, env=_env())
    assert r.returncode == 0, r.stderr[-2000:]
    lines = _lines(r.stdout)
    assert len(lines) == 1, r.stdout[-2000:]
    _check(lines[0], 2, 1)
    # the metric is the GPU arm's (bench.py's METRIC), so the driver can compare the two lines
    sys.path.insert(0, ROOT)
    import bench
    assert lines[0]["metric"] == bench.METRIC
    assert lines[0]["config"] == bench.config_of(type("A", (), {"searches": 8, "wave": 512})())


def test_reference_arm_under_two_ranks_prints_once():
    r = subprocess.run([sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
                        "--master-addr", "127.0.0.1", "--master-port", "29541", "bench.py", "--impl", "reference",
                        "--gpus", "2", "--steps", "1", "--warmup", "0", "--searches", "8"],
                       cwd=ROOT, capture_output=True, text=True, timeout=600, env=_env())
    assert r.returncode == 0, r.stderr[-2000:]
    lines = _lines(r.stdout)
    assert len(lines) == 1, r.stdout[-2000:]
    _check(lines[0], 1, 0)
    assert lines[0]["n_gpus"] == 2


def test_peak_bandwidth_file_forms(tmp_path):
    sys.path.insert(0, ROOT)
    import bench
    f = tmp_path / "peaks.json"
    assert bench.peaks(str(tmp_path / "absent.json")) == (6650.0, "fallback")
    f.write_text(json.dumps({"hbm_gbs": 6553.3, "bf16_tflops": 1590}))
    assert bench.peaks(str(f)) == (6553.3, "measured")
    f.write_text(json.dumps({"hbm_gbs": {"burst": 7001.5, "sustained": 6800}}))
    assert bench.peaks(str(f)) == (7001.5, "measured")
    for bad in ("{", json.dumps({"bf16_tflops": 1590}), json.dumps([1, 2]), json.dumps({"hbm_gbs": "n/a"})):
        f.write_text(bad)
        assert bench.peaks(str(f)) == (6650.0, "fallback"), bad
