"""The router timing script (baseline/route_times.py) on the CPU router, on the small seeded boards.

The CPU arm needs no GPU, so the parsing of the router's summary, iteration and --eval lines, the session digest
and the timeout path are checked here on pcbroute's own CPU router (baseline/_ref/pcbroute_cpu, built from the
pcbroute sources by baseline/Makefile; skipped when it was not built). CPU only.
"""
import importlib.util
import os
import tempfile

import pytest

from pcbroute_b200 import dsngen

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _script():
    if not os.path.exists(os.path.join(ROOT, "baseline", "_ref", "pcbroute_cpu")):
        pytest.skip("baseline/_ref/pcbroute_cpu not built (needs the pcbroute sources at build time)")
    spec = importlib.util.spec_from_file_location("route_times", os.path.join(ROOT, "baseline", "route_times.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


@pytest.mark.parametrize("board", ["t1:1", "t2:1", "c1:1"])
def test_cpu_router_line_is_parsed_and_deterministic_at_one_thread(board):
    m = _script()
    cfg = dsngen.CONFIGS[board.split(":")[0]]
    with tempfile.TemporaryDirectory() as d:
        dsn = m.board_file(d, board)
        a = m.run("pcbroute_cpu", dsn, ["-mt", "1"], 300)
        b = m.run("pcbroute_cpu", dsn, ["-mt", "1"], 300)
    assert a["rc"] == 0 and a["tail"] is None, a
    assert a["nets"] == cfg.nets + len(cfg.planes)
    # the router counts a net's pieces less one: pins whose pads already touch make one piece (adjacent SOIC-8 pads
    # of one net do on these boards), so it may count a few connections fewer than the pins do
    assert 0 <= cfg.connections - a["connections"] <= max(2, cfg.connections // 50), (a["connections"], cfg.connections)
    assert a["route_s"] is not None and a["route_s"] <= a["total_s"]
    assert a["rounds"] >= 1 and a["unrouted"] >= 0 and a["violations"] >= 0
    assert a["gpu_searches"] == 0 and a["commits"] > 0
    assert a["eval"].startswith("eval: ") and f"{a['connections']} connections" in a["eval"]
    # -mt 1 is the reference's deterministic session
    assert a["ses_sha256"] and a["ses_sha256"] == b["ses_sha256"] and a["eval"] == b["eval"]


def test_a_run_past_its_timeout_is_recorded_not_raised():
    m = _script()
    with tempfile.TemporaryDirectory() as d:
        r = m.run("pcbroute_cpu", m.board_file(d, "c2:1"), ["-mt", "1"], 0.05)
    assert r == {"rc": None, "route_s": None, "timeout_s": 0.05}
