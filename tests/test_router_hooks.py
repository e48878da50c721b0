"""The router built with the back end's hooks (baseline/_ref/pcbroute_b200x: baseline/patch_router.py adds the calls
of baseline/router_hooks.h to pcbroute's own src/router.cpp).

  * Cost grids mirrored in HBM: every search reads its rectangle from the device copy the hooks keep current, and
    the sessions and --eval lines are byte-identical to the oracle router's (oracle/_ref/pcbroute_oracle).
  * Learned speculation: conflict logs written in log mode train the predictor on the GPU; with it deciding which
    nets are searched ahead of the commit point, the sessions are still byte-identical, and it defers searches.
"""
import os
import tempfile

import numpy as np
import pytest

from pcbroute_b200 import dsngen, sched
from tests.test_router import _bin, _gpu_count, route

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BX = os.path.join(ROOT, "baseline", "_ref", "pcbroute_b200x")


def _bx():
    if not os.path.exists(BX):
        pytest.skip("baseline/_ref/pcbroute_b200x not built (needs the pcbroute sources at build time)")
    return BX


@pytest.mark.parametrize("cfg,seed", [("t1", 1), ("t2", 1), ("c1", 1)])
def test_mirrored_grids_give_the_oracle_routers_sessions(cfg, seed):
    board = dsngen.generate(cfg, seed)
    o = route(_bin("pcbroute_oracle"), board, "-mt", "1", "-v", "--gpu-pops", "1")
    x = route(_bx(), board, "-mt", "1", "-v", "--gpu-pops", "1")
    assert _gpu_count(x[0]) > 0, x[0][-1500:]
    assert o[1] and x[1] == o[1] and x[2] == o[2]
    x16 = route(_bx(), board, "-mt", "16", "--gpu-slots", "16", "-v", "--gpu-pops", "1")
    assert x16[1] == o[1] and x16[2] == o[2]


def test_learned_speculation_keeps_the_session():
    """Log mode on two training boards, the predictor trained on their pairs, then the learned router on a board
    it did not see: the same bytes as the oracle router and as the hooked router without the scheduler."""
    with tempfile.TemporaryDirectory() as d:
        logs = []
        for seed in (21, 22):
            log = os.path.join(d, f"log{seed}.bin")
            r = route(_bx(), dsngen.generate("t2", seed), "-mt", "16", "--gpu-slots", "16", "-v", "--gpu-pops", "1",
                      env={"PCBG_SCHED": "log", "PCBG_SCHED_LOG": log})
            assert r[1]
            if os.path.exists(log):
                logs.append(log)
        assert logs, "no conflict log was written"
        x, y = sched.read_router_log(logs[0])
        assert x.shape[1] == sched.FEATURES and len(x) == len(y) and len(y) > 0
        model = os.path.join(d, "model.bin")
        info = sched.train_router_model(logs, model, epochs=4)
        assert info["pairs"] > 0 and np.isfinite(info["loss"])
        board = dsngen.generate("c1", 1)
        o = route(_bin("pcbroute_oracle"), board, "-mt", "1", "-v", "--gpu-pops", "1")
        for thr in ("0.5", "0.05"):
            g = route(_bx(), board, "-mt", "16", "--gpu-slots", "16", "-v", "--gpu-pops", "1",
                      env={"PCBG_SCHED": "learned", "PCBG_SCHED_MODEL": model, "PCBG_SCHED_THRESHOLD": thr})
            assert g[1] == o[1] and g[2] == o[2], thr
