"""Router-level parity: pcbroute's own router objects linked with the oracle back end (oracle/_ref/pcbroute_oracle),
with the B200 back end (oracle/_ref/pcbroute_b200) and with none (oracle/_ref/pcbroute), built by oracle/Makefile.

Contract:
 (i)  with no search crossing --gpu-pops, sessions are byte-identical to the unmodified reference router;
 (ii) with the back end engaged (--gpu-pops 1), sessions and --eval results are byte-identical between the oracle
      router and the B200 router, at any -mt.
"""
import os
import re
import subprocess
import tempfile

import pytest

from pcbroute_b200 import dsngen

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_BIN = os.path.join(ROOT, "oracle", "_ref")


def _bin(name):
    """A router binary built by oracle/Makefile (python -c 'import __graft_entry__ as g; g.build()' builds them
    where the pcbroute sources are present; the built files travel with the working tree)."""
    p = os.path.join(REF_BIN, name)
    if not os.path.exists(p):
        pytest.skip(f"{p} not built (needs the pcbroute sources at build time)")
    return p


def route(binary, board, *args, env=None):
    """Route `board` (DSN text); returns (stderr, session text, --eval stdout). env: extra environment variables."""
    e = dict(os.environ)
    for k in ("PCBG_FAIL_SOLVE", "PCBG_MAX_ROUNDS", "PCBG_SCHED", "PCBG_SCHED_LOG", "PCBG_SCHED_MODEL"):
        e.pop(k, None)
    e.update(env or {})
    with tempfile.TemporaryDirectory() as d:
        p, s = os.path.join(d, "b.dsn"), os.path.join(d, "b.ses")
        with open(p, "w") as f:
            f.write(board)
        r = subprocess.run([binary, "-de", p, "-do", s, *args], capture_output=True, text=True, timeout=600,
                           env=e)
        assert r.returncode in (0, 2), r.stderr[-2000:]
        ses = open(s).read() if os.path.exists(s) else ""
        ev = subprocess.run([binary, "-de", p, "--eval", s], capture_output=True, text=True, timeout=600).stdout
        return r.stderr, ses, ev


def _gpu_count(err):
    m = re.search(r"(\d+) searches finished on the GPU", err)
    return int(m.group(1)) if m else 0


BOARDS = [("t1", 1), ("t1", 2), ("t2", 1)]


@pytest.mark.parametrize("cfg,seed", BOARDS)
def test_oracle_backend_idle_is_byte_identical_to_the_reference(cfg, seed):
    """(i): --gpu-pops 0 (and the default, which no search of these boards reaches)."""
    board = dsngen.generate(cfg, seed)
    a = route(_bin("pcbroute"), board, "-mt", "1")
    b = route(_bin("pcbroute_oracle"), board, "-mt", "1", "--gpu-pops", "0")
    c = route(_bin("pcbroute_oracle"), board, "-mt", "1")
    assert a[1] and a[1] == b[1] == c[1]
    assert a[2] == b[2] == c[2]


def test_reference_gpu_gate_checks_pass_with_the_oracle_backend():
    """The reference's own GPU gate test (tests/test_gpu_gate.py:62-68) on its own inline board, with the oracle as
    the back end: with --gpu-pops 1 searches finish on the back end and the board completes; with 0 it is off."""
    # oracle/Makefile extracts the test's inline board when it builds the routers
    path = os.path.join(REF_BIN, "gpu_gate_board.dsn")
    if not os.path.exists(path):
        pytest.skip("the reference's gate-test board was not extracted at build time")
    board = open(path).read()
    err, _, _ = route(_bin("pcbroute_oracle"), board, "-mt", "1", "-v", "--gpu-pops", "1")
    assert "0 unrouted" in err, err
    assert _gpu_count(err) > 0
    err0, _, _ = route(_bin("pcbroute_oracle"), board, "-mt", "1", "-v", "--gpu-pops", "0")
    assert "0 unrouted" in err0 and "on the GPU" not in err0


@pytest.mark.parametrize("cfg,seed", BOARDS[:2])
def test_oracle_backend_engaged_walks_back_every_search(cfg, seed):
    """With --gpu-pops 1 every search past its first pop is finished by the oracle and the router's float walk-back
    accepts every integer field (no chain breaks, src/router.cpp:1654)."""
    err, ses, ev = route(_bin("pcbroute_oracle"), dsngen.generate(cfg, seed), "-mt", "1", "-v", "--gpu-pops", "1")
    assert _gpu_count(err) > 0
    m = re.search(r"(\d+) back on the CPU \((\d+) solve failed, (\d+) chain", err)
    assert m and int(m.group(2)) == 0 and int(m.group(3)) == 0, err[-1500:]
    assert ses and "eval:" in ev


@pytest.mark.gpu
@pytest.mark.parametrize("cfg,seed", BOARDS + [("c1", 1)])
def test_b200_router_sessions_match_the_oracle_router(cfg, seed):
    """(ii): the same session bytes and --eval line with the oracle and the B200 back end, engaged on every search,
    at -mt 1 and with 16 workers (the seeded 50 x 40 mm, 2-layer c1 board included)."""
    board = dsngen.generate(cfg, seed)
    o = route(_bin("pcbroute_oracle"), board, "-mt", "1", "-v", "--gpu-pops", "1")
    g = route(_bin("pcbroute_b200"), board, "-mt", "1", "-v", "--gpu-pops", "1")
    assert _gpu_count(g[0]) > 0, g[0][-2000:]
    assert _gpu_count(g[0]) == _gpu_count(o[0])
    assert o[1] and g[1] == o[1]
    assert g[2] == o[2]
    g16 = route(_bin("pcbroute_b200"), board, "-mt", "16", "--gpu-slots", "16", "-v", "--gpu-pops", "1")
    assert g16[1] == o[1] and g16[2] == o[2]


def _failed(err):
    m = re.search(r"(\d+) back on the CPU \((\d+) solve failed", err)
    return int(m.group(2)) if m else 0


def test_injected_solve_failures_fall_back_deterministically():
    """Host-side fault injection (PCBG_FAIL_SOLVE=k:p fails the k-th search and every p-th after it): the router
    takes its CPU fallback for exactly those searches (src/router.cpp:1598, 1691-1700), completes the board, and
    writes the same session on every run."""
    board = dsngen.generate("t1", 1)
    inj = {"PCBG_FAIL_SOLVE": "2:3"}
    a = route(_bin("pcbroute_oracle"), board, "-mt", "1", "-v", "--gpu-pops", "1", env=inj)
    b = route(_bin("pcbroute_oracle"), board, "-mt", "1", "-v", "--gpu-pops", "1", env=inj)
    assert _failed(a[0]) > 0, a[0][-1500:]
    assert a[1] and a[1] == b[1] and a[2] == b[2]
    assert "eval:" in a[2]


@pytest.mark.gpu
def test_b200_router_with_injected_failures_matches_the_oracle_router():
    """The same injected failures in the B200 back end and in the oracle back end: the same searches fall back to
    the CPU, so the sessions and --eval lines are byte-identical."""
    board = dsngen.generate("t1", 1)
    inj = {"PCBG_FAIL_SOLVE": "2:3"}
    o = route(_bin("pcbroute_oracle"), board, "-mt", "1", "-v", "--gpu-pops", "1", env=inj)
    g = route(_bin("pcbroute_b200"), board, "-mt", "1", "-v", "--gpu-pops", "1", env=inj)
    assert _failed(g[0]) == _failed(o[0]) > 0, g[0][-1500:]
    assert o[1] and g[1] == o[1] and g[2] == o[2]


@pytest.mark.gpu
def test_b200_router_carries_on_when_launches_hit_the_round_cap():
    """PCBG_MAX_ROUNDS=2 makes every relaxation that needs more rounds stop with ERR_ROUNDS; those gpu_solve calls
    return -1 and the router finishes the searches on its CPU A* (src/router.cpp:1598, 1691-1700), the same way on
    every run."""
    board = dsngen.generate("t1", 1)
    env = {"PCBG_MAX_ROUNDS": "2"}
    a = route(_bin("pcbroute_b200"), board, "-mt", "1", "-v", "--gpu-pops", "1", env=env)
    b = route(_bin("pcbroute_b200"), board, "-mt", "1", "-v", "--gpu-pops", "1", env=env)
    assert _failed(a[0]) > 0, a[0][-1500:]
    assert a[1] and a[1] == b[1] and a[2] == b[2]
    assert "eval:" in a[2]
