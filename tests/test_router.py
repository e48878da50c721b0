"""Router-level parity: pcbroute's own router objects linked with the oracle back end (oracle/_ref/pcbroute_oracle),
with the B200 back end (oracle/_ref/pcbroute_b200) and with none (oracle/_ref/pcbroute), built by oracle/Makefile.

Contract:
 (i)  with no search crossing --gpu-pops, sessions are byte-identical to the unmodified reference router;
 (ii) with the back end engaged (--gpu-pops 1), sessions and --eval results are byte-identical between the oracle
      router and the B200 router, at any -mt.
"""
import importlib.util
import os
import re
import subprocess
import tempfile

import pytest

from pcbroute_b200 import dsngen

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_BIN = os.path.join(ROOT, "oracle", "_ref")
REF_SRC = os.environ.get("PCBROUTE_SRC", "/root/reference")


def _bin(name):
    p = os.path.join(REF_BIN, name)
    if not os.path.exists(p):
        if os.path.isdir(os.path.join(REF_SRC, "src")):
            subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), f"REF={REF_SRC}", "-j8"], check=True,
                           capture_output=True)
        else:
            pytest.skip(f"{p} not built (needs the pcbroute sources)")
    return p


def route(binary, board, *args):
    """Route `board` (DSN text); returns (stderr, session text, --eval stdout)."""
    with tempfile.TemporaryDirectory() as d:
        p, s = os.path.join(d, "b.dsn"), os.path.join(d, "b.ses")
        with open(p, "w") as f:
            f.write(board)
        r = subprocess.run([binary, "-de", p, "-do", s, *args], capture_output=True, text=True, timeout=600)
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
    path = os.path.join(REF_SRC, "tests", "test_gpu_gate.py")
    if not os.path.exists(path):
        pytest.skip("pcbroute tests not present on this machine")
    spec = importlib.util.spec_from_file_location("ref_gpu_gate", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    err, _, _ = route(_bin("pcbroute_oracle"), mod.BOARD, "-mt", "1", "-v", "--gpu-pops", "1")
    assert "0 unrouted" in err, err
    assert _gpu_count(err) > 0
    err0, _, _ = route(_bin("pcbroute_oracle"), mod.BOARD, "-mt", "1", "-v", "--gpu-pops", "0")
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
@pytest.mark.parametrize("cfg,seed", BOARDS)
def test_b200_router_sessions_match_the_oracle_router(cfg, seed):
    """(ii): the same session bytes and --eval line with the oracle and the B200 back end, engaged on every search."""
    board = dsngen.generate(cfg, seed)
    o = route(_bin("pcbroute_oracle"), board, "-mt", "1", "-v", "--gpu-pops", "1")
    g = route(_bin("pcbroute_b200"), board, "-mt", "1", "-v", "--gpu-pops", "1")
    assert _gpu_count(g[0]) > 0, g[0][-2000:]
    assert _gpu_count(g[0]) == _gpu_count(o[0])
    assert o[1] and g[1] == o[1]
    assert g[2] == o[2]
    g4 = route(_bin("pcbroute_b200"), board, "-mt", "4", "-v", "--gpu-pops", "1")
    assert g4[1] == o[1] and g4[2] == o[2]
