"""Where a router search's time goes on the B200 back end: pcbroute's router run with PCBG_TIMES=1, which prints one
line per search (window, rectangle, preparation, batch wait and size, relaxation, field download, total), summed
and averaged per build. The unmodified build packs each rectangle from host memory; the hooked build copies it from
the cost grids mirrored in HBM.

    python baseline/search_times.py --board c2:1 --router-args "-it 1 --ripups 0 --rescue 0"
"""
import argparse
import json
import os
import re
import subprocess
import sys
import tempfile

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
BIN = os.path.join(ROOT, "baseline", "_ref")

from pcbroute_b200 import dsngen  # noqa: E402

LINE = re.compile(r"pcbg: window (\d+)x(\d+)x(\d+) rect (\d+)x(\d+) \((\d+) tries\) prep ([\d.]+) ms, batch ([\d.]+) ms "
                  r"\((\d+) searches, relax ([\d.]+) ms\), field ([\d.]+) ms, total ([\d.]+) ms")
ROUTE = re.compile(r"route ([\d.]+) s")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--board", default="c2:1")
    ap.add_argument("--router-args", default="")
    ap.add_argument("--mt", type=int, default=0)
    ap.add_argument("--timeout", type=int, default=1800)
    a = ap.parse_args()
    mt = a.mt or os.cpu_count() or 1
    cfg, seed = a.board.split(":")
    with tempfile.TemporaryDirectory() as d:
        dsn = os.path.join(d, "b.dsn")
        with open(dsn, "w") as f:
            f.write(dsngen.generate(cfg, int(seed)))
        for name, binary in (("b200", "pcbroute_b200"), ("b200x", "pcbroute_b200x")):
            env = dict(os.environ, PCBG_TIMES="1")
            env.pop("PCBG_SCHED", None)
            r = subprocess.run([os.path.join(BIN, binary), "-de", dsn, "-do", os.path.join(d, "b.ses"), "-mt", str(mt),
                                "--gpu-slots", str(mt), "--gpu-pops", "1", *a.router_args.split()],
                               capture_output=True, text=True, timeout=a.timeout, env=env)
            rows = [tuple(float(x) for x in m.groups()) for m in LINE.finditer(r.stderr)]
            n = len(rows)
            if not n:
                print(json.dumps({"build": name, "rc": r.returncode, "tail": r.stderr[-500:]}))
                continue

            def mean(i):
                return round(sum(x[i] for x in rows) / n, 3)

            m = ROUTE.search(r.stderr)
            print(json.dumps({
                "build": name, "board": a.board, "args": a.router_args, "searches": n,
                "route_s": float(m.group(1)) if m else None,
                "mean_states": round(sum(x[3] * x[4] * x[2] for x in rows) / n),
                "prep_ms": mean(6), "batch_ms": mean(7), "batch_searches": mean(8), "relax_ms": mean(9),
                "field_ms": mean(10), "total_ms": mean(11),
            }), flush=True)


if __name__ == "__main__":
    main()
