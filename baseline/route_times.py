"""Router-level timing: the `route s` of pcbroute's summary line (src/main.cpp:303-307) on seeded boards, for

  cpu      the unmodified reference router on the host cores (-mt 1 and -mt all)
  refgpu   the reference router with its own CUDA back end (src/gpu.cu built for sm_100a): the plain GPU back end
  b200     the reference router linked with this repository's back end (libpcbgpu.so)

both GPU builds engaged on every search past its first pop (--gpu-pops 1) and at the reference default (300000).
The binaries come from baseline/Makefile. For each run the script prints one JSON line: route seconds, rounds,
unrouted and violation counts, the searches finished on the GPU, and a digest of the session bytes (the session of
the b200 build must not depend on -mt).

    python baseline/route_times.py [--boards c1:1,c2:1] [--arms cpu,refgpu,b200] [--out DIR]
"""
import argparse
import hashlib
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

SUMMARY = re.compile(r"(\d+) nets, (\d+) connections, (\d+) unrouted, (\d+) rounds, (\d+) violations, "
                     r"setup ([\d.]+) s, route ([\d.]+) s, total ([\d.]+) s")
ON_GPU = re.compile(r"(\d+) searches finished on the GPU")


def run(binary, dsn, args, timeout):
    with tempfile.TemporaryDirectory() as d:
        ses = os.path.join(d, "b.ses")
        r = subprocess.run([os.path.join(BIN, binary), "-de", dsn, "-do", ses, "-v", *args], capture_output=True,
                           text=True, timeout=timeout)
        data = open(ses, "rb").read() if os.path.exists(ses) else b""
        ev = subprocess.run([os.path.join(BIN, binary), "-de", dsn, "--eval", ses], capture_output=True, text=True,
                            timeout=timeout).stdout.strip() if data else ""
    m = SUMMARY.search(r.stderr)
    g = ON_GPU.search(r.stderr)
    return {
        "rc": r.returncode,
        "route_s": float(m.group(7)) if m else None,
        "total_s": float(m.group(8)) if m else None,
        "nets": int(m.group(1)) if m else None,
        "connections": int(m.group(2)) if m else None,
        "unrouted": int(m.group(3)) if m else None,
        "rounds": int(m.group(4)) if m else None,
        "violations": int(m.group(5)) if m else None,
        "gpu_searches": int(g.group(1)) if g else 0,
        "ses_sha256": hashlib.sha256(data).hexdigest()[:16] if data else None,
        "eval": ev.splitlines()[-1] if ev else None,
        "tail": None if m else r.stderr[-600:],
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--boards", default="c1:1,c2:1")
    ap.add_argument("--arms", default="cpu,refgpu,b200")
    ap.add_argument("--timeout", type=int, default=1200)
    ap.add_argument("--out", default=None, help="also write the JSON lines here")
    a = ap.parse_args()
    cores = os.cpu_count() or 1
    arms = a.arms.split(",")
    plan = []
    if "cpu" in arms:
        plan += [("cpu", "pcbroute_cpu", ["-mt", "1"]), ("cpu", "pcbroute_cpu", ["-mt", str(cores)])]
    for arm, binary in (("refgpu", "pcbroute_refgpu"), ("b200", "pcbroute_b200")):
        if arm in arms:
            plan += [(arm, binary, ["-mt", "1", "--gpu-pops", "1"]), (arm, binary, ["-mt", str(cores), "--gpu-pops", "1"]),
                     (arm, binary, ["-mt", str(cores)])]
    out = open(a.out, "w") if a.out else None
    with tempfile.TemporaryDirectory() as d:
        for spec in a.boards.split(","):
            cfg, seed = spec.split(":")
            dsn = os.path.join(d, f"{cfg}_{seed}.dsn")
            with open(dsn, "w") as f:
                f.write(dsngen.generate(cfg, int(seed)))
            for arm, binary, args in plan:
                res = run(binary, dsn, args, a.timeout)
                line = {"board": f"{cfg} seed {seed}", "arm": arm, "args": " ".join(args), "cores": cores, **res}
                print(json.dumps(line), flush=True)
                if out:
                    out.write(json.dumps(line) + "\n")
                    out.flush()


if __name__ == "__main__":
    main()
