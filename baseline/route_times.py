"""Router-level timing: the `route s` of pcbroute's summary line (src/main.cpp:303-307) on seeded boards, for

  cpu       the unmodified reference router on the host cores (-mt all; -mt 1 with --cpu1)
  refgpu    the reference router with its own CUDA back end (src/gpu.cu built for sm_100a): the plain GPU back end
  b200      the reference router linked with this repository's back end (libpcbgpu.so), unmodified
  b200x     the router with the back end's hooks (baseline/patch_router.py): cost grids mirrored in HBM, the
            router's own (plain) speculation
  learned   b200x with the learned speculation scheduler (PCBG_SCHED=learned), trained first on the conflict logs
            of b200x runs in log mode over the --train boards

GPU arms search on the back end past the first pop (--gpu-pops 1). Every run prints one JSON line: route seconds,
rounds, unrouted and violation counts, searches finished on the GPU, commits and rejected (wasted) speculative
searches of the negotiation rounds, the --eval line and a digest of the session bytes. The sessions of b200, b200x and
learned must be byte-identical (their searches are exact and the commit order is the router's).

    python baseline/route_times.py --boards c2:1 --arms cpu,refgpu,b200,b200x,learned --train c2:11,c2:12
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
ITER = re.compile(r"iteration +\d+: (\d+) commits, (\d+) rejected")


def run(binary, dsn, args, timeout, env=None):
    e = dict(os.environ)
    for k in ("PCBG_SCHED", "PCBG_SCHED_LOG", "PCBG_SCHED_MODEL", "PCBG_MIRROR", "PCBG_FAIL_SOLVE"):
        e.pop(k, None)
    e.update(env or {})
    with tempfile.TemporaryDirectory() as d:
        ses = os.path.join(d, "b.ses")
        try:
            r = subprocess.run([os.path.join(BIN, binary), "-de", dsn, "-do", ses, "-v", *args], capture_output=True,
                               text=True, timeout=timeout, env=e)
        except subprocess.TimeoutExpired:
            return {"rc": None, "route_s": None, "timeout_s": timeout}
        data = open(ses, "rb").read() if os.path.exists(ses) else b""
        ev = subprocess.run([os.path.join(BIN, binary), "-de", dsn, "--eval", ses], capture_output=True, text=True,
                            timeout=timeout, env=e).stdout.strip() if data else ""
    m = SUMMARY.search(r.stderr)
    g = ON_GPU.search(r.stderr)
    it = [(int(a), int(b)) for a, b in ITER.findall(r.stderr)]
    commits, rejected = sum(a for a, _ in it), sum(b for _, b in it)
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
        "commits": commits,
        "rejected": rejected,
        "wasted_fraction": round(rejected / (commits + rejected), 4) if commits + rejected else None,
        "ses_sha256": hashlib.sha256(data).hexdigest()[:16] if data else None,
        "eval": ev.splitlines()[-1] if ev else None,
        "tail": None if m else r.stderr[-600:],
    }


def board_file(d, spec):
    cfg, seed = spec.split(":")
    path = os.path.join(d, f"{cfg}_{seed}.dsn")
    if not os.path.exists(path):
        with open(path, "w") as f:
            f.write(dsngen.generate(cfg, int(seed)))
    return path


def train(d, specs, mt, timeout, extra, emit):
    """Conflict logs of b200x runs in log mode over the training boards, then the predictor fitted on the GPU."""
    from pcbroute_b200 import sched
    logs = []
    for spec in specs:
        log = os.path.join(d, f"log_{spec.replace(':', '_')}.bin")
        args = ["-mt", str(mt), "--gpu-slots", str(mt), "--gpu-pops", "1", *extra]
        res = run("pcbroute_b200x", board_file(d, spec), args, timeout, {"PCBG_SCHED": "log", "PCBG_SCHED_LOG": log})
        emit({"train_board": spec, "arm": "b200x log", "args": " ".join(args), **res})
        if os.path.exists(log):
            logs.append(log)
    model = os.path.join(d, "model.bin")
    info = sched.train_router_model(logs, model)
    return model, info


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--boards", default="c1:1,c2:1")
    ap.add_argument("--arms", default="cpu,refgpu,b200")
    ap.add_argument("--train", default="", help="boards whose b200x conflict logs train the learned arm")
    ap.add_argument("--model", default=None, help="a trained model instead of --train")
    ap.add_argument("--threshold", default="0.5")
    ap.add_argument("--mt", type=int, default=0, help="threads (default: all host cores)")
    ap.add_argument("--cpu1", action="store_true", help="also run the CPU router at -mt 1")
    ap.add_argument("--timeout", type=int, default=1800)
    ap.add_argument("--out", default=None, help="also write the JSON lines here")
    ap.add_argument("--router-args", default="", help="options given to every run, e.g. \"-it 2 --ripups 0\"")
    a = ap.parse_args()
    cores = os.cpu_count() or 1
    mt = a.mt or cores
    arms = a.arms.split(",")
    extra = a.router_args.split()
    out = open(a.out, "a") if a.out else None

    def emit(line):
        print(json.dumps(line), flush=True)
        if out:
            out.write(json.dumps(line) + "\n")
            out.flush()

    with tempfile.TemporaryDirectory() as d:
        model = a.model
        if "learned" in arms and not model:
            model, info = train(d, [s for s in a.train.split(",") if s], mt, a.timeout, extra, emit)
            emit({"trained": info, "boards": a.train})
        plan = []
        if "cpu" in arms:
            if a.cpu1:
                plan.append(("cpu", "pcbroute_cpu", ["-mt", "1"], None))
            plan.append(("cpu", "pcbroute_cpu", ["-mt", str(mt)], None))
        if "refgpu" in arms:
            plan.append(("refgpu", "pcbroute_refgpu", ["-mt", str(mt), "--gpu-slots", str(mt), "--gpu-pops", "1"], None))
        if "b200" in arms:
            plan.append(("b200", "pcbroute_b200", ["-mt", str(mt), "--gpu-slots", str(mt), "--gpu-pops", "1"], None))
        if "b200x" in arms:
            plan.append(("b200x", "pcbroute_b200x", ["-mt", str(mt), "--gpu-slots", str(mt), "--gpu-pops", "1"], None))
        if "learned" in arms:
            plan.append(("learned", "pcbroute_b200x", ["-mt", str(mt), "--gpu-slots", str(mt), "--gpu-pops", "1"],
                         {"PCBG_SCHED": "learned", "PCBG_SCHED_MODEL": model, "PCBG_SCHED_THRESHOLD": a.threshold}))
        for spec in a.boards.split(","):
            dsn = board_file(d, spec)
            for arm, binary, args, env in plan:
                args = args + extra
                res = run(binary, dsn, args, a.timeout, env)
                emit({"board": spec, "arm": arm, "args": " ".join(args), "cores": cores, **res})


if __name__ == "__main__":
    main()
