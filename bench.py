"""Benchmark of the B200 search back end: the batched-search microbenchmark workload.

Workload (seeded, synthetic): 4096 independent single-source single-target searches; window sides log-uniform in
[64, 2048) cells, 2-6 layers, per-(layer, cell) cost 1-16, ~15 % of cells blocked in value-noise blobs, via cost
8-32; about 5.4e9 states in all. They are solved in waves of 512 searches: one step = one wave, solved in one
persistent launch (pcbg_solve_batch). The workload cycles through the 8 waves.

Metric: Gcell-relax/s = 9 x (states of the windows solved) / time. A state has 9 incoming moves (8 in-layer
moves and a via); an exact single-source solve must relax every one of them at least once, so this counts the
problem solved, not the work an algorithm spends on it, and is the same number for the GPU tile solver and a CPU
Dijkstra.

  python bench.py [--gpus N --steps K --warmup W]      # this back end (one JSON line on rank 0)
  python bench.py --impl reference ...                  # the CPU arm (exact Dijkstra on all host cores)

Multi-GPU: one process per GPU (torchrun); each rank solves its own waves (no collective on the data path, weak
scaling); the step time is the max over ranks.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "route s to byte-identical SES: plain GPU vs learned-batched GPU; Gcell-relax/s"
UNIT = "Gcell-relax/s"
SEED = 20261203
WORKLOAD = ("batched-search microbenchmark: 4096 seeded single-source single-target searches, windows log-uniform "
            "64-2048 cells per side, 2-6 layers, cost 1-16 per cell, 15% blocked in value-noise blobs, via cost "
            "8-32; one step = one wave of 512 searches in one persistent launch")
# Algorithmic bytes of the relaxation: 12 per state visit (a 32-bit cost read, a 32-bit distance read and write),
# where a tile visit stages 32 x 32 states of each of its search's layers. The per-solved-state figure counts the
# same 12 bytes once per state of the windows solved.
BYTES_PER_STATE_VISIT = 12
# DRAM bytes moved per algorithmic byte by relax_kernel, from one ncu capture of the 64-search case
# (dram__bytes_read.sum + dram__bytes_write.sum over 12 B per state visit). A full wave is too large to capture; its
# traffic grows with the state visits, so the bench scales this ratio by the launch's algorithmic bytes.
NCU_TRAFFIC_PER_ALG_BYTE = 0.93


def peaks(path=None):
    """HBM copy bandwidth in GB/s and where it comes from: the measured figure of MEASURED_PEAKS.json (a number, or
    an object with a burst / value figure), else the fallback copy bandwidth of 6650 GB/s."""
    p = path or os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            v = json.load(f).get("hbm_gbs")
        if isinstance(v, dict):
            v = v.get("burst", v.get("value"))
        v = float(v)
        if v > 0:
            return v, "measured"
    except (OSError, ValueError, TypeError, AttributeError):
        pass
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms while the timed region runs."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def cost_map_roofline(lib, peak, nx=5000, ny=4000):
    """Device rebuild of the congestion cost maps (rebuild_costs, src/router.cpp:409-420) on a board the size of the
    8-layer stress configuration: 5000 x 4000 cells, 8 layers, 4 net classes. Algorithmic bytes per rebuild: per
    class and layer st 2 + oc 1 + cst 4 per cell; per class vst 2 + 8 ov + vcst 4 per cell; the 8 history planes
    (4 B) once."""
    nl, k = 8, 4
    h = lib.pcbg_costs_create(nx, ny, nl, k)
    if not h:
        return None
    try:
        ms = lib.pcbg_costs_time_rebuild(h, 2.5, 0, 10)
    finally:
        lib.pcbg_costs_destroy(h)
    n = nx * ny
    alg = k * (nl * n * 7 + n * (2 + nl + 4)) + nl * n * 4
    ach = alg / (ms / 1e3) / 1e9
    return {"kernel": "costs_rebuild_kernel", "workload": f"{nx} x {ny} cells, 8 layers, 4 classes",
            "ms": round(ms, 3), "bound": "hbm", "achieved": round(ach, 1), "peak": peak, "unit": "GB/s",
            "frac": round(ach / peak, 4), "algorithmic_bytes": alg}


def plain_gpu_comparison(n=48):
    """The one-search gpu_solve path of pcbroute's own CUDA back end (src/gpu.cu for sm_100a, built unchanged by
    baseline/Makefile) against this library's, on the first n searches of this workload from dense host arrays
    (upload, solve and field download in each timed call). Runs baseline/plain_gpu.py once per arm, each in its own
    process. None when the reference back end has not been built here."""
    if not os.path.exists(os.path.join(ROOT, "baseline", "_ref", "librefgpu.so")):
        return None
    out = {}
    for arm in ("ref", "b200"):
        r = subprocess.run([sys.executable, os.path.join(ROOT, "baseline", "plain_gpu.py"), "--arm", arm,
                            "--searches", str(n)], capture_output=True, text=True, timeout=900)
        if r.returncode != 0:
            return {"error": f"{arm}: " + r.stderr[-300:]}
        out[arm] = json.loads(r.stdout.strip().splitlines()[-1])
    return {"workload": f"first {n} searches of this workload, one gpu_solve call each from host arrays",
            "plain_gpu_gcell_relax_s": out["ref"]["gcell_relax_s"], "b200_gcell_relax_s": out["b200"]["gcell_relax_s"],
            "plain_gpu_seconds": out["ref"]["seconds"], "b200_seconds": out["b200"]["seconds"],
            "speedup_one_search_path": round(out["ref"]["seconds"] / out["b200"]["seconds"], 2)}


def learned_batching():
    """The speculative negotiation rounds on seeded 320 x 256 x 6 boards of 160 nets: the conflict predictor trained
    on the logs of plain rounds over 4 boards, then 3 rip-up-and-reroute iterations on 2 held-out boards with one
    search per launch (sequential), the plain batching (lookahead 16) and the learned batching. Host time of the
    rounds (searches, walk-backs, commits; the faster of 2 runs per board and iteration), the wasted-search
    fraction, and whether all three committed the same paths."""
    from pcbroute_b200 import sched
    kw = dict(nx=320, ny=256, nl=6, nnets=160, margin=12, span=(16, 128))
    r = sched.ab_report(range(100, 104), range(900, 902), kw, iters=3, width=16, epochs=12)
    out = {"workload": "2 held-out seeded boards 320x256x6, 160 two-pin nets, 3 iterations; predictor trained on "
                       "the conflict logs of 4 other boards",
           "identical_paths": r["identical_paths"], "log_pairs": r["log_pairs"], "train_s": r["train_s"]}
    for k in ("sequential", "plain", "learned"):
        out[k] = {x: r[k][x] for x in ("total_ms", "relax_ms", "searches", "wasted", "wasted_fraction", "batches")}
    out["speedup_learned_vs_sequential"] = round(r["sequential"]["total_ms"] / r["learned"]["total_ms"], 3)
    out["speedup_learned_vs_plain"] = round(r["plain"]["total_ms"] / r["learned"]["total_ms"], 3)
    return out


def route_seconds():
    """The router-level figures of the metric's first half (route s, plain GPU against learned-batched GPU), as
    baseline/route_times.py measured them on a B200 and committed them beside the ncu summaries: routing a seeded
    board takes minutes per arm, longer than this benchmark's run, so they are read, not re-measured, and the
    source says where they come from."""
    out = {}
    for board in ("c1", "c2"):
        path = os.path.join(ROOT, "profiles", f"router_route_times_{board}.txt")
        if not os.path.exists(path):
            continue
        arms = {}
        for ln in open(path):
            d = json.loads(ln)
            if "arm" not in d or "board" not in d:
                continue
            arms[d["arm"]] = {"route_s": d["route_s"], "wasted_fraction": d["wasted_fraction"],
                              "gpu_searches": d["gpu_searches"], "ses_sha256": d["ses_sha256"], "args": d["args"],
                              "cores": d["cores"]}
        if arms:
            out[board] = arms
    if not out:
        return None
    out["source"] = ("profiles/router_route_times.md: python baseline/route_times.py --arms cpu,refgpu,b200,b200x,"
                     "learned on one B200 box (16 host cores)")
    return out


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


# ------------------------------------------------------------------------------------------------- CPU baseline

CPU_SAMPLE = 128    # searches of the CPU sample: the first 128 of the workload (197 M states)


def config_of(args):
    """The workload configuration, identical in both arms."""
    return {"workload": WORKLOAD, "searches": args.searches, "wave": args.wave, "seed": SEED}


def cpu_sample(sizes, n):
    """The first n searches of the workload as dense host arrays, generated by numpy (synth.search_arrays, the same
    integer hash as the device generator; no CUDA library is loaded), longest first: the host threads take them in
    that order, so the largest searches start first."""
    from concurrent.futures import ThreadPoolExecutor
    from pcbroute_b200 import synth

    def gen(sz):
        rw, rh, nl, via, sseed = sz
        cf, fl, vcf, src, tgt = synth.search_arrays(sseed, rw, rh, nl, via)
        return dict(fac=synth.microbench_factors(nl), cf=cf, flags=fl, vcf=vcf,
                    start_idx=np.array([src] if src >= 0 else [], np.uint32),
                    start_d=np.zeros(1 if src >= 0 else 0, np.uint64), states=rw * rh * nl)

    with ThreadPoolExecutor(os.cpu_count() or 1) as ex:
        batch = list(ex.map(gen, sizes[:n]))
    batch.sort(key=lambda b: -b["states"])
    return batch


def cpu_solve(batch, threads):
    """One pass of the exact Dijkstra (oracle/pcb_oracle.c, stopping at the best target as the device solve does)
    over the sample on `threads` host threads. Returns (window states, reported states, seconds)."""
    from oracle import oracle
    t0 = time.perf_counter()
    res = oracle.solve_many(batch, threads)
    secs = time.perf_counter() - t0
    return sum(b["states"] for b in batch), sum(r[2] for r in res), secs


def cpu_sample_text(batch, threads):
    return (f"the first {len(batch)} searches of the workload ({sum(b['states'] for b in batch)} window states), "
            f"generated by numpy, largest first; exact Dijkstra (oracle/pcb_oracle.c) stopping at the best target, "
            f"{threads} host threads")


def run_reference(args):
    ws, rank, _ = dist_setup()
    if rank != 0:
        return
    from pcbroute_b200 import synth
    threads = os.cpu_count() or 1
    batch = cpu_sample(synth.microbench_sizes(SEED, args.searches), CPU_SAMPLE)
    for _ in range(args.warmup):
        cpu_solve(batch, threads)
    tot_states = tot_low = 0
    tot_s = 0.0
    for _ in range(args.steps):
        st, low, secs = cpu_solve(batch, threads)
        tot_states += st
        tot_low += low
        tot_s += secs
    v = 9.0 * tot_states / tot_s / 1e9
    line = {
        "impl": "reference", "metric": METRIC, "value": round(v, 4), "unit": UNIT, "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(1e3 * tot_s / args.steps, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int64", "data": "synthetic",
        "config": config_of(args),
        "parallelism": f"{threads} host threads",
        "reported_states": {"value": round(9.0 * tot_low / tot_s / 1e9, 4), "unit": UNIT,
                            "states_per_step": tot_low // args.steps,
                            "definition": "9 x the states at or below each search's best target cost, per second"},
        "cpu_baseline": {"value": round(v, 4), "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": cpu_sample_text(batch, threads) + ", one pass per step"},
        "e2e": {"value": round(v, 4), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------------------------------------- GPU arm

def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=8)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--searches", type=int, default=4096)
    ap.add_argument("--wave", type=int, default=512)
    ap.add_argument("--e2e-waves", type=int, default=2)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cpu-budget", type=float, default=15.0)
    ap.add_argument("--no-spec", action="store_true", help="skip the learned-vs-plain speculative batching A/B")
    ap.add_argument("--no-tune", action="store_true", help="skip the schedule autotuner (untuned rule)")
    ap.add_argument("--band", type=int, default=None,
                    help="relaxation round band (pcbg_set_round_band); default: the library's own")
    ap.add_argument("--order", type=int, default=None, choices=[0, 1, 2],
                    help="visit order of ordered rounds (pcbg_set_visit_order); default: the library's own")
    ap.add_argument("--cost-maps-only", type=int, nargs=2, metavar=("NX", "NY"), default=None,
                    help="only time the cost-map rebuild on an NX x NY x 8 board of 4 classes (a profiling case)")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
        return

    import torch
    import torch.distributed as dist
    from pcbroute_b200 import _lib, replicas, synth

    ws, rank, local = dist_setup()
    torch.cuda.set_device(local)
    if ws > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    lib = _lib.load()
    if args.band is not None:
        lib.pcbg_set_round_band(args.band)
    if args.order is not None:
        lib.pcbg_set_visit_order(args.order)
    if args.cost_maps_only:
        if rank == 0:
            print(json.dumps(cost_map_roofline(lib, peaks()[0], *args.cost_maps_only)))
        return
    if not lib.pcbg_available():
        raise RuntimeError("B200 back end unavailable: " + _lib.last_error())
    stream = torch.cuda.current_stream()
    sp = C.c_void_p(stream.cuda_stream)

    sizes = synth.microbench_sizes(SEED, args.searches)
    waves = [sizes[i:i + args.wave] for i in range(0, len(sizes), args.wave)]
    nw = len(waves)
    my = replicas.my_waves(waves, ws, rank)

    # generate every search of my waves on the device (pitched layout), once
    def make(sz):
        rw, rh, nl, via, sseed = sz
        pitch, hpad = -(-rw // 32) * 32, -(-rh // 32) * 32
        cf = torch.empty(nl * hpad * pitch, dtype=torch.float32, device="cuda")
        fl = torch.empty(nl * hpad * pitch, dtype=torch.uint8, device="cuda")
        vcf = torch.empty(hpad * pitch, dtype=torch.float32, device="cuda")
        st = torch.empty(2, dtype=torch.int64, device="cuda")
        assert lib.pcbg_synth_search(sseed, rw, rh, nl, pitch, hpad, via, cf.data_ptr(), fl.data_ptr(),
                                     vcf.data_ptr(), st.data_ptr(), sp) == 0
        return dict(rw=rw, rh=rh, nl=nl, pitch=pitch, hpad=hpad, cf=cf, fl=fl, vcf=vcf, st=st)

    dev_waves = [[make(sz) for sz in w] for w in my]
    torch.cuda.synchronize()

    # the library's schedule autotuner (round band and kernel build per layer and batch class), before any timing
    tune = None
    if not args.no_tune:
        ents = (_lib.TuneEntry * 8)()
        nt = lib.pcbg_autotune(sp, ents, 8)
        if nt < 0:
            raise RuntimeError("pcbg_autotune failed: " + _lib.last_error())
        tune = [{"layers": f"{e.layers_lo}-{e.layers_hi}", "batch_class": e.batch_class, "band": e.band,
                 "blocks_per_sm": e.blocks_per_sm, "ms": round(e.ms, 3), "ms_untuned": round(e.ms_untuned, 3),
                 "batch": f"{e.searches} x {e.rw}x{e.rh}x{e.nl}"} for e in ents[:nt]]

    def search_array(wave, outs=None):
        arr = (_lib.Search * len(wave))()
        keep = []
        for k, s in enumerate(wave):
            a = arr[k]
            a.rw, a.rh, a.nl, a.pitch, a.hpad = s["rw"], s["rh"], s["nl"], s["pitch"], s["hpad"]
            fac = synth.microbench_factors(s["nl"])
            for l in range(8):
                for m in range(8):
                    a.fac[l][m] = float(fac[l, m])
            a.cf, a.flags, a.vcf = s["cf"].data_ptr(), s["fl"].data_ptr(), s["vcf"].data_ptr()
            si = s["st"][:1].to(torch.int32).clamp_(min=0)
            sd = torch.zeros(1, dtype=torch.int64, device="cuda")
            keep += [si, sd]
            a.start_idx, a.start_d = si.data_ptr(), sd.data_ptr()
            a.n_starts = 1
            a.out = outs[k].data_ptr() if outs is not None else None
        return arr, keep

    def batch_fixed_cost(reps=200):
        """Per-batch fixed cost of pcbg_solve_batch: host time of a call (descriptor staging, copies, clears, the
        seed / relax / report launches, the result copy and its synchronisation) minus the relaxation's device time,
        on a batch of one small search (64 x 64 x 2) and on a router-sized batch (two 1024 x 768 x 4 searches)."""
        res = {}
        for name, szs in (("one 64x64x2 search", [(64, 64, 2, 12.0, 77)]),
                          ("two 1024x768x4 searches", [(1024, 768, 4, 12.0, 78), (1024, 768, 4, 20.0, 79)])):
            w = [make(sz) for sz in szs]
            arr, _keep = search_array(w)
            for _ in range(5):
                lib.pcbg_solve_batch(arr, len(arr), sp)
            torch.cuda.synchronize()
            n = reps if len(szs) == 1 else 20
            wall = relax = 0.0
            for _ in range(n):
                t0 = time.perf_counter()
                if lib.pcbg_solve_batch(arr, len(arr), sp) != 0:
                    raise RuntimeError(_lib.last_error())
                wall += time.perf_counter() - t0
                relax += lib.pcbg_last_batch_kernel_ms() / 1e3
            res[name] = {"calls": n, "wall_us": round(1e6 * wall / n, 1), "relax_us": round(1e6 * relax / n, 1),
                         "fixed_us": round(1e6 * (wall - relax) / n, 1),
                         "fixed_share": round((wall - relax) / wall, 4)}
        return res

    # searches whose source could not be placed are dropped from the wave (none are expected)
    # every step writes its reported fields: one device buffer, the size of the largest wave, that each wave's
    # searches fill (a caller that keeps its fields on the device reuses its buffer the same way)
    field_n = max(sum(sr["rw"] * sr["rh"] * sr["nl"] for sr in w) for w in dev_waves)
    field_buf = torch.empty(field_n, dtype=torch.float32, device="cuda")

    def field_views(w):
        views, o = [], 0
        for sr in w:
            m = sr["rw"] * sr["rh"] * sr["nl"]
            views.append(field_buf[o:o + m])
            o += m
        return views

    arrays = [search_array(w, field_views(w)) for w in dev_waves]
    # and on this run's own first wave (solved 24 times, untimed): its class's schedule for the timed steps
    if not args.no_tune:
        e = _lib.TuneEntry()
        arr0, _ = arrays[0]
        if lib.pcbg_autotune_batch(arr0, len(arr0), sp, C.byref(e)) != 1:
            raise RuntimeError("pcbg_autotune_batch failed: " + _lib.last_error())
        tune.append({"layers": f"{e.layers_lo}-{e.layers_hi}", "batch_class": e.batch_class, "band": e.band,
                     "blocks_per_sm": e.blocks_per_sm, "ms": round(e.ms, 3), "ms_untuned": round(e.ms_untuned, 3),
                     "batch": f"wave 0 of this run ({e.searches} searches, up to {e.nl} layers)"})
    states = [sum(s["rw"] * s["rh"] * s["nl"] for s in w) for w in dev_waves]

    iters = [0, 0, 0, 0]
    busy = [0.0]

    def solve(k):
        arr, _ = arrays[k % len(arrays)]
        rc = lib.pcbg_solve_batch(arr, len(arr), sp)
        if rc != 0:
            raise RuntimeError("pcbg_solve_batch failed: " + _lib.last_error())
        iters[0] += lib.pcbg_last_batch_local_iters()
        iters[1] += lib.pcbg_last_batch_deferred()
        iters[2] += lib.pcbg_last_batch_dropped()
        iters[3] += lib.pcbg_last_batch_settled()
        busy[0] += lib.pcbg_last_batch_busy_frac() * lib.pcbg_last_batch_kernel_ms()
        return (lib.pcbg_last_batch_kernel_ms(), lib.pcbg_last_batch_tile_visits(), lib.pcbg_last_batch_layer_visits(),
                lib.pcbg_last_batch_launches(), lib.pcbg_last_batch_rounds())

    def barrier():
        if ws > 1:
            dist.barrier()

    for k in range(args.warmup):
        solve(k)
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    kms, tv, lv, launches, rounds, st_done = 0.0, 0, 0, 0, 0, 0
    iters[:] = [0, 0, 0, 0]
    busy[0] = 0.0
    with ClockSampler(local) as clk:
        e0.record(stream)
        for k in range(args.steps):
            a, b, c, d, r = solve(k)
            kms += a
            tv += b
            lv += c
            launches += d
            rounds += r
            st_done += states[k % len(states)]
        e1.record(stream)
        torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    ms_max, states_all = replicas.max_time_sum_work(ms, st_done, "cuda", ws)
    value = 9.0 * states_all / (ms_max / 1e3) / 1e9
    settled_max, settled_all = replicas.max_time_sum_work(ms, iters[3], "cuda", ws)
    alg_bytes = BYTES_PER_STATE_VISIT * 1024 * lv
    solved_bytes = BYTES_PER_STATE_VISIT * st_done
    peak, peak_kind = peaks()
    achieved = alg_bytes / (kms / 1e3) / 1e9 if kms > 0 else 0.0
    achieved_solved = solved_bytes / (kms / 1e3) / 1e9 if kms > 0 else 0.0

    # ---- end to end: host (pinned) inputs -> device, solve, reported fields -> host, every step
    e2e = None
    if not args.no_e2e:
        ew_src = dev_waves[:max(1, min(args.e2e_waves, len(dev_waves)))]
        # A caller that keeps a wave's inputs in one pinned blob and its fields in another moves each with one copy:
        # every search's cf / flags / vcf (and its field) is a 256-byte-aligned slice of the wave's blob.
        ew, in_d, in_h, out_d, out_h, e_arrays = [], [], [], [], [], []
        for w in ew_src:
            offs, off = [], 0
            for sr in w:
                n = sr["cf"].numel()
                o_cf = off
                o_fl = o_cf + -(-n * 4 // 256) * 256
                o_vc = o_fl + -(-n // 256) * 256
                off = o_vc + -(-sr["vcf"].numel() * 4 // 256) * 256
                offs.append((o_cf, o_fl, o_vc))
            blob = torch.empty(off, dtype=torch.uint8, device="cuda")
            views = []
            for sr, (o_cf, o_fl, o_vc) in zip(w, offs):
                n, nv = sr["cf"].numel(), sr["vcf"].numel()
                v = dict(sr)
                v["cf"] = blob[o_cf:o_cf + 4 * n].view(torch.float32)
                v["fl"] = blob[o_fl:o_fl + n]
                v["vcf"] = blob[o_vc:o_vc + 4 * nv].view(torch.float32)
                v["cf"].copy_(sr["cf"])
                v["fl"].copy_(sr["fl"])
                v["vcf"].copy_(sr["vcf"])
                views.append(v)
            tot = sum(sr["rw"] * sr["rh"] * sr["nl"] for sr in w)
            od = torch.empty(tot, dtype=torch.float32, device="cuda")
            outs, o = [], 0
            for sr in w:
                m = sr["rw"] * sr["rh"] * sr["nl"]
                outs.append(od[o:o + m])
                o += m
            ew.append(views)
            in_d.append(blob)
            in_h.append(blob.cpu().pin_memory())
            out_d.append(od)
            out_h.append(torch.empty(tot, dtype=torch.float32).pin_memory())
            e_arrays.append(search_array(views, outs))
        h2d = [x.numel() for x in in_h]
        d2h = [x.numel() * 4 for x in out_h]
        e_states = [sum(sr["rw"] * sr["rh"] * sr["nl"] for sr in w) for w in ew]

        # Steps are pipelined the way a caller with two wave buffers would run them: the inputs of step k+1 go up
        # on one copy stream and the fields of step k come down on another while step k+1's launch runs. Every
        # step still moves its own inputs in and its own fields out inside the timed region.
        cs_in, cs_out = torch.cuda.Stream(), torch.cuda.Stream()
        ev_in = [torch.cuda.Event() for _ in ew]
        ev_out = [torch.cuda.Event() for _ in ew]

        def e2e_h2d(k):
            i = k % len(ew)
            with torch.cuda.stream(cs_in):
                in_d[i].copy_(in_h[i], non_blocking=True)
                ev_in[i].record(cs_in)

        def e2e_solve(k):
            i = k % len(ew)
            stream.wait_event(ev_in[i])      # this step's inputs are up
            stream.wait_event(ev_out[i])     # the fields of the wave that used these buffers before are down
            arr, _ = e_arrays[i]
            if lib.pcbg_solve_batch(arr, len(arr), sp) != 0:
                raise RuntimeError("pcbg_solve_batch failed: " + _lib.last_error())
            cs_out.wait_stream(stream)
            with torch.cuda.stream(cs_out):
                out_h[i].copy_(out_d[i], non_blocking=True)
                ev_out[i].record(cs_out)
            return e_states[i], h2d[i], d2h[i]

        def e2e_run(n):
            es = eb_in = eb_out = 0
            cs_in.wait_stream(stream)        # the first upload starts after the timing event
            e2e_h2d(0)
            for k in range(n):
                if k + 1 < n:
                    e2e_h2d(k + 1)
                a, b, c = e2e_solve(k)
                es += a
                eb_in += b
                eb_out += c
            for e in ev_out:
                stream.wait_event(e)
            return es, eb_in, eb_out

        e2e_run(min(args.warmup, 2))
        torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        es, eb_in, eb_out = e2e_run(args.steps)
        f1.record(stream)
        torch.cuda.synchronize()
        barrier()
        et, etot = replicas.max_time_sum_work(f0.elapsed_time(f1), es, "cuda", ws)
        e2e = {"value": round(9.0 * etot / (et / 1e3) / 1e9, 4), "unit": UNIT,
               "h2d_bytes_per_step": int(eb_in // args.steps), "d2h_bytes_per_step": int(eb_out // args.steps),
               "waves": len(ew), "api": "pcbg_solve_batch from pinned host buffers, reported fields read back; one copy each "
                                              "way per wave, overlapping the neighbouring steps' launches on two "
                                              "copy streams"}

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        threads = os.cpu_count() or 1
        batch = cpu_sample(sizes, CPU_SAMPLE)
        cst, clow, csecs = cpu_solve(batch, threads)
        cv = 9.0 * cst / csecs / 1e9
        cpu = {"value": round(cv, 4), "unit": UNIT, "cores": threads, "kind": "port",
               "sample": cpu_sample_text(batch, threads) + f", one pass, {csecs:.1f} s",
               "reported_states_value": round(9.0 * clow / csecs / 1e9, 4)}
        del batch

    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 4), "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms_max / args.steps, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
            "config": config_of(args),
            "parallelism": f"replicas x{ws}",
            "l2": "inputs larger than L2 (several GB per wave)",
            "timed_step": "one pcbg_solve_batch of a resident wave: clears, seeds, the relaxation launch, the report "
                          "kernel writing every search's field to device memory, the results back to the host",
            "reported_states": {"value": round(9.0 * settled_all / (ms_max / 1e3) / 1e9, 4), "unit": UNIT,
                                "states_per_step": int(settled_all // args.steps),
                                "definition": "9 x the states at or below each search's best target cost, per second"},
            "kernel_stats": {"states_per_step": int(states_all / args.steps),
                             "tile_visits_per_step": tv // args.steps, "rounds_per_step": rounds // args.steps,
                             "state_visits_per_state": round(lv * 1024 / max(1, st_done), 3),
                             "local_iters_per_visit": round(iters[0] / max(1, tv), 3),
                             "round_band": int(lib.pcbg_round_band()),
                             "blocks_per_sm": int(lib.pcbg_last_batch_blocks_per_sm()),
                             "visit_order": int(lib.pcbg_visit_order()),
                             "block_time_visiting": round(busy[0] / max(kms, 1e-9), 4),
                             "autotuned_schedules": tune,
                             "tiles_deferred_per_step": iters[1] // args.steps,
                             "tiles_dropped_per_step": iters[2] // args.steps},
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4),
                         "traffic": round(NCU_TRAFFIC_PER_ALG_BYTE * alg_bytes / args.steps / 1e9, 2),
                         "traffic_unit": "GB per launch (ncu ratio of the 64-search case x algorithmic bytes)",
                         "algorithmic_bytes": "12 B per state visit (tile visits x 32 x 32 x the search's layers)",
                         "per_solved_state": {"achieved": round(achieved_solved, 1),
                                              "frac": round(achieved_solved / peak, 4),
                                              "algorithmic_bytes": "12 B per state of the windows solved"},
                         "kernel": "relax_kernel (persistent tile relaxation)",
                         "kernel_ms_per_step": round(kms / args.steps, 3), "peak_kind": peak_kind},
            "gpu_launches": int(launches),
            "batch_fixed_cost": None if args.no_spec else batch_fixed_cost(),
            "clocks": clk.summary(),
            "cost_maps": cost_map_roofline(lib, peak),
            "learned_batching": None if args.no_spec else learned_batching(),
            "plain_gpu": None if args.no_spec else plain_gpu_comparison(),
            "e2e": e2e,
            "cpu_baseline": cpu,
            "route_s": route_seconds(),
        }
        print(json.dumps(line), flush=True)
    if ws > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
