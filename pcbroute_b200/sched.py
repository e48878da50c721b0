"""The learned speculation scheduler (csrc/sched.cu, csrc/mlp.cu): conflict logs from plain speculative rounds,
training on the GPU, and learned batch composition for pcbg_spec rounds."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib, spec

FEATURES, HIDDEN = 2176, 128


class Scheduler:
    def __init__(self, seed: int = 1):
        self.lib = _lib.load()
        self.h = self.lib.pcbg_sched_create(seed)
        if not self.h:
            raise RuntimeError(_lib.last_error())

    # ---- the network on host arrays ----
    def nparams(self) -> int:
        return int(self.lib.pcbg_sched_nparams(self.h))

    def params(self) -> np.ndarray:
        p = np.empty(self.nparams(), np.float32)
        assert self.lib.pcbg_sched_get_params(self.h, p.ctypes.data) == 0
        return p

    def set_params(self, p: np.ndarray) -> None:
        p = np.ascontiguousarray(p, np.float32)
        assert p.size == self.nparams()
        assert self.lib.pcbg_sched_set_params(self.h, p.ctypes.data) == 0

    def forward(self, x_bf16: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x_bf16, np.uint16)
        B = x.shape[0]
        p = np.empty(B, np.float32)
        if self.lib.pcbg_sched_forward_host(self.h, x.ctypes.data, B, p.ctypes.data) != 0:
            raise RuntimeError(_lib.last_error())
        return p

    def grad(self, x_bf16: np.ndarray, y: np.ndarray, w: np.ndarray) -> tuple[np.ndarray, float]:
        x = np.ascontiguousarray(x_bf16, np.uint16)
        y = np.ascontiguousarray(y, np.float32)
        w = np.ascontiguousarray(w, np.float32)
        g = np.empty(self.nparams(), np.float32)
        loss = C.c_float(0)
        if self.lib.pcbg_sched_grad_host(self.h, x.ctypes.data, y.ctypes.data, w.ctypes.data, x.shape[0],
                                         g.ctypes.data, C.byref(loss)) != 0:
            raise RuntimeError(_lib.last_error())
        return g, float(loss.value)

    # ---- logs, training, scheduling ----
    def log_rounds(self, r: "spec.Round") -> None:
        self.lib.pcbg_sched_attach_logger(self.h, r.s)

    def label(self, r: "spec.Round") -> int:
        n = int(self.lib.pcbg_sched_label(self.h, r.s))
        if n < 0:
            raise RuntimeError(_lib.last_error())
        return n

    def log_size(self) -> tuple[int, int]:
        pos = C.c_int64(0)
        n = int(self.lib.pcbg_sched_log_size(self.h, C.byref(pos)))
        return n, int(pos.value)

    def train(self, epochs: int, lr: float = 1e-3, batch: int = 256, seed: int = 7) -> float:
        loss = C.c_float(0)
        if self.lib.pcbg_sched_train(self.h, epochs, lr, batch, seed, C.byref(loss)) != 0:
            raise RuntimeError(_lib.last_error())
        return float(loss.value)

    def attach(self, r: "spec.Round", threshold: float = 0.5) -> None:
        self.lib.pcbg_sched_attach(self.h, r.s, threshold)

    def counts(self) -> tuple[int, int]:
        a, b = C.c_int64(0), C.c_int64(0)
        self.lib.pcbg_sched_counts(self.h, C.byref(a), C.byref(b))
        return int(a.value), int(b.value)

    def close(self):
        if self.h:
            self.lib.pcbg_sched_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def read_router_log(path: str) -> tuple[np.ndarray, np.ndarray]:
    """The labelled pairs a router wrote in log mode (PCBG_SCHED=log, include/pcbg.h): records of an int64 row count,
    rows x FEATURES bf16 bit patterns and rows u8 labels. Returns (x [n, FEATURES] uint16, y [n] float32)."""
    xs, ys = [], []
    with open(path, "rb") as f:
        while True:
            h = f.read(8)
            if len(h) < 8:
                break
            n = int(np.frombuffer(h, np.int64)[0])
            x = np.frombuffer(f.read(n * FEATURES * 2), np.uint16).reshape(n, FEATURES)
            y = np.frombuffer(f.read(n), np.uint8).astype(np.float32)
            xs.append(x)
            ys.append(y)
    if not xs:
        return np.zeros((0, FEATURES), np.uint16), np.zeros(0, np.float32)
    return np.concatenate(xs), np.concatenate(ys)


def train_router_model(log_paths: list[str], out_path: str, epochs: int = 12, lr: float = 1e-3, batch: int = 256,
                       seed: int = 1) -> dict:
    """Fit the conflict predictor on the GPU (the library's own forward / backward kernels and Adam) to the pairs
    routers logged, and write its parameters (float32, pcbg_sched_get_params order) to out_path for
    PCBG_SCHED_MODEL."""
    import time
    xs, ys = zip(*(read_router_log(p) for p in log_paths))
    x = np.ascontiguousarray(np.concatenate(xs))
    y = np.ascontiguousarray(np.concatenate(ys))
    sch = Scheduler(seed)
    if sch.lib.pcbg_sched_add_log_host(sch.h, x.ctypes.data, y.ctypes.data, len(y)) != 0:
        raise RuntimeError(_lib.last_error())
    loss = C.c_float(0)
    t0 = time.perf_counter()
    if sch.lib.pcbg_sched_train(sch.h, epochs, C.c_float(lr), batch, seed, C.byref(loss)) != 0:
        raise RuntimeError(_lib.last_error())
    secs = time.perf_counter() - t0
    sch.params().tofile(out_path)
    return {"pairs": int(len(y)), "positives": int(y.sum()), "epochs": epochs, "loss": float(loss.value),
            "train_s": round(secs, 3)}


def collect_logs(sch: Scheduler, boards: list[dict], iters: int, width: int) -> None:
    """Conflict logs of plain speculative rounds: every board negotiated `iters` iterations, pairs labelled after
    each iteration."""
    for b in boards:
        r = spec.Round(b)
        try:
            sch.log_rounds(r)
            for it in range(iters):
                r.iterate(spec.pres_of(it), spec.PLAIN, width)
                sch.label(r)
                if it + 1 < iters:
                    r.add_history(1.0)
        finally:
            r.close()


def run(b: dict, iters: int, width: int, sch: Scheduler | None = None, threshold: float = 0.5):
    """Negotiate a board with the plain batching (sch None) or the learned one; returns paths and stats."""
    r = spec.Round(b)
    try:
        if sch is not None:
            sch.attach(r, threshold)
        stats = []
        for it in range(iters):
            stats.append(r.iterate(spec.pres_of(it), spec.LEARNED if sch is not None else spec.PLAIN, width))
            if it + 1 < iters:
                r.add_history(1.0)
        return r.paths(), stats
    finally:
        r.close()


def ab_report(train_seeds, test_seeds, board_kw: dict, iters: int = 3, width: int = 16, epochs: int = 12,
              threshold: float = 0.5, seed: int = 21, repeat: int = 2) -> dict:
    """Train on the conflict logs of plain rounds over `train_seeds` boards, then negotiate the `test_seeds` boards
    sequentially (one search per launch), with the plain batching and with the learned one. Returns the totals per
    method (searches, wasted searches, launches, host and device milliseconds) and whether all three committed the
    same paths.

    Each method negotiates each board `repeat` times. The searches, launches and paths are deterministic, so every
    repeat gives the same counts; the milliseconds of an iteration are the lowest over the repeats, which keeps a
    stall of the host thread in one repeat out of the totals."""
    import time
    train = [spec.spec_board(s, **board_kw) for s in train_seeds]
    test = [spec.spec_board(s, **board_kw) for s in test_seeds]
    sch = Scheduler(seed)
    t0 = time.time()
    collect_logs(sch, train, iters=iters, width=width)
    n, pos = sch.log_size()
    t1 = time.time()
    loss = sch.train(epochs=epochs)
    t2 = time.time()
    out = {"train_boards": len(train), "test_boards": len(test), "board": board_kw, "iters": iters, "width": width,
           "log_pairs": n, "log_positives": pos, "train_loss": round(loss, 4), "log_s": round(t1 - t0, 2),
           "train_s": round(t2 - t1, 2), "threshold": threshold}
    ref = {}
    same = True
    for name, pol, s in (("sequential", spec.SEQUENTIAL, None), ("plain", spec.PLAIN, None),
                         ("learned", spec.LEARNED, sch)):
        tot = dict(searches=0, wasted=0, batches=0, total_ms=0.0, search_ms=0.0, relax_ms=0.0)
        for b in test:
            best = [None] * iters
            for rep in range(max(1, repeat)):
                r = spec.Round(b)
                try:
                    if s is not None:
                        s.attach(r, threshold)
                    for it in range(iters):
                        st = r.iterate(spec.pres_of(it), pol, width)
                        if best[it] is None:
                            best[it] = dict(st)
                        else:
                            for k in ("searches", "wasted", "batches"):
                                same &= best[it][k] == st[k]
                            for k in ("total_ms", "search_ms", "relax_ms"):
                                best[it][k] = min(best[it][k], st[k])
                        if it + 1 < iters:
                            r.add_history(1.0)
                    paths = r.paths()
                finally:
                    r.close()
                if name == "sequential" and rep == 0:
                    ref[b["seed"]] = paths
                else:
                    same &= all(np.array_equal(a, c) for a, c in zip(ref[b["seed"]], paths))
            for st in best:
                for k in tot:
                    tot[k] += st[k]
        tot["wasted_fraction"] = round(tot["wasted"] / max(1, tot["searches"]), 4)
        for k in ("total_ms", "search_ms", "relax_ms"):
            tot[k] = round(tot[k], 1)
        out[name] = tot
    out["identical_paths"] = bool(same)
    sch.close()
    return out


def main() -> None:
    import argparse
    import json
    ap = argparse.ArgumentParser(description="learned vs plain speculative batching on seeded boards (A/B)")
    ap.add_argument("--train", type=int, default=8)
    ap.add_argument("--test", type=int, default=4)
    ap.add_argument("--nx", type=int, default=320)
    ap.add_argument("--ny", type=int, default=256)
    ap.add_argument("--nl", type=int, default=6)
    ap.add_argument("--nets", type=int, default=160)
    ap.add_argument("--iters", type=int, default=3)
    ap.add_argument("--width", type=int, default=16)
    ap.add_argument("--epochs", type=int, default=12)
    ap.add_argument("--threshold", type=float, default=0.5)
    ap.add_argument("--repeat", type=int, default=2, help="negotiations per board and method; the fastest counts")
    a = ap.parse_args()
    kw = dict(nx=a.nx, ny=a.ny, nl=a.nl, nnets=a.nets, margin=12, span=(16, max(24, min(a.nx, a.ny) // 2)))
    r = ab_report(range(100, 100 + a.train), range(900, 900 + a.test), kw, a.iters, a.width, a.epochs, a.threshold,
                  repeat=a.repeat)
    print(json.dumps(r))


if __name__ == "__main__":
    main()
