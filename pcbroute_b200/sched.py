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
