"""Seeded synthetic inputs.

1. The batched-search microbenchmark workload: searches with log-uniform window sides in [64, 2048), 2-6 layers,
   per-(layer, cell) cost 1-16, ~15 % of cells blocked in clustered value-noise blobs, via cost 8-32, one free
   source and one free target. `search_arrays` regenerates exactly what the device generator pcbg_synth_search
   (csrc/synth.cu) writes, from the same integer hash.
2. Random GpuQuery boards (`random_query`) exercising every part of the query contract: owner grids, negated own
   copper, own-copper overrides, blocked cells, via rules, per-layer direction factors, unusable layers, learned
   priors with corridors, several starts and targets.
"""
from __future__ import annotations

import math

import numpy as np

from .query import GpuQuery

_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)
_TAGK = 0xD1B54A32D192ED03
MASK64 = (1 << 64) - 1
BLOCK_T = 128000


def _mix(z: np.ndarray) -> np.ndarray:
    z = np.asarray(z, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = z ^ (z >> np.uint64(30))
        z = z * _M1
        z = z ^ (z >> np.uint64(27))
        z = z * _M2
        return z ^ (z >> np.uint64(31))


def hash4(seed: int, tag: int, a, b) -> np.ndarray:
    """The generator's hash (csrc/synth.cu hash4), vectorised over a and b."""
    x = _mix(np.uint64(seed & MASK64) ^ np.uint64((tag * _TAGK) & MASK64))
    with np.errstate(over="ignore"):
        x = _mix(x + np.asarray(a, dtype=np.uint64))
        return _mix(x + np.asarray(b, dtype=np.uint64))


def _octave(seed: int, tag: int, l: int, ii: np.ndarray, jj: np.ndarray, sh: int) -> np.ndarray:
    s = 1 << sh
    ax, fx, by, fy = ii >> sh, ii & (s - 1), jj >> sh, jj & (s - 1)
    base = np.uint64(l) << np.uint64(32)

    def v(a, b):
        return (hash4(seed, tag, base | a.astype(np.uint64), b.astype(np.uint64)) >> np.uint64(56)).astype(np.int64)

    v00, v10, v01, v11 = v(ax, by), v(ax + 1, by), v(ax, by + 1), v(ax + 1, by + 1)
    return ((v00 * (s - fx) + v10 * fx) * (s - fy) + (v01 * (s - fx) + v11 * fx) * fy) << (2 * (4 - sh))


def blocked_layer(seed: int, l: int, rw: int, rh: int) -> np.ndarray:
    jj, ii = np.mgrid[0:rh, 0:rw].astype(np.int64)
    return 2 * _octave(seed, 2, l, ii, jj, 4) + _octave(seed, 3, l, ii, jj, 2) >= BLOCK_T


def _blocked_at(seed: int, l: int, i: int, j: int) -> bool:
    a = np.array([[i]], np.int64)
    b = np.array([[j]], np.int64)
    return bool(2 * _octave(seed, 2, l, a, b, 4)[0, 0] + _octave(seed, 3, l, a, b, 2)[0, 0] >= BLOCK_T)


def pick_src_tgt(seed: int, rw: int, rh: int, nl: int) -> tuple[int, int]:
    n, rn = rw * rh * nl, rw * rh
    src = tgt = -1
    for k in range(64):
        c = int(hash4(seed, 4, k, 0)) % n
        if not _blocked_at(seed, c // rn, c % rw, (c % rn) // rw):
            src = c
            break
    for k in range(64):
        c = int(hash4(seed, 5, k, 0)) % n
        if not _blocked_at(seed, c // rn, c % rw, (c % rn) // rw) and c != src:
            tgt = c
            break
    return src, tgt


def search_arrays(seed: int, rw: int, rh: int, nl: int, via: float):
    """Dense arrays of one generated search: cf [nl, rh, rw] f32, flags [nl, rh, rw] u8, vcf [rh, rw] f32, src, tgt."""
    cf = np.empty((nl, rh, rw), np.float32)
    fl = np.empty((nl, rh, rw), np.uint8)
    cells = (np.arange(rh, dtype=np.uint64)[:, None] * np.uint64(rw) + np.arange(rw, dtype=np.uint64)[None, :])
    for l in range(nl):
        b = blocked_layer(seed, l, rw, rh)
        h = hash4(seed, 1, np.uint64(l), cells)
        cost = (1 + ((h >> np.uint64(32)) % np.uint64(16))).astype(np.float32)
        cf[l] = np.where(b, np.float32(1e30), cost)
        fl[l] = np.where(b, 0, 1).astype(np.uint8)
    vcf = np.full((rh, rw), via, np.float32)
    src, tgt = pick_src_tgt(seed, rw, rh, nl)
    if tgt >= 0:
        l, c = divmod(tgt, rw * rh)
        fl[l, c // rw, c % rw] |= 2
    return cf, fl, vcf, src, tgt


def microbench_factors(nl: int) -> np.ndarray:
    """fac[l][m] of the microbenchmark: step 1, direction factors 1 (orthogonal moves cost 16 x the cell cost in
    fixed point, diagonals fl(cost * fl(sqrt 2)) x 16)."""
    fac = np.zeros((8, 8), np.float32)
    diag = np.float32(SQRT2_F)
    for l in range(8):
        fac[l, :4] = 1.0
        fac[l, 4:] = diag
    return fac


SQRT2_F = float(np.float32(math.sqrt(2.0)))


def microbench_sizes(seed: int, n: int) -> list[tuple[int, int, int, float, int]]:
    """(rw, rh, nl, via, search_seed) of the n searches of the microbenchmark workload."""
    out = []
    for k in range(n):
        u1 = int(hash4(seed, 10, k, 0)) / 2.0**64
        u2 = int(hash4(seed, 11, k, 0)) / 2.0**64
        rw = int(math.floor(64.0 * 2.0 ** (5.0 * u1)))
        rh = int(math.floor(64.0 * 2.0 ** (5.0 * u2)))
        nl = 2 + int(hash4(seed, 12, k, 0)) % 5
        via = float(8 + int(hash4(seed, 13, k, 0)) % 25)
        out.append((rw, rh, nl, via, int(hash4(seed, 14, k, 0))))
    return out


# ---------------------------------------------------------------------------------------------------------------
# random GpuQuery boards

def random_query(seed: int, nx: int = 96, ny: int = 80, nl: int = 3, *, window=None, prior: bool = False,
                 corridor: bool = False, vias: bool = True, n_starts: int = 3, n_targets: int = 4,
                 own: bool = True, unusable_layer: bool = False, big_costs: bool = False,
                 free_dirf: bool = False) -> GpuQuery:
    """A random search over a full grid of nx x ny x nl, as the router would hand it to gpu_solve."""
    rng = np.random.default_rng(seed)
    me = 7
    n = nx * ny
    cst = (1.0 + rng.integers(0, 4, size=(nl, n)) * rng.random((nl, n))).astype(np.float32)
    if big_costs:
        hot = rng.random((nl, n)) < 0.05
        cst = np.where(hot, np.float32(3e5) * rng.random((nl, n)).astype(np.float32) + 1, cst).astype(np.float32)
    st = np.zeros((nl, n), np.uint16)
    blk = rng.random((nl, n)) < 0.12
    cst[blk] = np.float32(1e30)
    st[blk] = 0xFFFF
    # other nets' own copper: negated costs, owner ids
    owned = (rng.random((nl, n)) < 0.08) & ~blk
    owners = rng.integers(1, 12, size=(nl, n)).astype(np.uint16)
    st = np.where(owned, owners, st)
    cst = np.where(owned, -cst, cst).astype(np.float32)
    vcst = (1.0 + rng.random(n)).astype(np.float32)
    vst = np.zeros(n, np.uint16)
    vblk = rng.random(n) < 0.1
    vcst[vblk] = np.float32(1e30)
    vst[vblk] = 0xFFFF
    vown = (rng.random(n) < 0.05) & ~vblk
    vst = np.where(vown, rng.integers(1, 12, size=n).astype(np.uint16), vst)
    vcst = np.where(vown, -vcst, vcst).astype(np.float32)
    if window is None:
        wi0, wj0 = int(rng.integers(0, nx // 4)), int(rng.integers(0, ny // 4))
        ww, wh = int(nx - wi0 - rng.integers(0, nx // 4)), int(ny - wj0 - rng.integers(0, ny // 4))
    else:
        wi0, wj0, ww, wh = window
    dirf = np.ones((8, 8), np.float32)
    for l in range(nl):
        w = np.float32(1.0 + rng.integers(0, 3) * 0.5)
        pref = int(rng.integers(0, 3))
        if pref:
            wd = np.float32(1.0 + (w - 1.0) / 2)
            dirf[l, :2] = 1.0 if pref == 1 else w
            dirf[l, 2:4] = w if pref == 1 else 1.0
            dirf[l, 4:] = wd
    if free_dirf:  # a factor per move (no x / y / diagonal classes)
        dirf[:nl] = (1.0 + rng.integers(0, 5, size=(nl, 8)) * 0.25).astype(np.float32)
    lay = np.zeros(8, np.uint8)
    lay[:nl] = 1
    if unusable_layer and nl > 1:
        lay[int(rng.integers(0, nl))] = 0
    fwn = ww * wh
    ws = fwn * nl
    tbit = np.zeros(ws // 64 + 1, np.uint64)

    def setbit(q):
        tbit[q >> 6] |= np.uint64(1) << np.uint64(q & 63)

    tg = set()
    while len(tg) < n_targets:
        tg.add(int(rng.integers(0, ws)))
    for q in tg:
        setbit(q)
    starts = []
    while len(starts) < n_starts:
        q = int(rng.integers(0, ws))
        if q in tg:
            continue
        starts.append((q, float(np.float32(50.0 * rng.random() * rng.integers(0, 2)))))
    own_cf, own_vcf = [], []
    if own:
        for _ in range(int(rng.integers(5, 40))):
            q = int(rng.integers(0, ws))
            own_cf.append((q, float(np.float32(1.0 + rng.random() * 3)) if rng.random() < 0.9 else 1e30))
        for _ in range(int(rng.integers(0, 10))):
            own_vcf.append((int(rng.integers(0, fwn)), float(np.float32(1.0 + rng.random()))))
    q = GpuQuery(nx=nx, ny=ny, NL=nl, wi0=wi0, wj0=wj0, ww=ww, wh=wh, me=me,
                 via_cost=float(np.float32(rng.integers(100, 600))) if vias else -1.0, step=50.0,
                 dirf=dirf, lay=lay, cst=cst, st=st, vcst=vcst, vst=vst, tbit=tbit,
                 own_cf=own_cf, own_vcf=own_vcf, starts=starts)
    # a few cells of the net's own (negated costs with st == me)
    mine = (rng.random((nl, n)) < 0.03) & ~blk
    q.st = np.where(mine, np.uint16(me), q.st).astype(np.uint16)
    q.cst = np.where(mine, -np.abs(q.cst), q.cst).astype(np.float32)
    if prior:
        pnl, ph, pw = nl, max(2, ny // 4), max(2, nx // 4)
        q.prior = rng.integers(0, 256, size=(pnl, ph, pw)).astype(np.uint8)
        q.pcol = (np.arange(nx) // 4).astype(np.int32)
        q.prow = (np.arange(ny) // 4).astype(np.int32)
        q.pi0, q.pj0 = int(rng.integers(0, 2)), int(rng.integers(0, 2))
        play = -np.ones(8, np.int32)
        play[:nl] = np.arange(nl)
        if nl > 1:
            play[nl - 1] = -1
        q.play = play
        q.mlf = (1.0 + 2.0 * (1.0 - np.minimum(1.0, np.arange(256) / 255.0 / 0.3))).astype(np.float32)
        q.corridor = corridor
        q.mthr = 40 if corridor else 0
    return q
