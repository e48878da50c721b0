"""Replicas on N GPUs: the searches of a round are independent given the committed board, so N processes (one per
GPU) each solve their own share of the waves with no collective on the data path. Only the timing is combined:
the step time is the slowest rank's, the work is the sum over ranks."""
from __future__ import annotations


def my_waves(waves: list, ws: int, rank: int) -> list:
    """Round-robin share of rank `rank` of `ws`: waves rank, rank + ws, ...; every rank gets the same count (ranks
    beyond the last wave wrap around), so per-rank work stays fixed as ws grows (weak scaling)."""
    nw = len(waves)
    return [waves[(rank + ws * k) % nw] for k in range(max(1, -(-nw // ws)))]


def max_time_sum_work(ms: float, work: float, device, ws: int) -> tuple[float, float]:
    """(max over ranks of ms, sum over ranks of work); a no-op reduction on one rank."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    w = torch.tensor([float(work)], dtype=torch.float64, device=device)
    if ws > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dist.all_reduce(w, op=dist.ReduceOp.SUM)
    return float(t.item()), float(w.item())
