"""pcbg_solve_noalloc: the entry point for callers that cannot allocate device memory.

Callers whose device memory belongs to another allocator, or whose threads must not be stalled by cudaFree,
call pcbg_solve_noalloc. It keeps its scratch in a static device array, so it must give exactly what
pcbg_solve_batch (which allocates from its own arena) gives for the same search. These tests check that on two
calls in a row with different searches, since the second call reuses the array the first one left behind. They
also check that a search above the stated limit is refused with a message. This file is collected last.
"""
import numpy as np
import pytest

from pcbroute_b200 import _lib, synth

pytestmark = pytest.mark.gpu


def _search(torch, seed, rw, rh, nl, via):
    lib = _lib.load()
    pitch, hpad = -(-rw // 32) * 32, -(-rh // 32) * 32
    t = dict(cf=torch.empty(nl * hpad * pitch, dtype=torch.float32, device="cuda"),
             fl=torch.empty(nl * hpad * pitch, dtype=torch.uint8, device="cuda"),
             vcf=torch.empty(hpad * pitch, dtype=torch.float32, device="cuda"),
             st=torch.empty(2, dtype=torch.int64, device="cuda"))
    assert lib.pcbg_synth_search(seed, rw, rh, nl, pitch, hpad, via, t["cf"].data_ptr(), t["fl"].data_ptr(),
                                 t["vcf"].data_ptr(), t["st"].data_ptr(), None) == 0
    t["si"] = t["st"][:1].to(torch.int32)
    t["sd"] = torch.zeros(1, dtype=torch.int64, device="cuda")
    arr = (_lib.Search * 1)()
    a = arr[0]
    a.rw, a.rh, a.nl, a.pitch, a.hpad = rw, rh, nl, pitch, hpad
    fac = synth.microbench_factors(nl)
    for l in range(8):
        for m in range(8):
            a.fac[l][m] = float(fac[l, m])
    a.cf, a.flags, a.vcf = t["cf"].data_ptr(), t["fl"].data_ptr(), t["vcf"].data_ptr()
    a.start_idx, a.start_d, a.n_starts = t["si"].data_ptr(), t["sd"].data_ptr(), 1
    return arr, t


def _solve(torch, noalloc, arr, n_out):
    lib = _lib.load()
    out = torch.full((n_out,), -1.0, dtype=torch.float32, device="cuda")
    arr[0].out = out.data_ptr()
    rc = lib.pcbg_solve_noalloc(arr, None) if noalloc else lib.pcbg_solve_batch(arr, 1, None)
    assert rc == 0, _lib.last_error()
    torch.cuda.synchronize()
    return out.cpu().numpy(), arr[0].best, arr[0].best_d, arr[0].status


def test_noalloc_matches_the_allocating_entry_point_on_two_calls_in_a_row():
    import torch
    assert torch.cuda.is_available()
    # the second search is smaller than the first: what call 1 left in the array must not leak into call 2
    cases = [(7001, 700, 520, 5, 12.0), (7002, 230, 170, 3, 20.0)]
    made = [_search(torch, *c) for c in cases]
    sizes = [rw * rh * nl for (_, rw, rh, nl, _) in cases]
    refs = [_solve(torch, False, arr, n) for (arr, _), n in zip(made, sizes)]
    gots = [_solve(torch, True, arr, n) for (arr, _), n in zip(made, sizes)]   # two no-alloc calls in a row
    for c, ref, got in zip(cases, refs, gots):
        assert got[1:] == ref[1:], (c, got[1:], ref[1:])
        assert got[1] >= 0
        # exact: the arithmetic is integer, the tolerance is zero
        assert np.array_equal(got[0].view(np.uint32), ref[0].view(np.uint32)), c


def test_noalloc_refuses_searches_above_its_limit():
    import torch
    lib = _lib.load()
    arr, t = _search(torch, 7003, 64, 64, 2, 10.0)
    arr[0].rw, arr[0].rh, arr[0].pitch, arr[0].hpad = 2048, 1056, 2048, 1056   # 2 x 2048 x 1056 > 2^21
    arr[0].out = None
    assert lib.pcbg_solve_noalloc(arr, None) == -1
    assert "exceeds the no-alloc limit" in _lib.last_error()
