"""The learned speculation scheduler: the network's forward and backward kernels against the numpy oracle
(oracle/mlp_oracle.py), the oracle's backward against finite differences, and the learned batch composition
against the plain one on held-out boards (same paths, fewer wasted searches)."""
import numpy as np
import pytest

from oracle import mlp_oracle as M

D0, H = M.D0, M.H


def _params(rng, scale=1.0):
    n = H * D0 + H * H + 3 * H + 1
    p = np.zeros(n, np.float32)
    p[:H * D0] = rng.normal(0, scale * np.sqrt(2.0 / D0), H * D0)
    p[H * D0:H * D0 + H * H] = rng.normal(0, scale * np.sqrt(2.0 / H), H * H)
    o = H * D0 + H * H
    p[o:o + 2 * H] = rng.normal(0, 0.05, 2 * H)
    p[o + 2 * H:o + 3 * H] = rng.normal(0, np.sqrt(2.0 / H), H)
    p[-1] = 0.1
    return p


def _batch(rng, B):
    x = rng.random((B, D0)).astype(np.float32) * (rng.random((B, D0)) < 0.3)
    y = (rng.random(B) < 0.3).astype(np.float32)
    w = np.where(y > 0, 2.0, 1.0).astype(np.float32)
    w[-5:] = 0.0  # padding rows
    return x, y, w


def test_oracle_backward_matches_finite_differences():
    """The restated backward formulas, in float64 without rounding, against central differences."""
    rng = np.random.default_rng(3)
    p = _params(rng).astype(np.float64)
    x, y, w = _batch(rng, 16)
    _, _, g = M.forward_backward(p, x, y, w, rounding=False)
    n1 = H * D0
    idx = list(rng.integers(0, n1, 6)) + list(n1 + rng.integers(0, H * H, 6)) + \
        list(range(n1 + H * H, n1 + H * H + 3 * H + 1, 41)) + [p.size - 1]
    for k in idx:
        e = np.zeros_like(p)
        e[k] = 1e-6
        lp = M.forward_backward(p + e, x, y, w, rounding=False)[1]
        lm = M.forward_backward(p - e, x, y, w, rounding=False)[1]
        num = (lp - lm) / 2e-6
        assert abs(num - g[k]) <= 1e-6 + 1e-4 * abs(g[k]), (k, num, g[k])


def test_bf16_rounding_is_nearest_even():
    a = np.array([1.0, 1.00390625, 1.01171875, -2.5, 3.0e38], np.float32)
    b = M.bf16_bits(a)
    assert list(M.bf16_to_f32(b)) == [1.0, 1.0, 1.015625, -2.5, np.float32(M.bf16_to_f32(b)[4])]


@pytest.mark.gpu
def test_device_forward_and_gradients_match_the_oracle(gpu):
    """Forward probabilities within 2e-3; every parameter block's gradient within 2 % relative (L2) of the oracle.
    The tolerance covers float32 against float64 accumulation and the bf16 roundings of h1 / dz that this moves."""
    from pcbroute_b200.sched import Scheduler
    rng = np.random.default_rng(11)
    s = Scheduler(5)
    p = _params(rng)
    s.set_params(p)
    x, y, w = _batch(rng, 128)
    xb = M.bf16_bits(x)
    xf = M.bf16_to_f32(xb)
    prob = s.forward(xb)
    g, loss = s.grad(xb, y, w)
    rp, rloss, rg = M.forward_backward(p, xf, y, w)
    assert np.max(np.abs(prob - rp)) < 2e-3
    assert abs(loss - rloss) < 1e-3 * max(1.0, abs(rloss))
    n1, n2 = H * D0, H * H
    cuts = [("W1", 0, n1), ("W2", n1, n1 + n2), ("b1", n1 + n2, n1 + n2 + H), ("b2", n1 + n2 + H, n1 + n2 + 2 * H),
            ("w3", n1 + n2 + 2 * H, n1 + n2 + 3 * H), ("b3", n1 + n2 + 3 * H, n1 + n2 + 3 * H + 1)]
    for name, a, b in cuts:
        ref = rg[a:b]
        err = np.linalg.norm(g[a:b] - ref) / max(np.linalg.norm(ref), 1e-12)
        assert err < 2e-2, (name, err)
    s.close()


@pytest.mark.gpu
def test_learned_batching_wastes_fewer_searches_with_the_same_paths(gpu):
    """Train on the conflict logs of plain rounds over seeded boards, then negotiate held-out boards with the plain
    and the learned batch composition: identical paths, and a lower wasted-search fraction for the learned one."""
    from pcbroute_b200 import spec
    from pcbroute_b200.sched import Scheduler, collect_logs, run
    train = [spec.spec_board(100 + k, nx=160, ny=128, nl=4, nnets=64, margin=10, span=(12, 70)) for k in range(6)]
    test = [spec.spec_board(900 + k, nx=160, ny=128, nl=4, nnets=64, margin=10, span=(12, 70)) for k in range(3)]
    s = Scheduler(21)
    collect_logs(s, train, iters=2, width=12)
    n, pos = s.log_size()
    assert n > 500 and 0 < pos < n
    s.train(epochs=12, lr=1e-3, batch=256)
    plain_w = plain_s = learn_w = learn_s = 0
    for b in test:
        pp, ps = run(b, 2, 12)
        lp, ls = run(b, 2, 12, sch=s, threshold=0.5)
        for k in range(len(pp)):
            assert np.array_equal(pp[k], lp[k]), k
        plain_w += sum(x["wasted"] for x in ps)
        plain_s += sum(x["searches"] for x in ps)
        learn_w += sum(x["wasted"] for x in ls)
        learn_s += sum(x["searches"] for x in ls)
    assert plain_w > 0
    assert learn_w / learn_s < plain_w / plain_s, (learn_w, learn_s, plain_w, plain_s)
    s.close()
