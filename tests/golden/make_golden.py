"""Golden fixtures of the oracle: rectangle, best target, tries and a digest of the reported field for seeded
GpuQuery cases. Regenerate with `python -m tests.golden.make_golden` (writes tests/golden/oracle_golden.npz)."""
from __future__ import annotations

import hashlib
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from pcbroute_b200 import synth  # noqa: E402


def cases():
    yield "plain", synth.random_query(1001, nx=90, ny=70, nl=3)
    yield "prior", synth.random_query(1002, nx=90, ny=70, nl=4, prior=True)
    yield "corridor", synth.random_query(1003, nx=90, ny=70, nl=3, prior=True, corridor=True)
    yield "novia", synth.random_query(1004, nx=90, ny=70, nl=2, vias=False)
    yield "unusable", synth.random_query(1005, nx=90, ny=70, nl=4, unusable_layer=True)
    q = synth.random_query(1006, nx=700, ny=600, nl=2, window=(5, 5, 690, 590), n_starts=1, n_targets=1)
    fwn = q.ww * q.wh
    q.starts = [(300 * q.ww + 300, 0.0)]
    q.tbit[:] = 0
    t = fwn + 320 * q.ww + 340
    q.tbit[t >> 6] |= np.uint64(1) << np.uint64(t & 63)
    yield "growth", q


def digest(field: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(field, np.float32).tobytes()).hexdigest()


def main() -> None:
    from oracle import oracle as O
    out = {}
    for name, q in cases():
        rc, r = O.solve(q)
        assert rc >= 1, name
        out[name + "_rect"] = np.array([r.rx0, r.ry0, r.rw, r.rh, r.best, r.tries])
        out[name + "_digest"] = np.array(digest(r.d))
        print(name, out[name + "_rect"], out[name + "_digest"])
    np.savez(os.path.join(os.path.dirname(os.path.abspath(__file__)), "oracle_golden.npz"), **out)


if __name__ == "__main__":
    main()
