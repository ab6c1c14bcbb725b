"""The finite-difference ladder of the adjoint check (bench.fd_ladder): per
pair, the value at the largest step size where the pair is resolved, central
before one-sided before ambiguous."""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import bench  # noqa: E402


def _cls(central, one_sided, ambiguous):
    return {"central": np.array(central), "one_sided": np.array(one_sided), "ambiguous": np.array(ambiguous)}


def test_ladder_takes_the_largest_resolved_step():
    inf = np.inf
    levels = [
        # pair 0 central at 1e-6; pair 1 unresolved; pair 2 one-sided; pair 3 ambiguous; pair 4 unresolved
        (1e-6, np.array([1e-9, inf, 2e-7, 5e-6, inf]),
         _cls([1, 0, 0, 0, 0], [0, 0, 1, 0, 0], [0, 0, 0, 1, 0])),
        # pair 1 central at 1e-7
        (1e-7, np.array([2e-9, 3e-8, inf, inf, inf]), _cls([1, 1, 0, 0, 0], [0, 0, 0, 0, 0], [0, 0, 0, 0, 0])),
        # pair 2 central at 1e-8 (wins over its one-sided value at 1e-6)
        (1e-8, np.array([4e-9, 5e-8, 6e-8, inf, inf]), _cls([1, 1, 1, 0, 0], [0, 0, 0, 0, 0], [0, 0, 0, 0, 0])),
    ]
    levels = [(h, r, {k: v.astype(bool) for k, v in c.items()}) for h, r, c in levels]
    out = bench.fd_ladder(levels)
    assert out["resolved_at"] == [2, 1, 1]  # pairs 0 and 3 at 1e-6, pair 1 at 1e-7, pair 2 at 1e-8
    assert out["unresolved"] == 1
    assert out["meets_1e-6"] == 3  # pair 3 (ambiguous, 5e-6) misses
    assert abs(out["meets_1e-6_frac"] - 0.6) < 1e-12
