"""Shared helpers of the test suite (conversions between the product's
population dicts and the oracle's Population, record comparison)."""
import math

import numpy as np


def to_oracle(oracle, pop):
    return oracle.Population(pop["x"], pop["y"], pop["z"], pop["vx"], pop["vy"], pop["vz"], pop["radius"],
                             pop["aom"], pop["bc_inv"], pop["id"], pop["parent"], pop["activity"])


def from_lists(rs, vs, ids, acts, masses, radii, parents=None, cd=2.2):
    """Builds a population like the reference tests' Particle(...) calls with
    calculateBcInv(0., 1., 1., 2.2)."""
    rs = np.asarray(rs, float)
    vs = np.asarray(vs, float)
    n = len(rs)
    aom = np.array([math.pi * radii[k] ** 2 * 1e-6 / masses[k] for k in range(n)])
    bc = np.full(n, cd * math.pi / 1.0)
    return dict(x=rs[:, 0], y=rs[:, 1], z=rs[:, 2], vx=vs[:, 0], vy=vs[:, 1], vz=vs[:, 2],
                radius=np.asarray(radii, float), aom=aom, bc_inv=bc, id=np.asarray(ids, np.uint64),
                parent=None if parents is None else np.asarray(parents, np.uint64),
                activity=np.asarray(acts, np.int8))


def records_equal(a, b):
    """Bit-exact equality of two record arrays (NaN == NaN by bit pattern)."""
    if len(a) != len(b):
        return False
    return a.tobytes() == b.tobytes()


def describe_diff(a, b, limit=5):
    sa = {(int(r["step"]), int(r["idA"]), int(r["idB"]), int(r["slotA"]), int(r["slotB"])): r for r in a}
    sb = {(int(r["step"]), int(r["idA"]), int(r["idB"]), int(r["slotA"]), int(r["slotB"])): r for r in b}
    only_a = sorted(set(sa) - set(sb))[:limit]
    only_b = sorted(set(sb) - set(sa))[:limit]
    diff = [k for k in sorted(set(sa) & set(sb)) if sa[k].tobytes() != sb[k].tobytes()][:limit]
    return f"len {len(a)} vs {len(b)}; only first {only_a}; only second {only_b}; differing {diff}"
