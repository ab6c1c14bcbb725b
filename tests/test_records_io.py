"""Conjunction record output in the reference's formats (host functions of the
C ABI): the CSV of io/ConjuctionLogger.cpp and the HDF5 CollisionInfo layout of
io/hdf5/HDF5Definitions.h:42-68.  No GPU needed."""
import math

import numpy as np
import pytest


@pytest.fixture(scope="module")
def capi():
    from ladds_b200 import build, capi

    build.build_gpu()
    return capi


def records(capi, rows):
    out = np.zeros(len(rows), dtype=capi.PAIR_DTYPE)
    for k, (step, a, b, dl2, flags) in enumerate(rows):
        out[k]["step"], out[k]["idA"], out[k]["idB"], out[k]["dl2"], out[k]["flags"] = step, a, b, dl2, flags
    return out


def test_pack_collision_info_layout(capi):
    recs = records(capi, [(3, 7, 9, 0.0025, capi.PAIR_COLLISION), (3, 1, 2, 0.5, capi.PAIR_EVASION),
                          (4, (1 << 32) + 5, 6, 1e-7, capi.PAIR_COLLISION | capi.PAIR_CONJUNCTION)])
    col = capi.pack_records(recs, capi.PAIR_COLLISION)
    assert col.dtype.itemsize == 12 and len(col) == 2
    assert col["idA"].tolist() == [7, 5]  # ids narrowed to unsigned int as the reference's static_cast
    assert col["idB"].tolist() == [9, 6]
    assert col["distanceSquared"].tolist() == [np.float32(0.0025), np.float32(1e-7)]
    eva = capi.pack_records(recs, capi.PAIR_EVASION)
    assert len(eva) == 1 and eva[0]["idA"] == 1 and eva[0]["distanceSquared"] == np.float32(0.5)


def test_csv_format_and_append(capi, tmp_path):
    path = str(tmp_path / "conjunctions.csv")
    recs = records(capi, [(12, 3, 4, 0.0025, 1), (12, 5, 8, 1e-05, 1), (13, 1, 2, 3.0, 2), (13, 6, 7, 1.5e16, 1),
                          (14, 9, 10, float("nan"), 1), (14, 11, 12, 0.1 + 0.2, 1)])
    capi.write_records_csv(path, recs[:3], capi.PAIR_COLLISION)
    capi.write_records_csv(path, recs[3:], capi.PAIR_COLLISION, append=True)
    lines = open(path).read().splitlines()
    assert lines[0] == "Iteration,P1,P2,SquaredDistance"
    assert lines[1:] == ["12,3,4,0.0025", "12,5,8,1e-05", "13,6,7,1.5e+16", "14,9,10,nan",
                         "14,11,12,0.30000000000000004"]
    # the distances parse back to the same doubles
    vals = [float(line.split(",")[3]) for line in lines[1:]]
    assert vals[0] == 0.0025 and vals[4] == 0.1 + 0.2 and math.isnan(vals[3])
    capi.write_records_csv(path, recs[2:3], capi.PAIR_EVASION)  # rewrite: header again, one line
    assert open(path).read().splitlines() == ["Iteration,P1,P2,SquaredDistance", "13,1,2,3"]
