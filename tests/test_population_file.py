"""Binary SoA population files (ladds_population_write / _read): the input
format the library, the oracle and the benchmark share.  Host code only."""
import ctypes as C
import os

import numpy as np
import pytest


@pytest.fixture(scope="module")
def capi():
    from ladds_b200 import capi

    return capi


def same(a, b, capi):
    return all(np.array_equal(a[k].view(np.uint8), b[k].view(np.uint8)) for k in capi.POP_FIELDS)


@pytest.mark.parametrize("which,n", [(0, 5000), (2, 4300), (4, 2000)])
def test_round_trip_is_bit_exact(capi, tmp_path, which, n):
    pop = capi.generate_population(which, 77, n)
    path = str(tmp_path / "pop.bin")
    capi.save_population(path, pop)
    assert os.path.getsize(path) == 24 + n * (11 * 8 + 1)
    assert same(capi.load_population(path), pop, capi)


def test_header_layout(capi, tmp_path):
    pop = capi.generate_population(0, 3, 10)
    path = str(tmp_path / "pop.bin")
    capi.save_population(path, pop)
    raw = open(path, "rb").read()
    assert raw[:8] == b"LADDSPOP"
    assert np.frombuffer(raw[8:16], "<u4").tolist() == [1, 12]
    assert int(np.frombuffer(raw[16:24], "<u8")[0]) == 10
    assert np.array_equal(np.frombuffer(raw[24:104], "<f8"), pop["x"])  # x first, then y ...
    assert np.array_equal(np.frombuffer(raw[-10:], "i1"), pop["activity"])  # activity last


def test_empty_population(capi, tmp_path):
    path = str(tmp_path / "empty.bin")
    capi.save_population(path, capi.empty_population(0))
    assert len(capi.load_population(path)["x"]) == 0


def test_capacity_and_skipped_arrays(capi, tmp_path):
    pop = capi.generate_population(0, 5, 100)
    path = str(tmp_path / "pop.bin")
    capi.save_population(path, pop)
    L = capi.lib()
    n = C.c_size_t()
    assert L.ladds_population_read(path.encode(), 99, C.byref(n), *([None] * 12)) == capi.ERR_CAPACITY
    assert n.value == 100
    ids = np.zeros(100, np.uint64)
    args = [None] * 12
    args[9] = ids.ctypes.data_as(C.c_void_p)  # ids only
    assert L.ladds_population_read(path.encode(), 100, C.byref(n), *args) == capi.OK
    assert np.array_equal(ids, pop["id"])


def test_rejects_other_files(capi, tmp_path):
    pop = capi.generate_population(0, 6, 50)
    good = str(tmp_path / "pop.bin")
    capi.save_population(good, pop)
    raw = open(good, "rb").read()
    cases = {"truncated": raw[:-1], "trailing": raw + b"\0", "magic": b"X" + raw[1:],
             "version": raw[:8] + b"\2" + raw[9:], "short header": raw[:20]}
    for name, data in cases.items():
        path = str(tmp_path / f"{name}.bin")
        open(path, "wb").write(data)
        with pytest.raises(capi.LaddsError):
            capi.load_population(path)
    with pytest.raises(capi.LaddsError):
        capi.load_population(str(tmp_path / "missing.bin"))
    with pytest.raises(capi.LaddsError):
        capi.save_population(str(tmp_path / "no_such_dir" / "p.bin"), pop)
