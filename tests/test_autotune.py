"""Autotuner: the tuned context produces exactly the records and states of an
untuned one (only the speed may change), and every trial is reported."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def capi():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from ladds_b200 import build, capi

    build.build_gpu()
    return capi


def test_autotune_keeps_results_and_reports_trials(capi):
    pop = capi.generate_population(0, 31, 200_000)
    cfg = dict(componentMask=capi.PROP_ALL, precision=capi.PRECISION_SPLIT)
    with capi.Context(capi.default_config(**cfg)) as tuned, capi.Context(capi.default_config(**cfg)) as plain:
        tuned.upload(pop)
        plain.upload(pop)
        tuned.step(3)
        plain.step(3)
        best, trials = tuned.autotune(6)
        assert len(trials) >= 6
        assert all(t["msPerStep"] > 0 for t in trials)
        assert best["msPerStep"] == min(t["msPerStep"] for t in trials)
        assert best["cellSize"] in {t["cellSize"] for t in trials}
        dims, reach, cell = tuned.grid()
        assert reach == best["reach"] and cell == pytest.approx(best["cellSize"])
        a = tuned.step(40)
        b = plain.step(40)
        assert a.records.tobytes() == b.records.tobytes()
        sa, sb = tuned.download(), plain.download()
        for k in ("x", "y", "z", "vx", "vy", "vz", "id"):
            assert np.array_equal(sa[k], sb[k]), k
