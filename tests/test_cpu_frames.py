"""Host logic of the frame-pair driver (no GPU): quick-stats' Stats and the
frame selection of turbo-metrics' compute_all."""
import numpy as np
import pytest

import conftest


@pytest.fixture(scope="module")
def frames():
    import importlib
    conftest.load_package()
    return importlib.import_module("tmb.frames")


def test_stats_match_numpy(frames):
    rng = np.random.default_rng(3)
    v = rng.normal(60, 12, 257)
    st = frames.Stats.compute(v)
    assert st.min == v.min() and st.max == v.max()
    assert st.mean == pytest.approx(v.mean(), rel=1e-14)
    assert st.var == pytest.approx(v.var(), rel=1e-12)
    assert st.sample_var == pytest.approx(v.var(ddof=1), rel=1e-12)
    assert st.stddev == pytest.approx(v.std(), rel=1e-12)
    for p in (1, 5, 50, 95, 99):
        assert getattr(st, "p%d" % p) == pytest.approx(np.percentile(v, p), rel=1e-14)


def test_stats_reference_example(frames):
    # quick-stats/src/lib.rs:104-107 runs Stats::compute(&[0.0, 1.0, 3.0, 4.0])
    st = frames.Stats.compute([0.0, 1.0, 3.0, 4.0])
    assert (st.min, st.max, st.mean) == (0.0, 4.0, 2.0)
    assert st.var == 2.5 and st.sample_var == pytest.approx(10 / 3)
    assert st.p50 == 2.0 and st.p1 == pytest.approx(0.03) and st.p99 == pytest.approx(3.97)
    one = frames.Stats.compute([5.0])
    assert one.var == 0.0 and one.p1 == one.p99 == 5.0


def test_frame_selection(frames):
    sel = lambda **kw: [a for a, _ in frames.select_frames(range(20), range(100, 115), **kw)]
    assert sel() == list(range(15))                      # pairs while both sources last
    assert sel(skip=2) == list(range(2, 15))
    assert [(a, b) for a, b in frames.select_frames(range(10), range(10), skip_ref=1, skip_dis=3)][:2] == [(1, 3), (2, 4)]
    assert sel(every=3) == [0, 3, 6, 9, 12]              # the first pair, then every 3rd
    assert sel(frames=4) == [0, 1, 2, 3]
    # `frames` counts decoded pairs, the ones `every` skips included (lib.rs:397-405)
    assert sel(every=2, frames=3) == [0, 2]
