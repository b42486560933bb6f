"""The tiled path's autotuner: pilots over CTA counts and poll pauses leave the
plan's state where it was, and the tuned shape gives the same FP64 raster
(int64 fixed-point arrival sums do not depend on how the neurons are tiled).
"""
import numpy as np
import pytest

from brainpy.state_b200 import brunel

pytestmark = pytest.mark.gpu


def _raster(pl):
    st, g = pl.spikes()
    return set(zip(st.tolist(), g.tolist()))


def test_tuned_shape_keeps_state_and_raster():
    ref, _ = brunel.build_plan(order=1000, precision=64, seed=77, rec_v=20)
    assert ref.engine == "tiled"
    ref.run(300)
    pl, _ = brunel.build_plan(order=1000, precision=64, seed=77, rec_v=20)
    grid, pause, ms = pl.tune_tiled(pilot_steps=200)
    assert pause in (200, 400, 700) and ms > 0
    assert grid >= 1
    assert pl.step == 0  # the pilots' state was restored
    assert pl.tiled_options()["poll_pause_ns"] == pause
    pl.run(300)
    assert len(_raster(ref)) > 100
    assert _raster(pl) == _raster(ref)
    np.testing.assert_array_equal(pl.v_trace(), ref.v_trace())
