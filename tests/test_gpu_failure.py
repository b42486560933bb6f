"""Failure detection on the GPU without a GPU fault: a CTA of the tiled kernel
withholds one spike record, so the bounded waits of every other CTA run out.
The run must end (its next synchronising call raises TimeoutError) within a
few seconds, since the waits give up after 2 s, and the CUDA context must stay
usable: a fresh plan afterwards
runs and matches the oracle."""
import time

import numpy as np
import pytest

from tests.netbuild import Net

pytestmark = pytest.mark.gpu


def _raster(steps, gids):
    return set(zip(steps.tolist(), gids.tolist()))


@pytest.mark.parametrize("delays", [(10, 30), (64, 80)])  # plain and pipelined windows
def test_withheld_record_times_out_and_context_survives(oracle, delays):
    net = Net(per_edge_delay=delays, delay=delays[0])
    pl = net.to_plan(precision=32, semantics=1)
    pl.debug_withhold_record(cta=3, window=2)
    t0 = time.monotonic()
    pl.run(400)  # asynchronous: the error comes back from the next synchronising call
    with pytest.raises(TimeoutError):
        pl.spikes()
    assert time.monotonic() - t0 < 20.0
    # the context still works: a new plan runs to the oracle's spikes
    rec = np.arange(0, 250, 9)
    pl2 = net.to_plan(precision=64, semantics=1, rec=rec)
    sim = net.to_oracle(oracle, semantics=1, rec=rec)
    pl2.run(150)
    st, g = pl2.spikes()
    ost, og, ov = sim.run(150)
    assert len(st) > 0
    assert _raster(st, g) == _raster(ost, og)
    np.testing.assert_allclose(pl2.v_trace(), ov, rtol=0, atol=1e-9)
    # the hook covered one run: the first plan runs again without it
    pl.run(20)
    pl.spikes()


def test_hook_needs_the_tiled_path(oracle):
    from brainpy.state_b200 import _lib
    pl = _lib.Plan(0.1, "aeif_cond_alpha", precision=64)
    pl.add_pop(10, [0.0, -60.0, 0.0, 30.0, 281.0, 0.0, -85.0, -70.6, 2.0, 144.0, 4.0, 80.5,
                    -50.4, 0.2, 2.0, 0.0, 1e-6])
    pl.upload()
    with pytest.raises(NotImplementedError):
        pl.debug_withhold_record(0, 0)
