"""Batched discs (fb_batch_*): several discs of different grid sizes and
parameters advanced by one graph launch per DT must give exactly the state
each disc reaches on its own with fb_algogas (same kernels, same order)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_batch_matches_single_discs(tmp_path):
    from dustyfargoadsg_b200 import Batch, sweep
    draws = sweep.draw_discs(5, seed=2, nrads=(32, 48, 64))
    solo = sweep.make_discs(draws, str(tmp_path / "solo"))
    together = sweep.make_discs(draws, str(tmp_path / "batch"))
    try:
        with Batch(together) as batch:
            for _ in range(2):
                reps = batch.step()
                for d in solo:
                    d.step()
                assert all(r.status == 0 for r in reps)
        for a, b, r in zip(solo, together, reps):
            sa, sb = a.download(), b.download()
            for k in ("dens", "vrad", "vtheta"):
                np.testing.assert_array_equal(sa[k], sb[k], err_msg=k)
            assert sa["PhysicalTime"] == sb["PhysicalTime"] == r.physical_time
    finally:
        for d in solo + together:
            d.close()


def test_batch_draws_are_seeded():
    from dustyfargoadsg_b200 import sweep
    a, b = sweep.draw_discs(64, seed=2), sweep.draw_discs(64, seed=2)
    assert a == b
    assert {d["Nrad"] for d in a} <= set(sweep.NRADS)
    assert all(d["Nsec"] == 3 * d["Nrad"] for d in a)
    assert all(1e-5 <= d["q"] <= 3e-3 and 1e-4 <= d["AlphaViscosity"] <= 1e-2 for d in a)
    assert all(0.03 <= d["AspectRatio"] <= 0.1 and 0.0 <= d["SigmaSlope"] <= 1.5 for d in a)
