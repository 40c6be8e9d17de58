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


def test_batched_corners_match_oracle(tmp_path):
    """Two batched discs at opposite corners of the sweep's parameter box
    (alpha 1e-2, h 0.1, q 3e-3, SigmaSlope 1.5; alpha 1e-4, h 0.03, q 1e-5,
    SigmaSlope 0) on 128 x 384, against the CPU oracle (the reference's own
    build): fields within 1e-11 (scale-relative) after each of two DTs, equal
    substep counts."""
    import os

    from dustyfargoadsg_b200 import Batch, sweep
    from tests import _oracle
    if not _oracle.have_oracle():
        pytest.skip("oracle not built")
    corners = [dict(Nrad=128, Nsec=384, q=3e-3, AlphaViscosity=1e-2, AspectRatio=0.1, SigmaSlope=1.5),
               dict(Nrad=128, Nsec=384, q=1e-5, AlphaViscosity=1e-4, AspectRatio=0.03, SigmaSlope=0.0)]
    wd = str(tmp_path)
    discs = sweep.make_discs(corners, wd)
    steps = 2
    try:
        refs = [_oracle.run_oracle(os.path.join(wd, "disc%03d.par" % d), steps=steps, noise=1e-4, seed=0)[0]
                for d in range(len(corners))]
        prev = [0] * len(corners)
        with Batch(discs) as batch:
            for s in range(1, steps + 1):
                reps = batch.step()
                for d, (disc, rep, ref) in enumerate(zip(discs, reps, refs)):
                    r = ref["state_%05d" % s]
                    assert rep.status == 0
                    assert rep.substeps == int(r["substeps"]) - prev[d], (d, s)
                    prev[d] = int(r["substeps"])
                    out = disc.download()
                    for k in ("dens", "vrad", "vtheta"):
                        err = _oracle.rel_err(out[k], r[k])
                        assert err <= 1e-11, (d, s, k, err)
    finally:
        for d in discs:
            d.close()
