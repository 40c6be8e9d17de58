"""Launch-shape tuning (fb_tune / fb_set_tuning): the tuner must leave the
disc exactly where it was, and a tuned disc must follow the same trajectory
as an untuned one (shapes change the work split, not the arithmetic; only
the order of the ring-mean sum of the azimuthal pass may differ)."""
import os

import numpy as np
import pytest

from tests import _oracle

pytestmark = pytest.mark.gpu
FIELDS = ("dens", "vrad", "vtheta")


def test_tune_restores_state_and_keeps_results(tmp_path):
    from dustyfargoadsg_b200 import Disc, read_par, tune
    par = _oracle.write_par(os.path.join(_oracle.CONFIG_DIR, "iso_128x384.par"), str(tmp_path),
                            Nrad=96, Nsec=288)
    with Disc(read_par(par), noise=1e-4, seed=0) as a, Disc(read_par(par), noise=1e-4, seed=0) as b:
        a.step()
        b.step()
        before = a.download()
        entry = tune.tune_disc(a, substeps=2)
        after = a.download()
        for k in FIELDS:
            np.testing.assert_array_equal(before[k], after[k], err_msg=k)
        assert before["PhysicalTime"] == after["PhysicalTime"]
        assert a.tuning() == {k: entry[k] for k in tune.FIELDS}
        for _ in range(2):
            ra, rb = a.step(), b.step()
            assert ra.substeps == rb.substeps
        sa, sb = a.download(), b.download()
        for k in FIELDS:
            assert _oracle.rel_err(sa[k], sb[k]) <= 1e-13, k


def test_tuning_table_lookup(tmp_path):
    from dustyfargoadsg_b200 import Disc, FbError, read_par
    par = _oracle.write_par(os.path.join(_oracle.CONFIG_DIR, "iso_128x384.par"), str(tmp_path),
                            Nrad=64, Nsec=192)
    table = {"iso": {"64x192": {"cell_block": 64, "azi_cells_per_thread": 2, "rad_columns": 32, "rad_rings": 8}}}
    with Disc(read_par(par), tuning=table) as d:
        assert d.tuning() == {"cell_block": 64, "azi_cells_per_thread": 2, "rad_columns": 32, "rad_rings": 8,
                              "azi_variant": 3}
        with pytest.raises(FbError):
            d.set_tuning({"cell_block": 48})
        d.step()


@pytest.mark.parametrize("cfg", ["adiabatic_sg_512x1536.par", "iso_128x384.par"])
@pytest.mark.parametrize("E", [1, 2, 3, 4])
def test_azimuthal_variants_are_bit_identical(tmp_path, E, cfg):
    """The narrow (three barriers per quantity), wide (all quantities per
    phase), packed (a cell's quantities side by side), register (E
    contiguous cells per thread, quantities in registers, each face flux
    evaluated once; E >= 2), staged (the register variant fed and drained
    by bulk asynchronous copies) and tile (one warp per tile of 32 E - 9
    cells with a halo, no barrier; here 3 or 4 tiles per ring, the last one
    wrapping around the ring; 128 or 168 registers) azimuthal passes do the same arithmetic: whole
    DTs, isothermal or with energy, cooling and self-gravity, must agree to
    the last bit."""
    from dustyfargoadsg_b200 import Disc, read_par
    nsec = 256 if E == 4 else 192  # the register variant needs nsec / E threads, a multiple of 32
    par = _oracle.write_par(os.path.join(_oracle.CONFIG_DIR, cfg), str(tmp_path), Nrad=64, Nsec=nsec)
    out = {}
    variants = (1, 2, 3, 4, 5, 6, 7, 8) if E >= 2 else (1, 2, 3)
    for variant in variants:
        with Disc(read_par(par), noise=1e-3, seed=4) as d:
            d.set_tuning({"cell_block": 128, "azi_cells_per_thread": E, "azi_variant": variant})
            assert d.tuning()["azi_variant"] == variant
            for _ in range(2):
                d.step()
            out[variant] = d.download()
    fields = FIELDS + (("energy",) if read_par(par).energy_equation else ())
    for v in variants[1:]:
        for k in fields:
            np.testing.assert_array_equal(out[1][k], out[v][k], err_msg="%s variant %d" % (k, v))


@pytest.mark.parametrize("E", [2, 3, 4])
def test_tile_variant_on_short_rings(tmp_path, E):
    """Rings shorter than one tile's 32 E loaded cells (nsec 64): the tile
    wraps around its ring more than once and must still give the narrow
    variant's results to the last bit (adiabatic disc with cooling and
    self-gravity, two DTs)."""
    from dustyfargoadsg_b200 import Disc, read_par
    par = _oracle.write_par(os.path.join(_oracle.CONFIG_DIR, "adiabatic_sg_512x1536.par"), str(tmp_path),
                            Nrad=48, Nsec=64)
    out = {}
    for variant in (1, 6, 7, 8):
        with Disc(read_par(par), noise=1e-3, seed=5) as d:
            d.set_tuning({"cell_block": 128, "azi_cells_per_thread": E, "azi_variant": variant})
            assert d.tuning()["azi_variant"] == variant
            for _ in range(2):
                d.step()
            out[variant] = d.download()
    for v in (6, 7, 8):
        for k in FIELDS + ("energy",):
            np.testing.assert_array_equal(out[1][k], out[v][k], err_msg="%s variant %d" % (k, v))
