"""Crash reporting and the step's error statuses.

The reference tests its state for negative values at every substep before
the gas update (DetectCrash, SourceEuler.c:51-69, as AlgoGas uses it at
:545-566): a substep "crashes" when the energy is negative somewhere (the
density test's result is overwritten by the energy test's), the first crash
prints "Crash! at time ..." and writes gas{dens,vrad,vtheta,energy}999.dat,
every crashed substep prints a 'c', and the run goes on.

The failures are made on the host: a state with one negative-energy cell
(the oracle flips the same cell before its first DT), one non-finite cell,
or a substep cap of one.  Tolerances: the 999 dumps are the uploaded state
and must match bit for bit; fields after each DT within 1e-11 (scale-relative),
the parity bar of one DT.
"""
import os
import re

import numpy as np
import pytest

from tests import _oracle

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not _oracle.have_oracle(), reason="oracle not built")]

ADI = os.path.join(_oracle.CONFIG_DIR, "adiabatic_sg_512x1536.par")
NR, NS = 48, 144
CELL = 20 * NS + 50  # ring 20, azimuth 50
TOL_DT = 1e-11


def _crash_par(wd):
    # inviscid: a negative energy gives a non-finite sound speed in its cell,
    # which alpha viscosity would spread through the ring's mean
    return _oracle.write_par(ADI, wd, Nrad=NR, Nsec=NS, SelfGravity="No", AlphaViscosity="0.0")


def _marks(stdout):
    """'c' marks of crashed substeps, from the lines of substep marks."""
    return sum(line.count("c") for line in stdout.splitlines() if re.fullmatch(r"[.c]+", line.strip() or "x"))


@pytest.fixture(scope="module")
def crashed_run(tmp_path_factory):
    wd = str(tmp_path_factory.mktemp("crash"))
    par = _crash_par(wd)
    os.environ["ORACLE_NEGATE_ENERGY"] = str(CELL)
    try:
        dumps, _, wd = _oracle.run_oracle(par, steps=2, noise=1e-4, seed=3, workdir=wd, keep=True)
    finally:
        del os.environ["ORACLE_NEGATE_ENERGY"]
    stdout = open(os.path.join(wd, "stdout.txt")).read()
    return par, dumps, stdout, wd


def _state(d):
    st = {k: d[k] for k in ("dens", "vrad", "vtheta", "energy", "SigmaMed", "EnergyMed", "VthetaMed", "VradMed",
                            "GLOBAL_SoundSpeed", "PhysicalTime", "OmegaFrame", "LostMass", "MINDT", "MAXDT",
                            "pl_mass", "pl_x", "pl_y", "pl_vx", "pl_vy", "stardiscbarycenter_x",
                            "stardiscbarycenter_y")}
    return st


def test_crash_matches_reference(crashed_run):
    from dustyfargoadsg_b200 import Disc, _ffi, read_par
    par, d, stdout, wd = crashed_run
    m = re.search(r"Crash! at time (\S+)", stdout)
    assert m, "the oracle did not crash"
    ref_time = float(m.group(1))
    init = d["state_init"]
    assert init["energy"][CELL] < 0.0
    with Disc(read_par(par), state=_state(init)) as disc:
        reps = [disc.step() for _ in (1, 2)]
        crash = disc.crash_state()
        out = disc.download()
    # the first DT crashed in its first substep only (the floor lifts the
    # transported energy), the second did not
    assert reps[0].status == _ffi.FB_ERR_NEGATIVE and reps[1].status == 0
    assert reps[0].crashes == 1 and reps[1].crashes == 1
    assert [r.crash_substeps for r in reps] == [1, 0]
    assert sum(r.crash_substeps for r in reps) == _marks(stdout)
    assert "%.12g" % reps[0].crash_time == "%.12g" % ref_time
    # the *999.dat dumps: the state at the start of the crashed substep
    n = NR * NS
    for k, name in (("dens", "gasdens"), ("vrad", "gasvrad"), ("vtheta", "gasvtheta"), ("energy", "gasenergy")):
        ref999 = np.fromfile(os.path.join(wd, "out", "%s999.dat" % name))
        assert ref999.size == n
        assert np.array_equal(crash[k], ref999), k
    # and the step went on like the reference's
    prev = 0
    for s, rep in zip((1, 2), reps):
        ref = d["state_%05d" % s]
        assert rep.substeps == int(ref["substeps"]) - prev
        prev = int(ref["substeps"])
    for k in ("dens", "vrad", "vtheta", "energy"):
        assert _oracle.rel_err(out[k], d["state_00002"][k]) <= TOL_DT, k


def test_no_crash_without_negative_energy(tmp_path):
    """A negative density alone is counted but is not a crash for AlgoGas
    (the energy test's result overwrites it)."""
    from dustyfargoadsg_b200 import Disc, read_par
    par = _crash_par(str(tmp_path))
    with Disc(read_par(par), noise=1e-4, seed=3) as disc:
        st = disc.download()
        st.update({k: v for k, v in zip(("SigmaMed", "EnergyMed", "VthetaMed", "VradMed", "GLOBAL_SoundSpeed"),
                                        (disc.prof[q] for q in ("sigma_med", "energy_med", "vtheta_med",
                                                                "vrad_med", "global_soundspeed")))})
        st["dens"] = st["dens"].copy()
        st["dens"][CELL] = -st["dens"][CELL]
        disc.set_state(st)
        rep = disc.step()
        assert rep.status == 0 and rep.crashes == 0 and rep.crash_substeps == 0
        assert rep.neg_density_substeps >= 1


def test_nonfinite_state_is_an_error(tmp_path):
    from dustyfargoadsg_b200 import Disc, FbError, _ffi, read_par
    par = _oracle.write_par(os.path.join(_oracle.CONFIG_DIR, "iso_128x384.par"), str(tmp_path), Nrad=32, Nsec=96)
    with Disc(read_par(par), noise=1e-4, seed=0) as disc:
        st = disc.download()
        st["dens"] = st["dens"].copy()
        st["dens"][5 * 96 + 7] = np.nan
        disc.set_state(st)
        with pytest.raises(FbError) as e:
            disc.step()
        assert e.value.code == -5  # FB_ERR_NAN
        assert _ffi.FB_ERR[e.value.code] == "FB_ERR_NAN"


def test_substep_cap_is_an_error(tmp_path, monkeypatch):
    from dustyfargoadsg_b200 import Disc, FbError, read_par
    par = _oracle.write_par(os.path.join(_oracle.CONFIG_DIR, "iso_128x384.par"), str(tmp_path), Nrad=32, Nsec=96)
    monkeypatch.setenv("FB_MAX_SUBSTEPS", "1")  # read when the context is created
    with Disc(read_par(par), noise=1e-4, seed=0) as disc:
        with pytest.raises(FbError) as e:
            disc.step()
        assert e.value.code == -7  # FB_ERR_SUBSTEPS
