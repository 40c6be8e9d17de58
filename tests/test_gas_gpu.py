"""GPU parity of the gas step against the CPU oracle (the reference's own
sequential build run on the same seeded inputs).

Tolerances (FP64 parity bar of this path): fields within 1e-11 relative after one DT;
single stages within 1e-12.  Errors are scale-relative:
max|gpu - ref| / max|ref| per field.
"""
import os

import numpy as np
import pytest

from tests import _oracle

CFG = _oracle.CONFIG_DIR
ISO = os.path.join(CFG, "iso_128x384.par")
pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not _oracle.have_oracle(), reason="oracle not built")]

FIELDS = ("dens", "vrad", "vtheta")
TOL_DT = 1e-11
TOL_STAGE = 1e-12


def _profiles(init):
    return {k: init[k] for k in ("SigmaMed", "EnergyMed", "VthetaMed", "VradMed", "GLOBAL_SoundSpeed")}


def _state_from(init, fields):
    st = dict(_profiles(init))
    for k in ("PhysicalTime", "OmegaFrame", "LostMass", "MINDT", "MAXDT"):
        st[k] = init[k]
    for k in ("pl_mass", "pl_x", "pl_y", "pl_vx", "pl_vy", "stardiscbarycenter_x", "stardiscbarycenter_y"):
        st[k] = init[k]
    st.update(fields)
    return st


@pytest.fixture(scope="module")
def staged(tmp_path_factory):
    wd = str(tmp_path_factory.mktemp("stage"))
    par = _oracle.write_par(ISO, wd, Nrad=64, Nsec=192)
    dumps, _, _ = _oracle.run_oracle(par, steps=1, noise=1e-4, seed=0, stage=True)
    return par, dumps


def _disc(par, state):
    from dustyfargoadsg_b200 import Disc, read_par
    return Disc(read_par(par), state=state)


def _cmp(out, ref, names, tol, rings=None):
    errs = {}
    for k in names:
        a, b = out[k], ref[k]
        if rings is not None:
            a, b = a[:rings], b[:rings]
        errs[k] = _oracle.rel_err(a, b)
    bad = {k: e for k, e in errs.items() if not e <= tol}
    assert not bad, "errors above %g: %s (all: %s)" % (tol, bad, errs)
    return errs


def test_stage_transport(staged):
    from dustyfargoadsg_b200 import _ffi
    par, d = staged
    inp, out_ref = d["stage_transport_in"], d["stage_transport_out"]
    with _disc(par, _state_from(d["state_init"], {k: inp[k] for k in ("dens", "vrad", "vtheta", "energy")})) as disc:
        disc.stage(_ffi.FB_STAGE_TRANSPORT, d["stage_dt"])
        out = disc.download()
    _cmp(out, out_ref, FIELDS, TOL_STAGE)


def test_stage_viscosity(staged):
    from dustyfargoadsg_b200 import _ffi
    par, d = staged
    inp, out_ref = d["stage_visc_in"], d["stage_visc_out"]
    with _disc(par, _state_from(d["state_init"], {k: inp[k] for k in ("dens", "vrad", "vtheta")})) as disc:
        disc.stage(_ffi.FB_STAGE_VISCOSITY, d["stage_dt"])
        out = disc.download()
    _cmp(out, out_ref, ("vrad", "vtheta"), TOL_STAGE)


def test_stage_boundary_and_damping(staged):
    from dustyfargoadsg_b200 import _ffi
    par, d = staged
    inp = d["stage_bc_in"]
    with _disc(par, _state_from(d["state_init"], {k: inp[k] for k in ("dens", "vrad", "vtheta", "energy")})) as disc:
        disc.stage(_ffi.FB_STAGE_BOUNDARY, d["stage_dt"])
        out = disc.download()
        _cmp(out, d["stage_bc_out"], FIELDS, 0.0)
        disc.stage(_ffi.FB_STAGE_DAMPING, d["stage_dt"])
        out = disc.download()
    _cmp(out, d["stage_damp_out"], FIELDS, TOL_STAGE)


@pytest.mark.parametrize("nrad,nsec,steps", [(32, 96, 3), (128, 384, 2)])
def test_algogas_matches_oracle(tmp_path, nrad, nsec, steps):
    """Whole DTs from the same seeded initial state (noise 1e-4, seed 0)."""
    from dustyfargoadsg_b200 import Disc, read_par
    par = _oracle.write_par(ISO, str(tmp_path), Nrad=nrad, Nsec=nsec)
    dumps, _, _ = _oracle.run_oracle(par, steps=steps, noise=1e-4, seed=0)
    with Disc(read_par(par), noise=1e-4, seed=0) as disc:
        init = disc.download()
        _cmp(init, dumps["state_init"], FIELDS, 0.0)
        for s in range(1, steps + 1):
            rep = disc.step()
            ref = dumps["state_%05d" % s]
            out = disc.download()
            assert rep.substeps == int(ref["substeps"]) - int(dumps["state_%05d" % (s - 1)]["substeps"]
                                                              if s > 1 else 0), "substep count differs"
            errs = _cmp(out, ref, FIELDS, TOL_DT)
            assert abs(out["PhysicalTime"] - ref["PhysicalTime"]) <= 1e-13 * abs(ref["PhysicalTime"])
            print("DT", s, "substeps", rep.substeps, "errors", errs)


ADI = os.path.join(CFG, "adiabatic_sg_512x1536.par")


@pytest.mark.parametrize("nrad,nsec,steps,beta,alpha", [(48, 144, 3, "Yes", "1e-3"), (64, 192, 2, "No", "0.0")])
def test_energy_equation_matches_oracle(tmp_path, nrad, nsec, steps, beta, alpha):
    """Adiabatic gas (SubStep2 energy, SubStep3 pdV + viscous heating + beta
    cooling, energy transport and floor) without self-gravity."""
    from dustyfargoadsg_b200 import Disc, read_par
    par = _oracle.write_par(ADI, str(tmp_path), Nrad=nrad, Nsec=nsec, SelfGravity="No",
                            BetaCooling=beta, AlphaViscosity=alpha)
    dumps, _, _ = _oracle.run_oracle(par, steps=steps, noise=1e-4, seed=3)
    with Disc(read_par(par), noise=1e-4, seed=3) as disc:
        init = disc.download()
        _cmp(init, dumps["state_init"], FIELDS + ("energy",), 0.0)
        prev = 0
        for s in range(1, steps + 1):
            rep = disc.step()
            ref = dumps["state_%05d" % s]
            out = disc.download()
            assert rep.substeps == int(ref["substeps"]) - prev
            prev = int(ref["substeps"])
            errs = _cmp(out, ref, FIELDS + ("energy",), TOL_DT)
            print("energy DT", s, "substeps", rep.substeps, errs)


@pytest.fixture(scope="module")
def sg_case(tmp_path_factory):
    wd = str(tmp_path_factory.mktemp("sg"))
    par = _oracle.write_par(ADI, wd, Nrad=64, Nsec=192)
    dumps, _, _ = _oracle.run_oracle(par, steps=2, noise=1e-4, seed=5)
    return par, dumps


def test_selfgravity_accelerations(sg_case):
    """compute_sgacc of the initial density: our FFT convolution vs the
    reference's (FFTW 2.1.5), scale-relative."""
    from dustyfargoadsg_b200 import _ffi
    par, d = sg_case
    init = d["state_init"]
    with _disc(par, _state_from(init, {k: init[k] for k in ("dens", "vrad", "vtheta", "energy")})) as disc:
        disc.stage(_ffi.FB_STAGE_SELFGRAV, 1.0)
        ar, at = disc.derived(6), disc.derived(7)
    nrs = disc.nr * disc.ns
    e_r = _oracle.rel_err(ar[:nrs], init["sg_accr"][:nrs])
    e_t = _oracle.rel_err(at[:nrs], init["sg_acct"][:nrs])
    print("SG accel errors", e_r, e_t)
    assert e_r < 1e-12 and e_t < 1e-12


@pytest.mark.parametrize("nrad,nsec", [(256, 768), (512, 1536)])
def test_selfgravity_accelerations_large(tmp_path, nrad, nsec):
    """The convolution on the benchmark's grids (2 Nr = 512 and 1024 point
    columns: radix-16 column passes) against FFTW 2.1.5."""
    from dustyfargoadsg_b200 import _ffi
    par = _oracle.write_par(ADI, str(tmp_path), Nrad=nrad, Nsec=nsec)
    d, _, _ = _oracle.run_oracle(par, steps=1, noise=1e-4, seed=5, max_substeps=1)
    init = d["state_init"]
    with _disc(par, _state_from(init, {k: init[k] for k in ("dens", "vrad", "vtheta", "energy")})) as disc:
        disc.stage(_ffi.FB_STAGE_SELFGRAV, 1.0)
        ar, at = disc.derived(6), disc.derived(7)
    nrs = disc.nr * disc.ns
    e_r = _oracle.rel_err(ar[:nrs], init["sg_accr"][:nrs])
    e_t = _oracle.rel_err(at[:nrs], init["sg_acct"][:nrs])
    print("SG accel errors", nrad, nsec, e_r, e_t)
    assert e_r < 1e-12 and e_t < 1e-12


def test_selfgravity_algogas_matches_oracle(sg_case, tmp_path):
    """Whole DTs with energy equation, beta cooling and self-gravity."""
    from dustyfargoadsg_b200 import Disc, read_par
    par, dumps = sg_case
    with Disc(read_par(par), noise=1e-4, seed=5) as disc:
        init = disc.download()
        errs0 = _cmp(init, dumps["state_init"], FIELDS + ("energy",), 1e-13)
        print("SG init", errs0)
        prev = 0
        for s in (1, 2):
            rep = disc.step()
            ref = dumps["state_%05d" % s]
            out = disc.download()
            assert rep.substeps == int(ref["substeps"]) - prev
            prev = int(ref["substeps"])
            errs = _cmp(out, ref, FIELDS + ("energy",), TOL_DT)
            print("SG DT", s, "substeps", rep.substeps, errs)
