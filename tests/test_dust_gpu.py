"""GPU parity of the Lagrangian dust particles (SemiUpdateDustPositions,
interpolation, UpdateDustVelocities) inside whole AlgoGas DTs, against the
CPU oracle run on the same seed.

Tolerances (FP64 parity bar of this path): particle positions and velocities within
1e-10 (scale-relative, max|gpu - ref| / max|ref|), gas fields within 1e-11,
and the drand48 stream of the turbulent kicks at exactly the reference's
position after every DT (the GPU draws the same Gaussian deviates, in
parallel, from the same stream).
"""
import os

import numpy as np
import pytest

from tests import _oracle

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not _oracle.have_oracle(), reason="oracle not built")]

CFG = _oracle.CONFIG_DIR
DUST = os.path.join(CFG, "dust_256x768.par")
ADI = os.path.join(CFG, "adiabatic_sg_512x1536.par")
TOL_GAS = 1e-11
TOL_DUST = 1e-10
DUST_KEYS = ("pc_r", "pc_th", "pc_vr", "pc_vth")

CASES = {
    # small grains (St ~ 1e-7): short-friction-time approximation, kicks
    "sfta_kicks": (DUST, dict(Nrad=64, Nsec=192, NbPart=2000, RminDust=0.6, RmaxDust=1.8), 3),
    # 10 cm - 1 m grains (St ~ 1e-2..1): semi-implicit integrator with the planet,
    # second interpolation (WRITEDUSTDENSITY), and the DUSTFEEDBACK substep
    # bound of half the minimum stopping time
    "implicit_feedback": (DUST, dict(Nrad=64, Nsec=192, NbPart=3000, SizeMinPart=0.1, SizeMaxPart=1.0,
                                     SizePartSlope=1.0, RminDust=0.6, RmaxDust=1.8, WriteDustDensity="Yes",
                                     DustFeedback="Yes"), 3),
    # energy equation + self-gravity: particles feel the disc's SG field
    "selfgravity": (ADI, dict(Nrad=64, Nsec=192, NbPart=2000, SizeMinPart=1e-4, SizeMaxPart=1e-1,
                              SizePartSlope=3.5, RhoPart=2.7, DustSlope=0.0, RminDust=0.5, RmaxDust=3.0,
                              DustFeelTurb="Yes"), 2),
}


def _rel(a, b):
    return _oracle.rel_err(np.asarray(a), np.asarray(b))


@pytest.mark.parametrize("case", sorted(CASES))
def test_particles_match_oracle(tmp_path, case):
    from dustyfargoadsg_b200 import Disc, read_par
    src, keys, steps = CASES[case]
    par = _oracle.write_par(src, str(tmp_path), **keys)
    dumps, _, _ = _oracle.run_oracle(par, steps=steps, noise=1e-4, seed=1)
    p = read_par(par)
    assert p.unsupported == 0
    with Disc(p, noise=1e-4, seed=1) as disc:
        init = disc.dust()
        ref0 = dumps["state_init"]
        for k in ("pc_r", "pc_th", "pc_size"):
            np.testing.assert_array_equal(init[k], ref0[k], err_msg=k)
        # Keplerian start; with self-gravity corrected by the azimuthal mean
        # of our SG field, which agrees with FFTW's to ~1e-15
        for k in ("pc_vr", "pc_vth"):
            assert _rel(init[k], ref0[k]) <= 1e-13, k
        # Stokes numbers of the interpolation call of main.c:287
        assert _rel(init["pc_stokes"], ref0["pc_stokes"]) <= 1e-12
        assert init["pc_rng_x"] == int(ref0["rng_state"])
        prev = 0
        for s in range(1, steps + 1):
            rep = disc.step()
            ref = dumps["state_%05d" % s]
            out = disc.download()
            dust = disc.dust()
            assert rep.substeps == int(ref["substeps"]) - prev, "substep count differs"
            prev = int(ref["substeps"])
            gas = {k: _rel(out[k], ref[k]) for k in ("dens", "vrad", "vtheta", "energy")}
            dus = {k: _rel(dust[k], ref[k]) for k in DUST_KEYS}
            st = _rel(dust["pc_stokes"], ref["pc_stokes"])
            print(case, "DT", s, "substeps", rep.substeps, "gas", gas, "dust", dus, "stokes", st,
                  "kicks", dust["pc_kicks"])
            assert all(e <= TOL_GAS for e in gas.values()), gas
            assert all(e <= TOL_DUST for e in dus.values()), dus
            assert st <= TOL_DUST
            assert dust["pc_rng_x"] == int(ref["rng_state"]), "random stream out of step"


def test_kicks_use_the_stream(tmp_path):
    """Turbulent kicks on: the stream advances by at least two uniforms per
    pair of kicks, and turning the kicks off leaves it untouched."""
    from dustyfargoadsg_b200 import Disc, read_par
    par = _oracle.write_par(DUST, str(tmp_path), Nrad=32, Nsec=96, NbPart=500, RminDust=0.7, RmaxDust=1.6)
    with Disc(read_par(par), seed=4) as disc:
        x0 = disc.dust()["pc_rng_x"]
        disc.step()
        d = disc.dust()
        assert d["pc_kicks"] > 0 and d["pc_rng_x"] != x0
    par = _oracle.write_par(DUST, str(tmp_path), Nrad=32, Nsec=96, NbPart=500, RminDust=0.7, RmaxDust=1.6,
                            DustFeelTurb="No")
    with Disc(read_par(par), seed=4) as disc:
        x0 = disc.dust()["pc_rng_x"]
        disc.step()
        d = disc.dust()
        assert d["pc_kicks"] == 0 and d["pc_rng_x"] == x0
