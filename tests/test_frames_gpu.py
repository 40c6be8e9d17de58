"""The frame corotating with the planet (FRAME C: OmegaFrame from the
planet's orbit at the start, src/main.c:228-247, then the angle the planet
turned through at every substep with CorrectVtheta, src/SourceEuler.c:
476-525), the reference's own AddNoise initial perturbation
(src/Pframeforce.c:317-320, seeded) and the energy relaxation TEMPPRESC
(src/SourceEuler.c:1159-1175), in the combinations the reference's example
parameter files use them: a corotating disc with non-reflecting edges, one
with the energy equation and radiative cooling, one with self-gravity, one
with the turbulent potential; a self-gravitating disc with AddNoise,
TempPresc, open inner edge and damping zones.  64 x 192 grids, 3 DTs, against
the CPU oracle (the reference's own build) on the same seeded start.

Tolerance (the one-DT parity bar of this path): fields within 1e-11
(scale-relative), equal substep counts, OmegaFrame and the planet within
1e-12 relative (its GET angle is an arcsine of a cross product, evaluated by
the GPU's libm).
"""
import os

import numpy as np
import pytest

from tests import _oracle

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not _oracle.have_oracle(), reason="oracle not built")]

CFG = _oracle.CONFIG_DIR
TOL_DT = 1e-11
GRID = dict(Nrad=64, Nsec=192)

CASES = {
    "corotating_nonreflecting": ("iso_128x384.par", dict(Frame="C", InnerBoundary="NONREFLECTING"), 1e-3),
    "corotating_free_planet": ("iso_128x384.par", dict(Frame="C", ForcedCircular="No"), 1e-3),
    "corotating_free_planet_short_dt": ("iso_128x384.par", dict(Frame="C", ForcedCircular="No", DT="0.01"), 1e-3),
    "free_planet": ("iso_128x384.par", dict(ForcedCircular="No"), 1e-3),
    "corotating_energy_cooling": ("adiabatic_sg_512x1536.par",
                                  dict(Frame="C", SelfGravity="No", BetaCooling="No", ThermalCooling="Yes"), 1e-3),
    "corotating_selfgravity": ("adiabatic_sg_512x1536.par", dict(Frame="C"), 1e-3),
    "corotating_turbulence": ("iso_128x384.par", dict(Frame="C", MHD="L", NbTurbModes="30", GammaTurb="1e-3",
                                                      TurbRmin="0.6", TurbRmax="2.0"), 1e-3),
    "addnoise_temppresc_open": ("adiabatic_sg_512x1536.par",
                                dict(AddNoise="Yes", TempPresc="Yes", BetaCooling="No", InnerBoundary="OPEN",
                                     PrescTime0="3.0"), 0.0),
    "temppresc_viscosity": ("adiabatic_sg_512x1536.par",
                            dict(TempPresc="Yes", BetaCooling="No", SelfGravity="No", AlphaViscosity="0.0",
                                 Viscosity="1e-5"), 1e-3),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_frame_and_init_options_match_oracle(tmp_path, case):
    from dustyfargoadsg_b200 import Disc, read_par
    name, keys, noise = CASES[case]
    par = _oracle.write_par(os.path.join(CFG, name), str(tmp_path), **dict(GRID, **keys))
    p = read_par(par)
    assert p.unsupported == 0
    steps = 3
    dumps, _, _ = _oracle.run_oracle(par, steps=steps, noise=noise, seed=13)
    fields = ("dens", "vrad", "vtheta") + (("energy",) if p.energy_equation else ())
    init = dumps.get("state_init")
    with Disc(p, noise=noise, seed=13) as disc:
        if init is not None:  # bit for bit, except where the initial self-gravity enters (vtheta)
            for k in fields:
                a, b = disc.fields[k][: p.nrad * p.nsec], init[k][: p.nrad * p.nsec]
                if p.self_gravity and k == "vtheta":
                    assert _oracle.rel_err(a, b) <= 1e-14, "initial " + k
                else:
                    np.testing.assert_array_equal(a, b, err_msg="initial " + k)
        prev = 0
        for s in range(1, steps + 1):
            rep = disc.step()
            ref = dumps["state_%05d" % s]
            out = disc.download()
            assert rep.substeps == int(ref["substeps"]) - prev, "substep count differs"
            prev = int(ref["substeps"])
            errs = {k: _oracle.rel_err(out[k], ref[k]) for k in fields}
            om = disc.st.omega_frame
            print(case, "DT", s, rep.substeps, errs, "OmegaFrame", om, float(ref["OmegaFrame"]),
                  "planet", disc.st.planets.x[0], disc.st.planets.y[0], float(ref["pl_x"][0]), float(ref["pl_y"][0]))
            assert all(e <= TOL_DT for e in errs.values()), errs
            assert abs(om - float(ref["OmegaFrame"])) <= 1e-12 * max(abs(float(ref["OmegaFrame"])), 1e-300) + 1e-300
            if p.corotating:
                assert om != 0.0
            for q in range(disc.st.planets.nb):
                for a, b in ((disc.st.planets.x[q], ref["pl_x"][q]), (disc.st.planets.y[q], ref["pl_y"][q])):
                    assert abs(a - b) <= 1e-12, (q, a, b)


def test_free_planet_single_substep(tmp_path):
    """One substep of a free planet (AdvanceSystemRK5 with the indirect
    term, RungeKunta.c:64-91): the GPU's planet after one short DT (a
    single substep) against the reference's, component by component."""
    from dustyfargoadsg_b200 import Disc, read_par
    par = _oracle.write_par(os.path.join(CFG, "iso_128x384.par"), str(tmp_path), Nrad=64, Nsec=192,
                            ForcedCircular="No", DT="0.01")
    p = read_par(par)
    dumps, _, _ = _oracle.run_oracle(par, steps=1, noise=1e-3, seed=13)
    init, ref = dumps["state_init"], dumps["state_00001"]
    with Disc(p, noise=1e-3, seed=13) as disc:
        disc.download()
        pl = disc.st.planets
        print("uploaded", pl.x[0], pl.y[0], pl.vx[0], pl.vy[0], pl.mass[0])
        print("oracle init", [float(init[k][0]) for k in ("pl_x", "pl_y", "pl_vx", "pl_vy", "pl_mass")])
        rep = disc.step()
        disc.download()
        pl = disc.st.planets
        got = (pl.x[0], pl.y[0], pl.vx[0], pl.vy[0])
    want = tuple(float(ref[k][0]) for k in ("pl_x", "pl_y", "pl_vx", "pl_vy"))
    print("substeps", rep.substeps, "gpu", got, "oracle", want)
    assert rep.substeps == 1
    for a, b in zip(got, want):
        assert abs(a - b) <= 1e-15 * max(1.0, abs(b)), (got, want)
