"""The stochastic turbulent potential (MHD L: ApplyLSAOnPotential,
src/turb.c:13-135, called by FillForcesArrays every substep,
src/Pframeforce.c:125-128) against the CPU oracle (the reference's own
build) on the same seeded start.

The modes are drawn on the GPU from the drand48 stream the reference draws
them from (seeded from the .par, after the initial noise when there is
some), so after every DT the stream must sit exactly where the reference's
is, and the fields must agree within the one-DT parity bar, 1e-11
(scale-relative), with equal substep counts.  The turbulent term is summed
as A cos(m phi) + B sin(m phi) instead of cos(m phi - P); the two differ by
the rounding of an argument of up to 1e4 radians times an amplitude of
about 1e-5 of the potential, far below the bar.  A run without the
potential must differ from it by much more than the bar, or the test would
not see the term at all.
"""
import os

import pytest

from tests import _oracle

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not _oracle.have_oracle(), reason="oracle not built")]

CFG = _oracle.CONFIG_DIR
TOL_DT = 1e-11
LSA = dict(MHD="L", NbTurbModes="50", GammaTurb="1e-3", TurbRmin="0.6", TurbRmax="2.0")

CASES = {
    "iso_noise": ("iso_128x384.par", dict(LSA), 1e-3),
    "iso_no_noise": ("iso_128x384.par", dict(LSA), 0.0),
    "iso_high_m_cutoff": ("iso_128x384.par", dict(LSA, HighMCutoff="Yes", NbTurbModes="80"), 1e-3),
    "adiabatic": ("adiabatic_sg_512x1536.par", dict(LSA, SelfGravity="No", TurbRmin="0.5", TurbRmax="3.0"),
                  1e-3),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_turbulent_potential_matches_oracle(tmp_path, case):
    from dustyfargoadsg_b200 import Disc, read_par
    name, keys, noise = CASES[case]
    par = _oracle.write_par(os.path.join(CFG, name), str(tmp_path), Nrad=64, Nsec=192, **keys)
    p = read_par(par)
    assert p.unsupported == 0 and p.mhd_lsa == 1
    steps = 3
    dumps, _, _ = _oracle.run_oracle(par, steps=steps, noise=noise, seed=11)
    fields = ("dens", "vrad", "vtheta") + (("energy",) if p.energy_equation else ())
    with Disc(p, noise=noise, seed=11) as disc:
        prev = 0
        for s in range(1, steps + 1):
            rep = disc.step()
            ref = dumps["state_%05d" % s]
            out = disc.download()
            assert rep.substeps == int(ref["substeps"]) - prev, "substep count differs"
            prev = int(ref["substeps"])
            assert disc.lsa_stream() == int(ref["rng_state"]), "turbulent modes' draws out of step"
            errs = {k: _oracle.rel_err(out[k], ref[k]) for k in fields}
            print(case, "DT", s, rep.substeps, errs)
            assert all(e <= TOL_DT for e in errs.values()), errs
    # the same disc without the turbulent potential ends elsewhere
    os.makedirs(str(tmp_path / "plain"))
    plain = _oracle.write_par(os.path.join(CFG, name), str(tmp_path / "plain"),
                              Nrad=64, Nsec=192, **{k: v for k, v in keys.items() if k != "MHD"})
    with Disc(read_par(plain), noise=noise, seed=11) as disc:
        for _ in range(steps):
            disc.step()
        quiet = disc.download()
    moved = _oracle.rel_err(quiet["vrad"], out["vrad"])
    print(case, "vrad change from the turbulent potential", moved)
    assert moved > 1e3 * TOL_DT

