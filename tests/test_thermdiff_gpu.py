"""Thermal diffusion of the energy equation (SubStep0, SourceEuler.c:722-762):
entropy diffusion (ComputeEntropyDiffusion, :1740-1789), explicit radiative
diffusion (ComputeRadiativeDiffusion, :1791-1876, with the time-step limit
of ConditionCFL, :1411-1428) and implicit radiative diffusion by red-black
successive over-relaxation (SORsolver_RadiativeDiffusion, :1878-2052),
alone and together with the radiative cooling that then uses the opacity
recomputed every substep; adiabatic 64 x 192 disc, 3 DTs, against the CPU
oracle (the reference's own build) on the same seeded start.

Tolerance (the one-DT parity bar of this path): fields within 1e-11
(scale-relative), equal substep counts.  The solver's residual norm is
summed in another order than the reference's sequential sweep: this can move
its stopping iteration only for a norm within ~1e-16 of the threshold.  A
run without the diffusion must differ by much more than the bar, or the
test would not see the term at all.
"""
import os

import pytest

from tests import _oracle

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not _oracle.have_oracle(), reason="oracle not built")]

CFG = _oracle.CONFIG_DIR
TOL_DT = 1e-11
BASE = dict(Nrad=64, Nsec=192, SelfGravity="No")

CASES = {
    "entropy": dict(EntropyDiffusion="Yes", Diffusivity="1e-4"),
    "radiative_explicit": dict(RadiativeDiffusion="Explicit"),
    "radiative_implicit": dict(RadiativeDiffusion="Implicit"),
    "entropy_explicit_cooling": dict(EntropyDiffusion="Yes", Diffusivity="1e-4", RadiativeDiffusion="Explicit",
                                     ThermalCooling="Yes"),
    "implicit_cooling": dict(RadiativeDiffusion="Implicit", ThermalCooling="Yes", EntropyDiffusion="Yes",
                             Diffusivity="1e-4"),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_thermal_diffusion_matches_oracle(tmp_path, case):
    from dustyfargoadsg_b200 import Disc, read_par
    keys = dict(BASE, **CASES[case])
    par = _oracle.write_par(os.path.join(CFG, "adiabatic_sg_512x1536.par"), str(tmp_path), **keys)
    p = read_par(par)
    assert p.unsupported == 0 and (p.entropy_diffusion or p.radiative_diffusion)
    steps = 3
    dumps, _, _ = _oracle.run_oracle(par, steps=steps, noise=1e-3, seed=12)
    fields = ("dens", "vrad", "vtheta", "energy")
    with Disc(p, noise=1e-3, seed=12) as disc:
        prev = 0
        for s in range(1, steps + 1):
            rep = disc.step()
            ref = dumps["state_%05d" % s]
            out = disc.download()
            assert rep.substeps == int(ref["substeps"]) - prev, "substep count differs"
            prev = int(ref["substeps"])
            errs = {k: _oracle.rel_err(out[k], ref[k]) for k in fields}
            cell = {k: _oracle.cell_rel_err(out[k], ref[k]) for k in ("dens", "energy")}
            print(case, "DT", s, rep.substeps, errs, cell)
            assert all(e <= TOL_DT for e in errs.values()), errs
            assert all(e <= TOL_DT for e in cell.values()), cell
    # the same disc without the diffusion ends elsewhere
    os.makedirs(str(tmp_path / "plain"))
    plain_keys = {k: v for k, v in keys.items() if k not in ("EntropyDiffusion", "RadiativeDiffusion")}
    plain = _oracle.write_par(os.path.join(CFG, "adiabatic_sg_512x1536.par"), str(tmp_path / "plain"), **plain_keys)
    with Disc(read_par(plain), noise=1e-3, seed=12) as disc:
        for _ in range(steps):
            disc.step()
        quiet = disc.download()
    moved = _oracle.rel_err(quiet["energy"], out["energy"])
    print(case, "energy change from the diffusion", moved)
    assert moved > 1e3 * TOL_DT
