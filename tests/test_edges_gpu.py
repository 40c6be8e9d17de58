"""The inner and outer edges other than the wall (ApplyBoundaryCondition,
SideEuler.c:1102-1131): OpenBoundary (SideEuler.c:300-410), its Kley &
Nelson variant (INNERBOUNDARY K) and NonReflectingBoundary
(SideEuler.c:569-794), isothermal and adiabatic, against the CPU oracle (the
reference's own build) on the same seeded start.

Tolerance (the one-DT parity bar of this path): fields within 1e-11
(scale-relative) after each DT, equal substep counts.  The non-reflecting
edge takes ring means, which the GPU sums in a tree order: its rounding
stays at the 1e-16 level of those means.
"""
import os

import numpy as np
import pytest

from tests import _oracle

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not _oracle.have_oracle(), reason="oracle not built")]

CFG = _oracle.CONFIG_DIR
TOL_DT = 1e-11

CASES = {
    "open_iso": ("iso_128x384.par", dict(InnerBoundary="OPEN")),
    "knopen_iso": ("iso_128x384.par", dict(InnerBoundary="KNOPEN")),
    "nonreflecting_iso": ("iso_128x384.par", dict(InnerBoundary="NONREFLECTING")),
    "open_adiabatic": ("adiabatic_sg_512x1536.par", dict(InnerBoundary="OPEN", SelfGravity="No")),
    "nonreflecting_adiabatic": ("adiabatic_sg_512x1536.par", dict(InnerBoundary="NONREFLECTING",
                                                                  SelfGravity="No")),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_edges_match_oracle(tmp_path, case):
    from dustyfargoadsg_b200 import Disc, read_par
    name, keys = CASES[case]
    par = _oracle.write_par(os.path.join(CFG, name), str(tmp_path), Nrad=64, Nsec=192, **keys)
    p = read_par(par)
    assert p.unsupported == 0 and p.wall_boundary == 0
    steps = 3
    dumps, _, _ = _oracle.run_oracle(par, steps=steps, noise=1e-3, seed=7)
    fields = ("dens", "vrad", "vtheta") + (("energy",) if p.energy_equation else ())
    with Disc(p, noise=1e-3, seed=7) as disc:
        prev = 0
        for s in range(1, steps + 1):
            rep = disc.step()
            ref = dumps["state_%05d" % s]
            out = disc.download()
            assert rep.substeps == int(ref["substeps"]) - prev, "substep count differs"
            prev = int(ref["substeps"])
            errs = {k: _oracle.rel_err(out[k], ref[k]) for k in fields + ("energy",)}
            print(case, "DT", s, rep.substeps, errs)
            if not all(e <= TOL_DT for e in errs.values()):  # where: the rings of the largest differences
                ns = p.nsec
                for k in ("dens", "energy", "vrad"):
                    d = np.abs(out[k] - ref[k]).reshape(-1, ns).max(axis=1)
                    print(k, "worst rings", np.argsort(d)[::-1][:6].tolist(), d[np.argsort(d)[::-1][:6]].tolist())
            assert all(e <= TOL_DT for e in errs.values()), errs


@pytest.mark.parametrize("opacity", ["BellLin", "constant", "irradiated", "luminosity"])
def test_thermal_cooling_matches_oracle(tmp_path, opacity):
    """Radiative cooling in SubStep3 (SourceEuler.c:1201-1290), with the Bell &
    Lin opacities of the initial state
    (ComputeOpacities, SourceEuler.c:1608-1701, which the reference computes
    once, in InitEuler) or an imposed constant one, and with the star's
    irradiation as a background temperature or from its luminosity;
    adiabatic 64 x 192 disc, 3 DTs, fields within 1e-11."""
    from dustyfargoadsg_b200 import Disc, read_par
    keys = dict(Nrad=64, Nsec=192, SelfGravity="No", BetaCooling="No", ThermalCooling="Yes")
    if opacity == "constant":
        keys.update(SetConstantOpacity="Yes", ImposedConstantOpacity="0.5")
    if opacity == "irradiated":  # a background temperature profile (SourceEuler.c:1218-1226)
        keys.update(StellarIrradiation="Yes", BackgroundTemperature="30.0", SlopeBackgroundTemperature="-0.5")
    if opacity == "luminosity":  # heating by the star's imposed luminosity (SourceEuler.c:1227-1268)
        keys.update(StellarIrradiation="L", StellarLuminosity="1.0", FlaringIndex="0.25")
    par = _oracle.write_par(os.path.join(CFG, "adiabatic_sg_512x1536.par"), str(tmp_path), **keys)
    p = read_par(par)
    assert p.unsupported == 0 and p.thermal_cooling == 1
    steps = 3
    dumps, _, _ = _oracle.run_oracle(par, steps=steps, noise=1e-3, seed=8)
    with Disc(p, noise=1e-3, seed=8) as disc:
        prev = 0
        for s in range(1, steps + 1):
            rep = disc.step()
            ref = dumps["state_%05d" % s]
            out = disc.download()
            assert rep.substeps == int(ref["substeps"]) - prev, "substep count differs"
            prev = int(ref["substeps"])
            errs = {k: _oracle.rel_err(out[k], ref[k]) for k in ("dens", "vrad", "vtheta", "energy")}
            print("thermal cooling", opacity, "DT", s, rep.substeps, errs)
            assert all(e <= TOL_DT for e in errs.values()), errs


def _state_from(init, fields):
    st = {k: init[k] for k in ("SigmaMed", "EnergyMed", "VthetaMed", "VradMed", "GLOBAL_SoundSpeed", "PhysicalTime",
                               "OmegaFrame", "LostMass", "MINDT", "MAXDT", "pl_mass", "pl_x", "pl_y", "pl_vx",
                               "pl_vy", "stardiscbarycenter_x", "stardiscbarycenter_y")}
    st.update(fields)
    return st


@pytest.mark.parametrize("case", sorted(CASES))
def test_edges_stage_matches_oracle(tmp_path, case):
    """ApplyBoundaryCondition alone (fb_stage FB_STAGE_BOUNDARY) on the
    reference's own input of its first call: within 1e-12 of its output (the
    ring means of the non-reflecting edge are summed in another order)."""
    from dustyfargoadsg_b200 import Disc, _ffi, read_par
    name, keys = CASES[case]
    par = _oracle.write_par(os.path.join(CFG, name), str(tmp_path), Nrad=64, Nsec=192, **keys)
    d, _, _ = _oracle.run_oracle(par, steps=1, noise=1e-3, seed=7, stage=True)
    inp, ref = d["stage_bc_in"], d["stage_bc_out"]
    with Disc(read_par(par), state=_state_from(d["state_init"], {k: inp[k] for k in
                                                                 ("dens", "vrad", "vtheta", "energy")})) as disc:
        disc.stage(_ffi.FB_STAGE_BOUNDARY, d["stage_dt"])
        out = disc.download()
    ns = 192
    errs = {k: _oracle.rel_err(out[k], ref[k]) for k in ("dens", "vrad", "vtheta", "energy")}
    print(case, "stage", errs)
    for k in ("dens", "energy", "vrad", "vtheta"):
        dd = np.abs(out[k] - ref[k]).reshape(-1, ns).max(axis=1)
        if dd.max() > 0:
            print(k, "worst rings", np.argsort(dd)[::-1][:4].tolist(), dd[np.argsort(dd)[::-1][:4]].tolist())
    assert all(e <= 1e-12 for e in errs.values()), errs
