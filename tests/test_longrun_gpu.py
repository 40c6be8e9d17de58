"""100 orbits of the 128 x 384 isothermal disc against the oracle.

tests/golden/longrun_iso_128x384.npz holds the oracle's (the reference's own
sequential build) state after 2,000 DTs (100 orbits) from the seeded start
(white noise 1e-4, seed 0), and its own `-a` monitoring lines: GasTotalMass
(SideEuler.c:15) and GasMomentum (SideEuler.c:114) after every DT
(main.c:390-395).  tests/golden/make_longrun.py made it.

Tolerances (the long-run parity bar of this path): after 100 orbits, density
within 1e-8 per cell and radial / azimuthal velocity within 1e-8
scale-relative; the same total substep count; disc mass and angular momentum
tracking the reference's after every DT (1e-10 of their initial values), and
their drift over the run no larger than the reference's (to 1e-6 of it, plus
1e-14 of the initial value for the summation order).
"""
import os

import numpy as np
import pytest

from tests import _oracle

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "longrun_iso_128x384.npz")
pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not os.path.exists(GOLDEN), reason="fixture missing")]

TOL_FIELD = 1e-8
TOL_TRACK = 1e-10


@pytest.mark.parametrize("mode", ["parity", "fast"])
def test_hundred_orbits_match_oracle(mode):
    """Both builds of the library: the parity one, and the fast one (fused
    multiply-adds, approximate-reciprocal slopes) against the same bar."""
    from dustyfargoadsg_b200 import Disc, read_par
    g = np.load(GOLDEN)
    steps = int(g["steps"])
    with Disc(read_par(os.path.join(_oracle.CONFIG_DIR, "iso_128x384.par")), noise=1e-4, seed=0,
              mode=mode) as disc:
        m0, j0 = disc.diagnostics()
        mass, mom, substeps = np.zeros(steps), np.zeros(steps), 0
        for s in range(steps):
            rep = disc.step()
            substeps += rep.substeps
            mass[s], mom[s] = disc.diagnostics()
        out = disc.download()
    assert substeps == int(g["substeps"])
    assert abs(out["PhysicalTime"] - float(g["physical_time"])) <= 1e-12 * float(g["physical_time"])
    errs = {"dens per cell": _oracle.cell_rel_err(out["dens"], g["dens"]),
            "vrad": _oracle.rel_err(out["vrad"], g["vrad"]),
            "vtheta": _oracle.rel_err(out["vtheta"], g["vtheta"])}
    ref_m0, ref_j0 = float(g["mass0"]), float(g["momentum0"])
    track_m = float(np.max(np.abs(mass - g["mass"]))) / ref_m0
    track_j = float(np.max(np.abs(mom - g["momentum"]))) / ref_j0
    drift = {"mass gpu": (mass[-1] - m0) / m0, "mass ref": (g["mass"][-1] - ref_m0) / ref_m0,
             "momentum gpu": (mom[-1] - j0) / j0, "momentum ref": (g["momentum"][-1] - ref_j0) / ref_j0}
    print(mode, "100 orbits:", substeps, "substeps; errors", errs, "tracking", track_m, track_j, "drift", drift)
    assert all(e <= TOL_FIELD for e in errs.values()), errs
    assert abs(m0 - ref_m0) <= 1e-14 * ref_m0 and abs(j0 - ref_j0) <= 1e-14 * abs(ref_j0)
    assert track_m <= TOL_TRACK and track_j <= TOL_TRACK, (track_m, track_j)
    assert abs(mass[-1] - m0) <= abs(g["mass"][-1] - ref_m0) * (1 + 1e-6) + 1e-14 * ref_m0
    assert abs(mom[-1] - j0) <= abs(g["momentum"][-1] - ref_j0) * (1 + 1e-6) + 1e-14 * abs(ref_j0)
