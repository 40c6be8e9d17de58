"""Generates tests/golden/longrun_iso_128x384.npz: the oracle (the
reference's own sequential build, oracle/_ref/fargo_oracle) run for 100
orbits (2,000 DTs) on the 128x384 isothermal disc of
dustyfargoadsg_b200/configs/iso_128x384.par, white noise 1e-4 from seed 0.

TEST INFRASTRUCTURE ONLY.  Run where the oracle is built:
    python tests/golden/make_longrun.py
The fixture holds the fields after the last DT (dens, vrad, vtheta), the
substep count, PhysicalTime, LostMass, and the reference's own per-DT
monitoring lines of `-a` (main.c:390-395): GasMomentum (SideEuler.c:114)
and GasTotalMass (SideEuler.c:15) after every DT, printed with %.18g, plus
both quantities of the initial state summed in the reference's loop order
(SideEuler.c:15-27, :114-133) from the initial dump.
"""
import os
import re
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

from tests import _oracle  # noqa: E402

STEPS = 2000
OUT = os.path.join(HERE, "longrun_iso_128x384.npz")


def gas_mass(dens, surf, nrad, nsec):
    """GasTotalMass (SideEuler.c:15-27): sequential sum over active rings."""
    terms = (surf[:nrad, None] * dens[: nrad * nsec].reshape(nrad, nsec)).ravel()
    return float(np.cumsum(terms)[-1])


def gas_momentum(dens, vth, surf, rmed, omega_frame, nrad, nsec):
    """GasMomentum (SideEuler.c:114-133) in the reference's order."""
    d = dens[: nrad * nsec].reshape(nrad, nsec)
    v = vth[: nrad * nsec].reshape(nrad, nsec)
    vn = np.roll(v, -1, axis=1)
    vc = 0.5 * (v + vn) + rmed[:nrad, None] * omega_frame
    terms = (((surf[:nrad, None] * d) * rmed[:nrad, None]) * vc).ravel()
    return float(np.cumsum(terms)[-1])


def main():
    import tempfile
    wd = tempfile.mkdtemp(prefix="fb_longrun_")
    par = _oracle.write_par(os.path.join(_oracle.CONFIG_DIR, "iso_128x384.par"), wd)
    t0 = time.time()
    dumps, timing, wd = _oracle.run_oracle(par, steps=STEPS, noise=1e-4, seed=0, dump_every=STEPS,
                                           workdir=wd, timeout=7200, flags=["-a"])
    wall = time.time() - t0
    txt = open(os.path.join(wd, "stdout.txt"), errors="replace").read()
    mom = [float(x) for x in re.findall(r"Gas Momentum\s*:\s*(\S+)", txt)]
    mass = [float(x) for x in re.findall(r"Gas total Mass\s*:\s*(\S+)", txt)]
    assert len(mom) == STEPS and len(mass) == STEPS, (len(mom), len(mass))
    init, fin = dumps["state_init"], dumps["state_%05d" % STEPS]
    nr, ns = init["_nrad"], init["_nsec"]
    m0 = gas_mass(init["dens"], init["Surf"], nr, ns)
    j0 = gas_momentum(init["dens"], init["vtheta"], init["Surf"], init["Rmed"], init["OmegaFrame"], nr, ns)
    # the restated sums reproduce the reference's printed values on the final state
    assert gas_mass(fin["dens"], init["Surf"], nr, ns) == mass[-1]
    assert gas_momentum(fin["dens"], fin["vtheta"], init["Surf"], init["Rmed"], fin["OmegaFrame"], nr, ns) == mom[-1]
    np.savez_compressed(OUT, dens=fin["dens"], vrad=fin["vrad"], vtheta=fin["vtheta"],
                        substeps=int(fin["substeps"]), physical_time=fin["PhysicalTime"],
                        lost_mass=fin["LostMass"], mass=np.array(mass), momentum=np.array(mom),
                        mass0=m0, momentum0=j0, steps=STEPS, nrad=nr, nsec=ns)
    print("wrote %s: %d substeps in %.0f s; mass drift %.3e, momentum drift %.3e"
          % (OUT, int(fin["substeps"]), wall, (mass[-1] - m0) / m0, (mom[-1] - j0) / j0))


if __name__ == "__main__":
    main()
