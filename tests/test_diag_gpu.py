"""Vortensity and azimuthal-mean diagnostics (no reference counterpart) on
the GPU against a float64 numpy restatement of the same definitions, on a
disc state evolved for two DTs so that the velocities are non-trivial."""
import os

import numpy as np
import pytest

from tests import _oracle

pytestmark = pytest.mark.gpu


def vortensity_numpy(rho, vr, vt, rinf, rmed, nr, ns, dphi, omega_frame):
    rho, vr, vt = (a.reshape(nr + 1, ns) for a in (rho, vr, vt))
    xi = np.zeros((nr + 1, ns))
    i = np.arange(1, nr)[:, None]
    jm = np.roll(np.arange(ns), 1)
    drvt = (rmed[i] * vt[1:nr] - rmed[i - 1] * vt[0:nr - 1]) / (rmed[i] - rmed[i - 1])
    dvr = (vr[1:nr] - vr[1:nr][:, jm]) * (1.0 / dphi)
    omega = (drvt - dvr) / rinf[i] + 2.0 * omega_frame
    sig = 0.25 * (rho[1:nr] + rho[0:nr - 1] + rho[1:nr][:, jm] + rho[0:nr - 1][:, jm])
    xi[1:nr] = omega / sig
    return xi


def test_vortensity_and_profiles(tmp_path):
    from dustyfargoadsg_b200 import Disc, read_par
    par = _oracle.write_par(os.path.join(_oracle.CONFIG_DIR, "iso_128x384.par"), str(tmp_path),
                            Nrad=64, Nsec=192)
    p = read_par(par)
    with Disc(p, noise=1e-4, seed=0) as disc:
        disc.step()
        disc.step()
        st = disc.download()
        sm, vm, field = disc.vortensity(field=True)
    nr, ns = p.nrad, p.nsec
    # the geometry of FillPolar1DArrays, log spacing
    radii = p.rmin * np.exp(np.arange(nr + 1) / nr * np.log(p.rmax / p.rmin))
    rinf = radii[:nr]
    rmed = 2.0 / 3.0 * (radii[1:] ** 3 - radii[:-1] ** 3) / (radii[1:] ** 2 - radii[:-1] ** 2)
    dphi = (p.pmax - p.pmin) / ns
    ref = vortensity_numpy(st["dens"], st["vrad"], st["vtheta"], rinf, rmed, nr, ns, dphi, p.omegaframe)
    assert _oracle.rel_err(field, ref.ravel()) <= 1e-12
    np.testing.assert_allclose(sm, st["dens"].reshape(nr + 1, ns)[:nr].mean(axis=1), rtol=1e-13, atol=0)
    np.testing.assert_allclose(vm[1:], ref[1:nr].mean(axis=1), rtol=1e-12, atol=0)
    assert vm[0] == 0.0
    # Keplerian disc: vortensity ~ Omega/(2 Sigma) > 0 away from the planet
    assert np.all(vm[1:] > 0)
