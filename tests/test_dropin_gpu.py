"""The drop-in proof: the reference's own main(), init, SendOutput and planet
logs, with AlgoGas answered by libfargo_b200.so through
dustyfargoadsg_b200/host/algogas_dropin.c, against the reference's own
AlgoGas on the same seeded run.  Compares the state after every DT and the
gas*N.dat output files the reference writes."""
import os

import numpy as np
import pytest

from tests import _oracle

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not (_oracle.have_oracle() and os.path.exists(_oracle.DROPIN_BIN)),
                                 reason="oracle / drop-in binaries not built")]


@pytest.mark.parametrize("par_name,keys", [
    ("iso_128x384.par", dict(Nrad=64, Nsec=192)),
    ("adiabatic_sg_512x1536.par", dict(Nrad=64, Nsec=192)),
    ("dust_256x768.par", dict(Nrad=64, Nsec=192, NbPart=2000, RminDust=0.6, RmaxDust=1.8)),
    ("iso_128x384.par", dict(Nrad=64, Nsec=192, MHD="L", NbTurbModes=50, GammaTurb="1e-3", TurbRmin=0.6,
                             TurbRmax=2.0)),
    ("iso_128x384.par", dict(Nrad=64, Nsec=192, Frame="C", InnerBoundary="NONREFLECTING")),
    ("iso_128x384.par", dict(Nrad=64, Nsec=192, Frame="C", ForcedCircular="No", MassTaper="5.0")),
    ("adiabatic_sg_512x1536.par", dict(Nrad=64, Nsec=192, AddNoise="Yes", TempPresc="Yes", BetaCooling="No",
                                       InnerBoundary="OPEN", EntropyDiffusion="Yes", Diffusivity="1e-4")),
])
def test_dropin_matches_reference(tmp_path, par_name, keys):
    src = os.path.join(_oracle.CONFIG_DIR, par_name)
    steps = 5
    par = _oracle.write_par(src, str(tmp_path), **keys)
    wa, wb = str(tmp_path / "ref"), str(tmp_path / "gpu")
    os.makedirs(wa)
    os.makedirs(wb)
    extra = {"Ninterm": 2}
    ref, _, _ = _oracle.run_oracle(par, steps, noise=1e-4, seed=2, workdir=wa, keep=True, extra_keys=extra)
    gpu, _, _ = _oracle.run_oracle(par, steps, noise=1e-4, seed=2, workdir=wb, keep=True, extra_keys=extra,
                                   binary=_oracle.DROPIN_BIN)
    for s in range(1, steps + 1):
        a, b = gpu["state_%05d" % s], ref["state_%05d" % s]
        for k in ("dens", "vrad", "vtheta", "energy"):
            assert _oracle.rel_err(a[k], b[k]) <= 1e-11, (s, k)
        assert abs(a["PhysicalTime"] - b["PhysicalTime"]) <= 1e-13 * b["PhysicalTime"]
        # the frame's angular velocity the binding hands back (planet*.dat prints it)
        assert abs(a["OmegaFrame"] - b["OmegaFrame"]) <= 1e-12 * max(abs(b["OmegaFrame"]), 1.0), s
        if "pc_r" in b:  # particles
            for k in ("pc_r", "pc_th", "pc_vr", "pc_vth", "pc_stokes"):
                assert _oracle.rel_err(a[k], b[k]) <= 1e-10, (s, k)
        # the libc drand48 stream the drop-in hands back (particle kicks,
        # turbulent modes; untouched otherwise)
        assert a["rng_state"] == b["rng_state"], s
    # output files written by the reference's SendOutput (Output.c:178-218)
    nr, ns = keys["Nrad"], keys["Nsec"]
    for n in (0, 1, 2):
        for name in ("gasdens", "gasvrad", "gasvtheta"):
            fa = os.path.join(wa, "out", "%s%d.dat" % (name, n))
            fb = os.path.join(wb, "out", "%s%d.dat" % (name, n))
            xa, xb = np.fromfile(fa), np.fromfile(fb)
            assert xa.size == nr * ns and xb.size == nr * ns
            assert _oracle.rel_err(xb, xa) <= 1e-11, (name, n)
    pa = np.loadtxt(os.path.join(wa, "out", "planet0.dat"))
    pb = np.loadtxt(os.path.join(wb, "out", "planet0.dat"))
    np.testing.assert_allclose(pb, pa, rtol=1e-10, atol=1e-14)
    # the per-DT planet logs of UpdateLog (Force.c:266-328), fed by the GPU's
    # ComputeForce, and the indirect terms of compindirectterm.dat
    # (Output.c): each column within 1e-10 of its largest value (the force
    # sums are added in another order, and torques cancel).  The last two
    # columns of compindirectterm.dat, the barycentre's second difference
    # (SideEuler.c:91-112), divide sums that cancel to ~1e-8 by dt^2: their
    # summation order shows at 1e-6 of the direct term's size.  A torque or
    # power is a sum of cell contributions that cancel; where the planet is
    # still light (MassTaper) the net is 1e-6 of the contributions' absolute
    # sum, and a 1e-14 difference in the fields moves it by 1e-10 of itself.
    # Those columns are held to 1e-10 of their largest value or 1e-14 of the
    # absolute sum (the rounding of a sum of 1e4 terms, sqrt(N) eps),
    # whichever is larger.
    from dustyfargoadsg_b200 import read_par
    p = read_par(par)
    fabs, fstar = _abs_force_sums(os.path.join(wa, "out"), p, nr, ns, pa)
    for name in ("tqwk0.dat", "indtq0.dat", "compindirectterm.dat"):
        la = np.atleast_2d(np.loadtxt(os.path.join(wa, "out", name)))
        lb = np.atleast_2d(np.loadtxt(os.path.join(wb, "out", name)))
        assert la.shape == lb.shape and la.shape[0] >= 2, (name, la.shape, lb.shape)
        scale = np.maximum(np.max(np.abs(la), axis=0), 1e-300)
        tol = 1e-10 * scale
        if name == "tqwk0.dat":
            r_p = np.hypot(pa[0, 1], pa[0, 2])
            v_p = np.hypot(pa[0, 3], pa[0, 4])
            tol[1:5] = np.maximum(tol[1:5], 1e-14 * r_p * fabs)
            tol[5:9] = np.maximum(tol[5:9], 1e-14 * v_p * fabs)
        if name == "indtq0.dat":  # the disc's pull on the star, the same kind of sum
            tol[1] = max(tol[1], 1e-14 * np.hypot(pa[0, 1], pa[0, 2]) * fstar)
        if name == "compindirectterm.dat":
            tol[1:3] = np.maximum(tol[1:3], 1e-14 * fstar)
            tol[3:] = 1e-6 * max(scale[1], scale[2])
        diff = np.abs(lb - la)
        print(name, "max |diff| / column scale", np.max(diff, axis=0) / scale)
        bad = diff > tol
        assert not np.any(bad), (name, np.argwhere(bad).tolist(), la[bad].tolist(), lb[bad].tolist())


def _abs_force_sums(outdir, p, nr, ns, planets):
    """The sizes of the terms two force sums add up, on the reference's
    initial density: over cells, |G m_cell d / (d^2 + eps^2)^(3/2)| for the
    first planet at its starting place (ComputeForce, Force.c:153-236) and
    |G m_cell / r^2| for the star (the disc's pull on the primary,
    SourceEuler.c:482, SideEuler.c:282-298)."""
    rad = np.loadtxt(os.path.join(outdir, "used_rad.dat"))[: nr + 1]
    rinf, rsup = rad[:-1], rad[1:]
    rmed = 2.0 / 3.0 * (rsup ** 3 - rinf ** 3) / (rsup ** 2 - rinf ** 2)
    surf = np.pi * (rsup ** 2 - rinf ** 2) / ns
    dens = np.fromfile(os.path.join(outdir, "gasdens0.dat")).reshape(nr, ns)
    th = 2.0 * np.pi * np.arange(ns) / ns
    x, y = planets[0, 1], planets[0, 2]
    r = np.hypot(x, y)
    eps = p.thicknesssmoothing * p.aspectratio * r ** (1.0 + p.flaringindex)
    d2 = (rmed[:, None] * np.cos(th) - x) ** 2 + (rmed[:, None] * np.sin(th) - y) ** 2
    m = surf[:, None] * np.abs(dens)
    return float(np.sum(m * np.sqrt(d2) / (d2 + eps * eps) ** 1.5)), float(np.sum(m / rmed[:, None] ** 2))


def test_dropin_crash_report(tmp_path):
    """The reference's crash report through the drop-in: the same "Crash!"
    line and the same gas*999.dat files as the reference's own AlgoGas, from
    a start with one negative-energy cell; the run goes on."""
    nr, ns, cell = 48, 144, 20 * 144 + 50
    par = _oracle.write_par(os.path.join(_oracle.CONFIG_DIR, "adiabatic_sg_512x1536.par"), str(tmp_path),
                            Nrad=nr, Nsec=ns, SelfGravity="No", AlphaViscosity="0.0")
    wa, wb = str(tmp_path / "ref"), str(tmp_path / "gpu")
    os.makedirs(wa)
    os.makedirs(wb)
    os.environ["ORACLE_NEGATE_ENERGY"] = str(cell)
    try:
        ref, _, _ = _oracle.run_oracle(par, 2, noise=1e-4, seed=3, workdir=wa, keep=True)
        gpu, _, _ = _oracle.run_oracle(par, 2, noise=1e-4, seed=3, workdir=wb, keep=True,
                                       binary=_oracle.DROPIN_BIN)
    finally:
        del os.environ["ORACLE_NEGATE_ENERGY"]
    crash = [[line for line in open(os.path.join(w, "stdout.txt")).read().splitlines() if "Crash!" in line]
             for w in (wa, wb)]
    assert crash[0] and crash[0] == crash[1]
    for name in ("gasdens", "gasvrad", "gasvtheta", "gasenergy"):
        xa = np.fromfile(os.path.join(wa, "out", "%s999.dat" % name))
        xb = np.fromfile(os.path.join(wb, "out", "%s999.dat" % name))
        assert xa.size == nr * ns and np.array_equal(xa, xb), name
    for k in ("dens", "vrad", "vtheta", "energy"):
        assert _oracle.rel_err(gpu["state_00002"][k], ref["state_00002"][k]) <= 1e-11, k


def test_dropin_restart(tmp_path):
    """-s N restart (Init.c:93-211, main.c:97-100) through the drop-in: the
    reference's own restart code reads the N-th outputs of an earlier run and
    the GPU continues from what it read.  The reference's restart is not
    exact itself (it does not restore everything the run carried, e.g. the
    barycentre history), so the drop-in's next output is compared with the
    reference restarted from the same files: within 1e-11."""
    import shutil
    nr, ns = 64, 192
    par = _oracle.write_par(os.path.join(_oracle.CONFIG_DIR, "adiabatic_sg_512x1536.par"), str(tmp_path),
                            Nrad=nr, Nsec=ns)
    wa = str(tmp_path / "first")
    os.makedirs(wa)
    extra = {"Ninterm": 2}
    _oracle.run_oracle(par, 5, noise=1e-4, seed=2, workdir=wa, keep=True, extra_keys=extra)
    names = ("gasdens", "gasvrad", "gasvtheta", "Temperature")
    runs = {}
    for tag, binary in (("ref", _oracle.ORACLE_BIN), ("gpu", _oracle.DROPIN_BIN)):
        w = str(tmp_path / tag)
        shutil.copytree(os.path.join(wa, "out"), os.path.join(w, "out"))
        for name in names:
            os.remove(os.path.join(w, "out", "%s2.dat" % name))
        _oracle.run_oracle(par, 5, noise=1e-4, seed=2, workdir=w, keep=True, extra_keys=extra, binary=binary,
                           flags=["-s", "1"])
        runs[tag] = w
    for name in names:
        xa = np.fromfile(os.path.join(runs["ref"], "out", "%s2.dat" % name))
        xb = np.fromfile(os.path.join(runs["gpu"], "out", "%s2.dat" % name))
        assert xa.size == nr * ns and xb.size == nr * ns, name
        assert _oracle.rel_err(xb, xa) <= 1e-11, name
