"""Parameter sweeps of isothermal discs: the seeded draws of the batched
workload (64 discs of uneven grids and parameters advanced together) and the
file plumbing that turns one draw into a reference-style .par + planet .cfg.

A draw varies, around the plain isothermal disc of configs/iso_128x384.par:
  Nrad in {128, 256, 384, 512, 768} with Nsec = 3 Nrad (log grid, 0.4-2.5),
  planet mass q log-uniform in [1e-5, 3e-3],
  alpha log-uniform in [1e-4, 1e-2],
  aspect ratio h uniform in [0.03, 0.1],
  SigmaSlope uniform in [0, 1.5].
The draws come from numpy's Mersenne Twister seeded with the given seed, in
that order per disc, so a seed fixes the whole sweep.
"""
import os

import numpy as np

from . import CONFIG_DIR, Disc, read_par

ISO_PAR = os.path.join(CONFIG_DIR, "iso_128x384.par")
NRADS = (128, 256, 384, 512, 768)


def draw_discs(n, seed, nrads=NRADS):
    """n parameter draws (dicts of .par keys plus 'q')."""
    rng = np.random.RandomState(seed)
    out = []
    for _ in range(n):
        nr = int(nrads[rng.randint(len(nrads))])
        q = float(10.0 ** rng.uniform(np.log10(1e-5), np.log10(3e-3)))
        alpha = float(10.0 ** rng.uniform(-4.0, -2.0))
        h = float(rng.uniform(0.03, 0.1))
        slope = float(rng.uniform(0.0, 1.5))
        out.append(dict(Nrad=nr, Nsec=3 * nr, q=q, AlphaViscosity=alpha, AspectRatio=h, SigmaSlope=slope))
    return out


def write_disc_files(draw, workdir, tag, base_par=ISO_PAR):
    """Write <tag>.par and <tag>.cfg for one draw; returns the .par path."""
    os.makedirs(workdir, exist_ok=True)
    cfg = os.path.join(workdir, tag + ".cfg")
    with open(cfg, "w") as f:
        f.write("# Planet Name   Distance   Mass    Accretion   Feels Disk   Feels Others\n")
        f.write("Planet          1.0        %.9e    0.0         No           No\n" % draw["q"])
    keys = {k: v for k, v in draw.items() if k != "q"}
    keys["PlanetConfig"] = cfg
    keys["OutputDir"] = os.path.join(workdir, tag + "_out")
    lines, seen = [], set()
    with open(base_par) as f:
        for line in f:
            tok = line.split()
            if tok and not tok[0].startswith("#"):
                key = next((k for k in keys if k.upper() == tok[0].upper()), None)
                if key is not None:
                    line = "%s %s\n" % (tok[0], keys[key])
                    seen.add(key)
            lines.append(line)
    for k, v in keys.items():
        if k not in seen:
            lines.append("%s %s\n" % (k, v))
    par = os.path.join(workdir, tag + ".par")
    with open(par, "w") as f:
        f.writelines(lines)
    return par


def make_discs(draws, workdir, noise=1e-4, seed=0, tuning=None):
    """One Disc (device context, initial state uploaded) per draw, with the
    launch shapes of `tuning` (a table of tune.py) where it has the grid."""
    discs = []
    for d, draw in enumerate(draws):
        par = write_disc_files(draw, workdir, "disc%03d" % d)
        discs.append(Disc(read_par(par), noise=noise, seed=seed, tuning=tuning))
    return discs


def orbits_per_dt(params):
    """Orbits at r = 1 advanced by one DT."""
    return float(params.dt) / (2.0 * np.pi)
