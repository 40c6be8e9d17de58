"""Launch-shape autotuner: times the candidate shapes of the per-cell,
azimuthal-transport and radial-transport kernels (fb_tune) on one disc of
each grid size of the batched sweep and keeps a table of the fastest,

    {"iso": {"128x384": {"cell_block": .., "azi_cells_per_thread": ..,
                         "rad_columns": .., "rad_rings": .., "ms_per_substep": ..}, ...},
     "energy": {...}}

which Disc(..., tuning=table) and the batch apply per grid.  Each timed disc
is also recorded in a manifest line (its parameters, the shapes tried and
the result) so that the sweep's runs can be reused as training inputs.

    python -m dustyfargoadsg_b200.tune [--out FILE] [--substeps N] [--energy]
"""
import argparse
import ctypes as C
import json
import os
import tempfile

from . import Disc, read_par, sweep
from ._ffi import FbTuning, check

DEFAULT_TABLE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "configs", "tuning_b200.json")
FIELDS = ("cell_block", "azi_cells_per_thread", "rad_columns", "rad_rings", "azi_variant")


def grid_key(nr, ns):
    return "%dx%d" % (nr, ns)


def tune_disc(disc, substeps=4):
    """Run fb_tune on a Disc; returns the table entry."""
    t = FbTuning()
    ms = C.c_double()
    check(disc.lib.fb_tune(disc.ctx, int(substeps), C.byref(t), C.byref(ms)), "fb_tune", disc.ctx)
    entry = {f: int(getattr(t, f)) for f in FIELDS}
    entry["ms_per_substep"] = ms.value
    return entry


def load_table(path=DEFAULT_TABLE):
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def lookup(table, nr, ns, energy):
    return (table or {}).get("energy" if energy else "iso", {}).get(grid_key(nr, ns))


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=DEFAULT_TABLE)
    ap.add_argument("--manifest", default=None, help="JSON-lines manifest of the tuned discs")
    ap.add_argument("--substeps", type=int, default=4)
    ap.add_argument("--nrads", default=",".join(str(n) for n in sweep.NRADS))
    ap.add_argument("--energy", action="store_true", help="also tune the adiabatic (energy) kernels")
    args = ap.parse_args(argv)
    table = load_table(args.out)
    wd = tempfile.mkdtemp(prefix="fb_tune_")
    manifest = []
    kinds = [("iso", {})] + ([("energy", {"EnergyEquation": "Yes", "AdiabaticIndex": 1.4})] if args.energy else [])
    for kind, extra in kinds:
        for nr in [int(x) for x in args.nrads.split(",")]:
            draw = dict(Nrad=nr, Nsec=3 * nr, q=1e-3, AlphaViscosity=1e-3, AspectRatio=0.05, SigmaSlope=0.5)
            draw.update(extra)
            par = sweep.write_disc_files(draw, wd, "%s_%d" % (kind, nr))
            with Disc(read_par(par), noise=1e-4, seed=0) as disc:
                disc.step()  # a developed flow, not the axisymmetric start
                entry = tune_disc(disc, args.substeps)
            table.setdefault(kind, {})[grid_key(nr, 3 * nr)] = entry
            manifest.append({"kind": kind, "draw": draw, "tuning": entry})
            print(kind, grid_key(nr, 3 * nr), entry, flush=True)
    os.makedirs(os.path.dirname(os.path.abspath(args.out)), exist_ok=True)
    with open(args.out, "w") as f:
        json.dump(table, f, indent=1, sort_keys=True)
    if args.manifest:
        with open(args.manifest, "a") as f:
            for m in manifest:
                f.write(json.dumps(m) + "\n")


if __name__ == "__main__":
    main()
