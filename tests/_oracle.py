"""Test helpers: run the CPU oracle (the reference's own sequential build,
oracle/_ref/fargo_oracle) and read its full-precision dumps.

TEST INFRASTRUCTURE ONLY -- imported by tests/, bench.py's CPU baseline and
__graft_entry__.smoke() to check results, never by the product path.
"""
import json
import os
import shutil
import subprocess
import tempfile

import numpy as np

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_BIN = os.path.join(REPO, "oracle", "_ref", "fargo_oracle")
DROPIN_BIN = os.path.join(REPO, "oracle", "_ref", "fargo_dropin")
CONFIG_DIR = os.path.join(REPO, "dustyfargoadsg_b200", "configs")


SCALARS = {"PhysicalTime", "OmegaFrame", "LostMass", "MINDT", "MAXDT", "substeps", "nplanets", "nbpart",
           "rng_state"}


def have_oracle():
    return os.path.exists(ORACLE_BIN)


def read_fbd(path):
    """Read an FBD1 dump: JSON header line + raw float64 payload."""
    with open(path, "rb") as f:
        head = f.readline()
        meta = json.loads(head)
        payload = np.frombuffer(f.read(), dtype=np.float64)
    out = {"_nrad": meta["nrad"], "_nsec": meta["nsec"]}
    for name, (off, cnt) in meta["arrays"].items():
        a = payload[off:off + cnt]
        out[name] = float(a[0]) if name in SCALARS else a.copy()
    return out


def write_par(src_par, dst_dir, **keys):
    """Copy a .par file into dst_dir with some keys replaced (absolute
    PlanetConfig, OutputDir inside dst_dir)."""
    keys = {k.upper(): v for k, v in keys.items()}
    lines = []
    seen = set()
    with open(src_par) as f:
        for line in f:
            tok = line.split()
            if tok and not tok[0].startswith("#"):
                k = tok[0].upper()
                if k == "PLANETCONFIG" and "PLANETCONFIG" not in keys:
                    cfg = tok[1]
                    if not os.path.isabs(cfg):
                        cfg = os.path.join(os.path.dirname(os.path.abspath(src_par)), cfg)
                    line = "PlanetConfig %s\n" % cfg
                if k in keys:
                    line = "%s %s\n" % (tok[0], keys[k])
                    seen.add(k)
            lines.append(line)
    for k, v in keys.items():
        if k not in seen:
            lines.append("%s %s\n" % (k, v))
    out = os.path.join(dst_dir, os.path.basename(src_par))
    with open(out, "w") as f:
        f.writelines(lines)
    return out


def run_oracle(par, steps, noise=0.0, seed=0, dump_every=1, stage=False, workdir=None,
               timeout=3600, max_substeps=None, keep=False, extra_keys=None, binary=None, flags=()):
    """Run the reference for `steps` AlgoGas calls (NTOT = steps-1) and
    return (dumps, timing, workdir).  dumps maps tag -> dict of arrays.
    `flags` are the reference's own command-line switches (e.g. "-a" for
    the per-DT mass and momentum lines of main.c:390-395); the run's
    standard output is kept in workdir/stdout.txt."""
    binary = binary or ORACLE_BIN
    if not os.path.exists(binary):
        raise RuntimeError("%s missing: run `make -C oracle all dropin` where the reference is present" % binary)
    wd = workdir or tempfile.mkdtemp(prefix="fb_oracle_")
    out = os.path.join(wd, "out")
    os.makedirs(out, exist_ok=True)
    keys = {"Ntot": max(steps - 1, 0), "OutputDir": out, "Ninterm": max(steps, 1) * 1000}
    if extra_keys and "Ninterm" in extra_keys:
        keys.pop("Ninterm")
    keys.update(extra_keys or {})
    p = write_par(par, wd, **keys)
    env = dict(os.environ)
    env.update(ORACLE_DUMP_DIR=os.path.join(wd, "dump"), ORACLE_DUMP_EVERY=str(dump_every),
               ORACLE_SEED=str(seed), ORACLE_TIMING_FILE=os.path.join(wd, "timing.json"))
    if noise:
        env["ORACLE_NOISE"] = repr(float(noise))
    if stage:
        env["ORACLE_STAGE_DUMP"] = "1"
    if max_substeps:
        env["ORACLE_MAX_SUBSTEPS"] = str(int(max_substeps))
    r = subprocess.run([binary] + list(flags) + [p], cwd=wd, env=env, stdout=subprocess.PIPE,
                       stderr=subprocess.PIPE, timeout=timeout)
    with open(os.path.join(wd, "stdout.txt"), "wb") as f:
        f.write(r.stdout)
    if r.returncode != 0:
        raise RuntimeError("oracle failed (%d): %s" % (r.returncode, r.stderr[-2000:].decode(errors="replace")))
    dumps = {}
    ddir = os.path.join(wd, "dump")
    if os.path.isdir(ddir):
        for fn in sorted(os.listdir(ddir)):
            if fn.endswith(".fbd"):
                dumps[fn[:-4]] = read_fbd(os.path.join(ddir, fn))
        dtf = os.path.join(ddir, "stage_transport_dt.txt")
        if os.path.exists(dtf):
            dumps["stage_dt"] = float(open(dtf).read())
    timing = None
    tf = os.path.join(wd, "timing.json")
    if os.path.exists(tf):
        timing = json.load(open(tf))
    if not keep and workdir is None:
        shutil.rmtree(wd, ignore_errors=True)
    return dumps, timing, wd


def rel_err(a, b, floor=0.0):
    """max |a-b| / max(|b|) over the array (scale-relative error)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    scale = max(np.max(np.abs(b)), floor)
    if scale == 0.0:
        return float(np.max(np.abs(a - b)))
    return float(np.max(np.abs(a - b)) / scale)


def cell_rel_err(a, b):
    """max over cells of |a-b| / |b|, for strictly positive fields (density,
    energy): the per-cell relative error.  Cells where b is exactly zero (ring
    nrad of a PolarGrid, which the step never writes for these fields) must
    match exactly."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    zero = b == 0.0
    if np.any(a[zero] != 0.0):
        return float("inf")
    return float(np.max(np.abs(a[~zero] - b[~zero]) / np.abs(b[~zero])))
