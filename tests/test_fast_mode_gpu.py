"""The fast build of the library (libfargo_b200_fast.so: fused multiply-adds,
van Leer slope quotients through a refined approximate reciprocal) against
the CPU oracle at the one-DT parity bar of this path: fields within 1e-11
(scale-relative, and per cell for density and energy) after each DT, equal
substep counts.  Its 100-orbit and full-size checks are the `fast` cases of
test_longrun_gpu.py and test_parity_full_gpu.py."""
import os

import pytest

from tests import _oracle

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not _oracle.have_oracle(), reason="oracle not built")]

CFG = _oracle.CONFIG_DIR
TOL_DT = 1e-11

CASES = {
    "iso_128x384": ("iso_128x384.par", {}, 3, ("dens", "vrad", "vtheta")),
    "adiabatic_sg_64x192": ("adiabatic_sg_512x1536.par", dict(Nrad=64, Nsec=192), 2,
                            ("dens", "vrad", "vtheta", "energy")),
    "iso_768x2304": ("iso_768x2304.par", {}, 1, ("dens", "vrad", "vtheta")),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_fast_build_matches_oracle(tmp_path, case):
    from dustyfargoadsg_b200 import Disc, read_par
    name, keys, steps, fields = CASES[case]
    par = _oracle.write_par(os.path.join(CFG, name), str(tmp_path), **keys)
    dumps, _, _ = _oracle.run_oracle(par, steps=steps, noise=1e-4, seed=0, timeout=3000)
    with Disc(read_par(par), noise=1e-4, seed=0, mode="fast") as disc:
        assert b"--fmad=true" in disc.lib.fb_build_info()
        prev = 0
        for s in range(1, steps + 1):
            rep = disc.step()
            ref = dumps["state_%05d" % s]
            out = disc.download()
            assert rep.substeps == int(ref["substeps"]) - prev, "substep count differs"
            prev = int(ref["substeps"])
            errs = {k: _oracle.rel_err(out[k], ref[k]) for k in fields}
            cell = {k: _oracle.cell_rel_err(out[k], ref[k]) for k in ("dens", "energy") if k in fields}
            print(case, "DT", s, "scale-relative", errs, "per cell", cell)
            assert all(e <= TOL_DT for e in errs.values()), errs
            assert all(e <= TOL_DT for e in cell.values()), cell
