"""Learned closure on the GPU: the BF16 tensor-core forward and backward
kernels against the float64 restatement (tests/closure_ref.py, which
rounds to bfloat16 where the GPU stores bfloat16), conservation of the
applied corrections, conservative coarse-graining, and that training lowers
the loss."""
import ctypes as C
import os

import numpy as np
import pytest

from tests import _oracle
from tests import closure_ref as R

pytestmark = pytest.mark.gpu
ISO = os.path.join(_oracle.CONFIG_DIR, "iso_128x384.par")


def _fp(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _geometry(p):
    nr, ns = p.nrad, p.nsec
    radii = p.rmin * np.exp(np.arange(nr + 1) / nr * np.log(p.rmax / p.rmin))
    surf = np.pi * (radii[1:] ** 2 - radii[:-1] ** 2) / ns
    rmed = 2.0 / 3.0 * (radii[1:] ** 3 - radii[:-1] ** 3) / (radii[1:] ** 2 - radii[:-1] ** 2)
    return radii, surf, rmed


def _closure(disc, capacity, batch, seed=0):
    from dustyfargoadsg_b200 import _ffi
    c = C.c_void_p()
    _ffi.check(disc.lib.fb_closure_create(disc.ctx, capacity, batch, seed, C.byref(c)), "fb_closure_create")
    return c


def test_kernels_match_reference(tmp_path):
    from dustyfargoadsg_b200 import Disc, _ffi, read_par
    par = _oracle.write_par(ISO, str(tmp_path), Nrad=8, Nsec=64)
    p = read_par(par)
    nr, ns, B = p.nrad, p.nsec, 2
    _, surf, _ = _geometry(p)
    params = R.init_params(seed=5, scale=0.6)
    rng = np.random.RandomState(6)
    x = R.bf16_round(rng.uniform(-1, 1, (B, nr, ns, 16)))
    y = rng.standard_normal((B, nr, ns)) * 0.05
    sig = rng.uniform(0.5, 2.0, (B, nr)).astype(np.float32).astype(np.float64)
    scale, w = 0.02, 1.5
    with Disc(p) as disc:
        lib = disc.lib
        c = _closure(disc, 4, B)
        try:
            wt, bt = R.flatten(params)
            _ffi.check(lib.fb_closure_params(c, _fp(wt), _fp(bt), 0), "params")
            sc, wq = np.array([scale, 1.0, 1.0]), np.array([w, 1.0, 1.0])
            _ffi.check(lib.fb_closure_scales(c, _dp(sc), _dp(wq), 0), "scales")
            for s in range(B):
                xs = np.ascontiguousarray(x[s], dtype=np.float32)
                ys = np.zeros((3, nr, ns), dtype=np.float32)
                ys[0] = y[s]
                ss = np.ascontiguousarray(sig[s], dtype=np.float32)
                _ffi.check(lib.fb_closure_set_sample(c, s, _fp(xs), _fp(ys), _fp(ss)), "sample")
            # forward of sample 0
            out = np.zeros(nr * ns * 16, dtype=np.float32)
            _ffi.check(lib.fb_closure_infer(c, None, 0, _fp(out)), "infer")
            ref_out, _, _ = R.forward(params, x[:1], bf16=True)
            e_out = np.linalg.norm(out - ref_out.ravel()) / np.linalg.norm(ref_out)
            # loss and gradients of both samples
            nw, nb = C.c_int(), C.c_int()
            lib.fb_closure_num_params(c, C.byref(nw), C.byref(nb))
            gw = np.zeros(nw.value, dtype=np.float32)
            gb = np.zeros(nb.value, dtype=np.float32)
            L = C.c_double()
            _ffi.check(lib.fb_closure_loss_grad(c, 0, B, C.byref(L), _fp(gw), _fp(gb)), "loss_grad")
        finally:
            lib.fb_closure_destroy(c)
    Lr, grads = R.loss_and_grads(params, x, y, scale, w, surf, sig, bf16=True)
    rw, rb = R.flatten([(g[0], g[1]) for g in grads])
    print("forward rel err", e_out, "loss", L.value, Lr)
    assert e_out < 2e-3
    assert abs(L.value - Lr) <= 1e-3 * Lr
    ow = ob = 0
    for l, (cin, cout) in enumerate(R.LAYERS):
        n = cout * 9 * cin
        ew = np.linalg.norm(gw[ow:ow + n] - rw[ow:ow + n]) / np.linalg.norm(rw[ow:ow + n])
        eb = np.linalg.norm(gb[ob:ob + cout] - rb[ob:ob + cout]) / max(np.linalg.norm(rb[ob:ob + cout]), 1e-30)
        print("layer", l, "grad rel err W", ew, "b", eb)
        assert ew < 1e-2 and eb < 1e-2, (l, ew, eb)
        ow += n
        ob += cout


def _totals(st, p):
    nr, ns = p.nrad, p.nsec
    _, surf, rmed = _geometry(p)
    rho = st["dens"].reshape(nr + 1, ns)[:nr]
    vt = st["vtheta"].reshape(nr + 1, ns)[:nr]
    mass = np.sum(surf[:, None] * rho)
    J = 0.5 * (np.roll(rho, 1, axis=1) + rho) * rmed[:, None] * vt
    return mass, np.sum(surf[:, None] * J)


def test_apply_conserves_mass_and_angular_momentum(tmp_path):
    from dustyfargoadsg_b200 import Disc, _ffi, read_par
    par = _oracle.write_par(ISO, str(tmp_path), Nrad=32, Nsec=128)
    p = read_par(par)
    with Disc(p, noise=1e-3, seed=1) as disc:
        disc.step()
        c = _closure(disc, 1, 1, seed=7)
        try:
            w, b = R.flatten(R.init_params(seed=8, scale=1.0))
            _ffi.check(disc.lib.fb_closure_params(c, _fp(w), _fp(b), 0), "params")
            m0, j0 = _totals(disc.download(), p)
            _, surf, _ = _geometry(p)
            # fluxes of ~1e-2 of the local mass per DT
            scale = np.array([1e-2 * np.mean(surf), 1.0, 1.0])
            _ffi.check(disc.lib.fb_closure_scales(c, _dp(scale), _dp(np.ones(3)), 0), "scales")
            before = disc.download()
            _ffi.check(disc.lib.fb_closure_apply(c, disc.ctx), "apply")
            after = disc.download()
        finally:
            disc.lib.fb_closure_destroy(c)
    m1, j1 = _totals(after, p)
    dm = np.max(np.abs(after["dens"] - before["dens"])) / np.max(before["dens"])
    print("relative change of the fields", dm, "mass", (m1 - m0) / m0, "J", (j1 - j0) / j0)
    assert dm > 1e-6  # the corrections are not negligible...
    assert abs(m1 - m0) <= 1e-13 * m0  # ...yet mass and angular momentum hold
    assert abs(j1 - j0) <= 1e-13 * abs(j0)


def test_downsample_conserves_mass(tmp_path):
    from dustyfargoadsg_b200 import Disc, _ffi, read_par
    fine_par = _oracle.write_par(ISO, str(tmp_path), Nrad=64, Nsec=256)
    os.makedirs(str(tmp_path / "c"))
    coarse_par = _oracle.write_par(ISO, str(tmp_path / "c"), Nrad=16, Nsec=64)
    pf, pc = read_par(fine_par), read_par(coarse_par)
    with Disc(pf, noise=1e-3, seed=2) as fine, Disc(pc) as coarse:
        fine.step()
        _ffi.check(fine.lib.fb_downsample(fine.ctx, coarse.ctx), "downsample")
        sf, sc = fine.download(), coarse.download()
    mf, _ = _totals(sf, pf)
    mc, _ = _totals(sc, pc)
    assert abs(mf - mc) <= 1e-13 * mf
    assert sc["PhysicalTime"] == sf["PhysicalTime"]


def test_training_lowers_the_loss(tmp_path):
    from dustyfargoadsg_b200 import closure
    res = closure.train_small(str(tmp_path), coarse_nr=16, coarse_ns=64, factor=4, samples=6, iters=60)
    print(res)
    assert res["loss_last"] < 0.7 * res["loss_first"]
