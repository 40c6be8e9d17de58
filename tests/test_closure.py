"""Learned closure: the float64 numpy restatement is checked against finite
differences here (CPU), and the GPU kernels (BF16 tensor cores, FP32
accumulation) against the restatement in test_closure_gpu.py."""
import numpy as np

from tests import closure_ref as R


def _geometry(nr, ns, rmin=0.4, rmax=2.5):
    radii = rmin * np.exp(np.arange(nr + 1) / nr * np.log(rmax / rmin))
    surf = np.pi * (radii[1:] ** 2 - radii[:-1] ** 2) / ns
    return radii, surf


def test_reference_gradients_match_finite_differences():
    nr, ns, B = 5, 12, 2
    rng = np.random.RandomState(1)
    _, surf = _geometry(nr, ns)
    params = R.init_params(seed=2, scale=0.5)
    x = rng.uniform(-1, 1, (B, nr, ns, 16))
    y = rng.standard_normal((B, nr, ns)) * 0.1
    sig = rng.uniform(0.5, 2.0, (B, nr))
    scale, wq = 0.02, 1.7
    L, grads = R.loss_and_grads(params, x, y, scale, wq, surf, sig, bf16=False)
    eps = 1e-6
    for l in range(len(params)):
        w, b = params[l]
        for idx in [(0, 4, 0), (3, 8, 2), (w.shape[0] - 1, 0, w.shape[2] - 1), (1, 4, 5)]:
            wp = w.copy()
            wp[idx] += eps
            wm = w.copy()
            wm[idx] -= eps
            pp = list(params)
            pp[l] = (wp, b)
            Lp, _ = R.loss_and_grads(pp, x, y, scale, wq, surf, sig, bf16=False)
            pp[l] = (wm, b)
            Lm, _ = R.loss_and_grads(pp, x, y, scale, wq, surf, sig, bf16=False)
            num = (Lp - Lm) / (2 * eps)
            ana = grads[l][0][idx]
            assert abs(num - ana) <= 1e-6 * max(1.0, abs(num)) + 1e-9, (l, idx, num, ana)
        for o in (0, b.shape[0] - 1):
            bp = b.copy()
            bp[o] += eps
            bm = b.copy()
            bm[o] -= eps
            pp = list(params)
            pp[l] = (w, bp)
            Lp, _ = R.loss_and_grads(pp, x, y, scale, wq, surf, sig, bf16=False)
            pp[l] = (w, bm)
            Lm, _ = R.loss_and_grads(pp, x, y, scale, wq, surf, sig, bf16=False)
            num = (Lp - Lm) / (2 * eps)
            assert abs(num - grads[l][1][o]) <= 1e-6 * max(1.0, abs(num)) + 1e-9, (l, o)


def test_flux_difference_conserves():
    nr, ns = 7, 16
    _, surf = _geometry(nr, ns)
    rng = np.random.RandomState(3)
    O = rng.standard_normal((1, nr, ns, 16))
    sig = rng.uniform(0.5, 2.0, (1, nr))
    dq = R.flux_diff(O, 1.3, surf, sig)
    total = np.sum(dq[0] * surf[:, None])
    assert abs(total) < 1e-12 * np.sum(np.abs(dq[0] * surf[:, None]))


def test_adjoint_is_the_transpose():
    nr, ns = 6, 8
    _, surf = _geometry(nr, ns)
    rng = np.random.RandomState(4)
    O = rng.standard_normal((2, nr, ns, 16))
    O[..., 2:] = 0.0
    G = rng.standard_normal((2, nr, ns))
    sig = rng.uniform(0.5, 2.0, (2, nr))
    lhs = np.sum(R.flux_diff(O, 0.7, surf, sig) * G)
    rhs = np.sum(O * R.flux_diff_adjoint(G, 0.7, surf, sig))
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)


def test_bf16_rounding():
    v = np.array([1.0, 1.00390625, 1.005859375, -3.14159, 1e-20])
    r = R.bf16_round(v)
    assert r[0] == 1.0 and r[1] == 1.0  # halfway, ties to even
    assert r[2] == 1.0078125
    assert abs(r[3] + 3.140625) < 1e-12
