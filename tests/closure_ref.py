"""Float64 numpy restatement of the learned closure (test infrastructure: the
test reference of the GPU kernels in dustyfargoadsg_b200/csrc/fb_closure.cu).

Network: 4 layers of 3x3 convolutions on NHWC arrays [sample][ring][azimuth]
[channel], periodic in azimuth, zero-padded in radius; channels 16 -> 32 ->
32 -> 32 -> 16; GELU after the first three.  Loss: the mass correction built
from the two output face fluxes (scaled by the disc's initial density at the
face) by the flux-difference operator, against targets.

`bf16=True` rounds to bfloat16 where the GPU stores bfloat16 (weights, the
input, hidden activations, every back-propagated pre-activation gradient),
so that the only remaining differences are float32 accumulation order.
"""
import numpy as np
from math import erf

LAYERS = [(16, 32), (32, 32), (32, 32), (32, 16)]
_erf = np.vectorize(erf)


def bf16_round(a):
    """Round float64/float32 values to bfloat16 (nearest, ties to even)."""
    f = np.asarray(a, dtype=np.float32).copy()
    u = f.view(np.uint32)
    lsb = (u >> 16) & 1
    u = (u + 0x7FFF + lsb) & 0xFFFF0000
    return u.view(np.float32).astype(np.float64)


def gelu(x):
    return 0.5 * x * (1.0 + _erf(x / np.sqrt(2.0)))


def gelu_grad(x):
    return 0.5 * (1.0 + _erf(x / np.sqrt(2.0))) + x * np.exp(-0.5 * x * x) / np.sqrt(2.0 * np.pi)


def shift(x, dy, dx):
    """x[b, i+dy, j+dx, c]: periodic in j, zero outside 0..nr-1 in i."""
    out = np.roll(x, -dx, axis=2)
    if dy != 0:
        out = np.roll(out, -dy, axis=1)
        if dy > 0:
            out[:, -dy:] = 0.0
        else:
            out[:, :-dy] = 0.0
    return out


def conv(x, w, b=None):
    """x [B,nr,ns,cin], w [cout,9,cin] -> [B,nr,ns,cout]"""
    y = 0.0
    for tap in range(9):
        dy, dx = tap // 3 - 1, tap % 3 - 1
        y = y + np.einsum("bijc,oc->bijo", shift(x, dy, dx), w[:, tap, :])
    if b is not None:
        y = y + b
    return y


def conv_wgrad(x, dz):
    """dW[o,tap,c] = sum_p dz[p,o] x[p+off(tap),c]"""
    cout, cin = dz.shape[-1], x.shape[-1]
    g = np.zeros((cout, 9, cin))
    for tap in range(9):
        dy, dx = tap // 3 - 1, tap % 3 - 1
        g[:, tap, :] = np.einsum("bijo,bijc->oc", dz, shift(x, dy, dx))
    return g


def conv_data_grad(dz, w):
    """dX[p,c] = sum_{tap,o} w[o,tap,c] dz[p-off(tap),o]"""
    dx_ = 0.0
    for tap in range(9):
        dy, dx = tap // 3 - 1, tap % 3 - 1
        dx_ = dx_ + np.einsum("bijo,oc->bijc", shift(dz, -dy, -dx), w[:, tap, :])
    return dx_


def sig_face(sig):
    """Sigma0 at the radial faces 0..nr (geometric mean; 0 at the edges)."""
    nr = sig.shape[-1]
    f = np.zeros(sig.shape[:-1] + (nr + 1,))
    f[..., 1:nr] = np.sqrt(sig[..., :-1] * sig[..., 1:])
    return f


def flux_diff(O, scale, surf, sig):
    """dSigma [B,nr,ns] from the network output O [B,nr,ns,16]: channel 0 is
    the flux through each cell's inner radial face, channel 1 through its
    lower azimuthal face, in units of scale * Sigma0(face); sig [B,nr]."""
    B, nr, ns, _ = O.shape
    sf = sig_face(sig)  # [B, nr+1]
    fr = O[..., 0] * sf[:, :nr, None]
    fr_out = np.zeros_like(fr)
    fr_out[:, :-1] = O[:, 1:, :, 0] * sf[:, 1:nr, None]
    dft = (O[..., 1] - np.roll(O[..., 1], -1, axis=2)) * sig[:, :, None]
    return scale * ((fr - fr_out) + dft) / surf[None, :, None]


def flux_diff_adjoint(G, scale, surf, sig):
    """dL/dO [B,nr,ns,16] from G = dL/d(dSigma) [B,nr,ns]."""
    B, nr, ns = G.shape
    sf = sig_face(sig)
    g = G / surf[None, :, None]
    gm = np.zeros_like(g)
    gm[:, 1:] = g[:, :-1]
    dO = np.zeros((B, nr, ns, 16))
    dO[..., 0] = scale * sf[:, :nr, None] * (g - gm)
    dO[..., 1] = scale * sig[:, :, None] * (g - np.roll(g, 1, axis=2))
    return dO


def forward(params, x, bf16=True):
    r = bf16_round if bf16 else (lambda a: a)
    acts, zs = [r(x)], []
    h = r(x)
    for l, (w, b) in enumerate(params):
        z = conv(h, r(w), b)
        if l < len(params) - 1:
            zs.append(z)
            h = r(gelu(z))
            acts.append(h)
        else:
            out = z
    return out, acts, zs


def loss_and_grads(params, x, y, scale, w, surf, sig, bf16=True):
    """Loss and [(dW, db)] per layer for samples x [B,nr,ns,16], mass targets
    y [B,nr,ns], initial density profiles sig [B,nr]."""
    r = bf16_round if bf16 else (lambda a: a)
    out, acts, zs = forward(params, x, bf16)
    B, nr, ns, _ = out.shape
    d = flux_diff(out, scale, surf, sig) - y
    n = B * nr * ns
    L = w * np.sum(d ** 2) / n
    G = 2.0 * w * d / n
    dz = r(flux_diff_adjoint(G, scale, surf, sig))
    grads = [None] * len(params)
    for l in range(len(params) - 1, -1, -1):
        wl = r(params[l][0])
        grads[l] = (conv_wgrad(acts[l], dz), dz.sum(axis=(0, 1, 2)))
        if l > 0:
            dz = r(conv_data_grad(dz, wl) * gelu_grad(zs[l - 1]))
    return L, grads


def init_params(seed=0, scale=0.2):
    rng = np.random.RandomState(seed)
    params = []
    for cin, cout in LAYERS:
        params.append((rng.standard_normal((cout, 9, cin)) * scale / np.sqrt(cin),
                       rng.standard_normal(cout) * 0.05))
    return params


def flatten(params):
    w = np.concatenate([p[0].ravel() for p in params]).astype(np.float32)
    b = np.concatenate([p[1].ravel() for p in params]).astype(np.float32)
    return w, b


def unflatten(w, b):
    out, ow, ob = [], 0, 0
    for cin, cout in LAYERS:
        nw = cout * 9 * cin
        out.append((np.asarray(w[ow:ow + nw], dtype=np.float64).reshape(cout, 9, cin),
                    np.asarray(b[ob:ob + cout], dtype=np.float64)))
        ow += nw
        ob += cout
    return out
