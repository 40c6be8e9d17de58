"""Learned coarse-grid closure: data generation from fine runs, training on
the GPU, the corrected coarse solver and its check against the plain fine
method.

The network and its kernels live in libfargo_b200.so (fb_closure_*); this
module drives them:

* samples (`record_samples`): a fine disc and a coarse disc with the same
  radii and parameters; per sample the coarse disc is set to the
  coarse-grained fine state, its features are recorded, the plain method
  advances it one DT, the fine disc advances one DT too, and the target is
  the coarse-graining of the fine result minus the plain coarse result, in
  the conservative variables (mass, angular momentum, radial momentum);
* training (`Closure.train`): Adam on random minibatches, the loss being the
  weighted squared error of the correction the network's face fluxes imply;
* the corrected solver (`run_coarse`): after every DT of the plain coarse
  method, one correction by the network (fb_closure_apply);
* the evaluation (`evaluate`): azimuthally averaged surface density and vortensity
  of the corrected coarse run, the plain coarse run and the coarse-grained
  plain fine run (the reference); the corrected run is accepted only when
  both errors are within 1%, otherwise the fine method is the answer.

    python -m dustyfargoadsg_b200.closure --help
"""
import argparse
import ctypes as C
import json
import os
import tempfile
import time

import numpy as np

from . import Disc, FbError, read_par, sweep
from ._ffi import check, load

TOLERANCE = 0.01  # accepted azimuthally averaged Sigma / vortensity error


def _fp(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class Closure:
    """The network and its device-side training set (fb_closure)."""

    def __init__(self, coarse_disc, capacity=256, batch=8, seed=0):
        self.lib = coarse_disc.lib
        self.c = C.c_void_p()
        check(self.lib.fb_closure_create(coarse_disc.ctx, int(capacity), int(batch), int(seed), C.byref(self.c)),
              "fb_closure_create")
        self.capacity, self.batch, self.count = capacity, batch, 0
        nw, nb = C.c_int(), C.c_int()
        self.lib.fb_closure_num_params(self.c, C.byref(nw), C.byref(nb))
        self.nw, self.nb = nw.value, nb.value

    # -- parameters -------------------------------------------------------
    def get_params(self):
        w, b = np.zeros(self.nw, dtype=np.float32), np.zeros(self.nb, dtype=np.float32)
        check(self.lib.fb_closure_params(self.c, _fp(w), _fp(b), 1), "fb_closure_params")
        s, q = np.zeros(3), np.zeros(3)
        check(self.lib.fb_closure_scales(self.c, _dp(s), _dp(q), 1), "fb_closure_scales")
        return {"w": w, "b": b, "scale": s, "wq": q}

    def set_params(self, d):
        w = np.ascontiguousarray(d["w"], dtype=np.float32)
        b = np.ascontiguousarray(d["b"], dtype=np.float32)
        check(self.lib.fb_closure_params(self.c, _fp(w), _fp(b), 0), "fb_closure_params")
        s = np.ascontiguousarray(d["scale"], dtype=np.float64)
        q = np.ascontiguousarray(d["wq"], dtype=np.float64)
        check(self.lib.fb_closure_scales(self.c, _dp(s), _dp(q), 0), "fb_closure_scales")

    def save(self, path, meta=None):
        d = self.get_params()
        np.savez(path, meta=json.dumps(meta or {}), **d)

    def load(self, path):
        z = np.load(path)
        self.set_params({k: z[k] for k in ("w", "b", "scale", "wq")})
        return json.loads(str(z["meta"]))

    # -- data, training, use --------------------------------------------
    def record(self, coarse_disc, slot, what):
        check(self.lib.fb_closure_record(self.c, coarse_disc.ctx, int(slot), int(what)), "fb_closure_record")
        if what == 2:
            self.count = max(self.count, slot + 1)

    def autoscale(self, count=None):
        check(self.lib.fb_closure_autoscale(self.c, int(count or self.count)), "fb_closure_autoscale")

    def loss(self, first, nb):
        L = C.c_double()
        check(self.lib.fb_closure_loss_grad(self.c, int(first), int(nb), C.byref(L), None, None),
              "fb_closure_loss_grad")
        return L.value

    def train(self, first, count, iters, lr=1e-3, seed=0, batch=None):
        losses = np.zeros(max(iters, 1))
        check(self.lib.fb_closure_train(self.c, int(first), int(count), int(batch or self.batch), int(iters),
                                        float(lr), int(seed), _dp(losses)), "fb_closure_train")
        return losses[:iters]

    def apply(self, coarse_disc):
        check(self.lib.fb_closure_apply(self.c, coarse_disc.ctx), "fb_closure_apply")

    def set_gain(self, gain):
        check(self.lib.fb_closure_set_gain(self.c, float(gain)), "fb_closure_set_gain")

    def close(self):
        if self.c:
            self.lib.fb_closure_destroy(self.c)
            self.c = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def downsample(fine, coarse):
    check(fine.lib.fb_downsample(fine.ctx, coarse.ctx), "fb_downsample")


def disc_pair(draw, workdir, tag, coarse_nr, factor, noise=1e-4, seed=0, coarse_ns=None):
    """Fine and coarse Discs of one parameter draw (same radii); the coarse
    grid has nsec = 3 nrad unless given."""
    coarse_ns = coarse_ns or 3 * coarse_nr
    fine_draw = dict(draw, Nrad=coarse_nr * factor, Nsec=coarse_ns * factor)
    coarse_draw = dict(draw, Nrad=coarse_nr, Nsec=coarse_ns)
    fine = Disc(read_par(sweep.write_disc_files(fine_draw, workdir, tag + "_fine")), noise=noise, seed=seed)
    coarse = Disc(read_par(sweep.write_disc_files(coarse_draw, workdir, tag + "_coarse")))
    return fine, coarse


def record_samples(net, fine, coarse, first_slot, nsamples, every=1):
    """Samples first_slot.. from the fine run, one every `every` DTs of the
    fine disc: each is one DT of the plain coarse method from the
    coarse-grained fine state against the coarse-graining of the fine
    disc's own DT."""
    slot = first_slot
    for _ in range(nsamples):
        downsample(fine, coarse)
        net.record(coarse, slot, 0)
        coarse.step()
        net.record(coarse, slot, 1)
        fine.step()
        downsample(fine, coarse)
        net.record(coarse, slot, 2)
        slot += 1
        for _ in range(every - 1):
            fine.step()
    return slot


def record_rollout_samples(net, fine, coarse, first_slot, nsamples, every=1, horizon=4):
    """Samples on the states the corrected solver itself visits (data
    aggregation: S. Ross, G. Gordon, D. Bagnell, AISTATS 2011): the coarse
    disc starts from the coarse-grained fine state and runs `horizon` DTs of
    the plain method, each followed by the network's correction, beside the
    fine disc; from that corrected state one sample is taken as
    record_samples takes it (features, the plain DT, the coarse-grained fine
    DT), so its target also undoes the drift the corrected run has
    gathered."""
    slot = first_slot
    for _ in range(nsamples):
        downsample(fine, coarse)
        for _ in range(horizon):
            coarse.step()
            net.apply(coarse)
            fine.step()
        net.record(coarse, slot, 0)
        coarse.step()
        net.record(coarse, slot, 1)
        fine.step()
        downsample(fine, coarse)
        net.record(coarse, slot, 2)
        slot += 1
        for _ in range(every - 1):
            fine.step()
    return slot


def train_small(workdir, coarse_nr=16, coarse_ns=64, factor=4, samples=6, iters=60, seed=0):
    """A small end-to-end training run (tests): one disc, a few samples."""
    draw = dict(q=1e-3, AlphaViscosity=1e-3, AspectRatio=0.05, SigmaSlope=0.5)
    fine, coarse = disc_pair(draw, workdir, "small", coarse_nr, factor, noise=1e-3, seed=seed, coarse_ns=coarse_ns)
    net = Closure(coarse, capacity=samples, batch=2, seed=seed)
    try:
        for _ in range(3):
            fine.step()
        record_samples(net, fine, coarse, 0, samples)
        net.autoscale()
        first = net.loss(0, 2)
        losses = net.train(0, samples, iters, lr=3e-3, seed=seed, batch=2)
        last = net.loss(0, 2)
        return {"loss_first": first, "loss_last": last, "train_losses": losses[::10].tolist()}
    finally:
        net.close()
        fine.close()
        coarse.close()


# ------------------------------------------------------------ evaluation
def profiles(disc):
    """Azimuthal means of Sigma and of the vortensity."""
    sm, vm = disc.vortensity()
    return sm, vm


def profile_errors(test, ref):
    """Largest relative deviation over rings of the Sigma profile and of the
    vortensity profile (interface rings 1..nr-1)."""
    es = float(np.max(np.abs(test[0] - ref[0]) / np.abs(ref[0])))
    ev = float(np.max(np.abs(test[1][1:] - ref[1][1:]) / np.abs(ref[1][1:])))
    return es, ev


def run_coarse(coarse, ndt, net=None):
    """ndt DTs of the coarse disc, corrected by `net` after each; GPU time (s)."""
    t = 0.0
    for _ in range(ndt):
        t0 = time.perf_counter()
        coarse.step()
        if net is not None:
            net.apply(coarse)
        t += time.perf_counter() - t0
    return t


def evaluate(net, draw, workdir, tag, coarse_nr, factor, ndt, seed=0, gains=(1.0,)):
    """Fine, plain coarse and corrected coarse runs of one draw from the
    same start; returns errors, times and whether the corrected run stands
    (a corrected run that fails counts as not within tolerance)."""
    fine, coarse = disc_pair(draw, workdir, tag, coarse_nr, factor, seed=seed)
    plain = Disc(coarse.p)
    runs = []
    try:
        downsample(fine, plain)
        t0 = time.perf_counter()
        for _ in range(ndt):
            fine.step()
        t_fine = time.perf_counter() - t0
        t_plain = run_coarse(plain, ndt)
        ref = Disc(coarse.p)
        downsample(fine, ref)  # the reference on the coarse grid
        p_ref = profiles(ref)
        ref.close()
        e_plain = profile_errors(profiles(plain), p_ref)
        fine.close()
        fine = None
        for gain in gains:
            fresh_fine, _ = None, None
            run = {"gain": gain}
            try:
                net.set_gain(gain)
                # restart the corrected run from the same coarse start
                start, _c = disc_pair(draw, workdir, tag + "_g", coarse_nr, factor, seed=seed)
                downsample(start, coarse)
                start.close()
                _c.close()
                run["t_s"] = run_coarse(coarse, ndt, net)
                e = profile_errors(profiles(coarse), p_ref)
                run["err_sigma"], run["err_vort"] = e
                run["ok"] = bool(np.all(np.isfinite(e)))
            except FbError as exc:
                run["ok"], run["error"] = False, str(exc)
            runs.append(run)
        good = [r for r in runs if r["ok"]]
        best = min(good, key=lambda r: max(r["err_sigma"], r["err_vort"])) if good else None
        accepted = best is not None and max(best["err_sigma"], best["err_vort"]) <= TOLERANCE
        out = {"draw": draw, "dt": ndt, "err_sigma_plain": e_plain[0], "err_vort_plain": e_plain[1],
               "t_fine_s": t_fine, "t_coarse_plain_s": t_plain, "runs": runs, "accepted": accepted,
               "answer": "coarse+cnn" if accepted else "fine (fallback)"}
        if best is not None:
            out.update(gain=best["gain"], err_sigma_cnn=best["err_sigma"], err_vort_cnn=best["err_vort"],
                       t_coarse_cnn_s=best["t_s"], speedup_cnn_vs_fine=t_fine / best["t_s"])
        return out
    finally:
        for d in (fine, coarse, plain):
            if d is not None:
                d.close()


def main(argv=None):
    ap = argparse.ArgumentParser(description="train and evaluate the learned closure")
    ap.add_argument("--coarse-nr", type=int, default=128)
    ap.add_argument("--factor", type=int, default=4)
    ap.add_argument("--train-discs", type=int, default=8)
    ap.add_argument("--val-discs", type=int, default=2, help="of the training discs, held out for early stopping")
    ap.add_argument("--spinup-dt", type=int, default=100, help="fine DTs before the first sample")
    ap.add_argument("--samples-per-disc", type=int, default=24)
    ap.add_argument("--every", type=int, default=10, help="fine DTs between samples")
    ap.add_argument("--iters", type=int, default=2000)
    ap.add_argument("--rollout-rounds", type=int, default=0,
                    help="rounds of samples taken on the corrected solver's own states, each followed by "
                         "more training (data aggregation)")
    ap.add_argument("--rollout-horizon", type=int, default=4, help="corrected DTs before such a sample")
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--eval-discs", type=int, default=4)
    ap.add_argument("--eval-dt", type=int, default=400)
    ap.add_argument("--gains", default="1.0,0.5,0.25", help="correction strengths tried in the evaluation")
    ap.add_argument("--out", default=None, help="model .npz")
    ap.add_argument("--report", default=None, help="JSON report")
    args = ap.parse_args(argv)
    wd = tempfile.mkdtemp(prefix="fb_closure_")
    draws = sweep.draw_discs(args.train_discs, seed=3)
    cap = args.train_discs * args.samples_per_disc * (1 + args.rollout_rounds)
    report = {"coarse": [args.coarse_nr, 3 * args.coarse_nr], "factor": args.factor}
    t0 = time.perf_counter()
    net = None
    slot = 0
    for d, draw in enumerate(draws):
        draw = dict(draw)
        draw.pop("Nrad"), draw.pop("Nsec")
        fine, coarse = disc_pair(draw, wd, "train%02d" % d, args.coarse_nr, args.factor)
        if net is None:
            net = Closure(coarse, capacity=cap, batch=8, seed=3)
        for _ in range(args.spinup_dt):
            fine.step()
        slot = record_samples(net, fine, coarse, slot, args.samples_per_disc, args.every)
        fine.close()
        coarse.close()
        print("disc", d, "samples", slot, "%.1f s" % (time.perf_counter() - t0), flush=True)
    report["t_data_s"] = time.perf_counter() - t0
    # the last `val_discs` discs are held out for validation (early stopping)
    nval = args.val_discs * args.samples_per_disc
    ntrain = slot - nval
    net.autoscale(ntrain)

    def val_loss():
        return float(np.mean([net.loss(ntrain + q, 1) for q in range(0, nval, max(1, nval // 8))]))

    report["loss_val_before"] = best_val = val_loss()
    best = net.get_params()
    t1 = time.perf_counter()
    losses, curve = [], []
    chunk = max(1, args.iters // 12)
    for it in range(0, args.iters, chunk):
        losses.extend(net.train(0, ntrain, min(chunk, args.iters - it), lr=args.lr, seed=4 + it).tolist())
        v = val_loss()
        curve.append([it + chunk, float(np.mean(losses[-chunk:])), v])
        if v < best_val:
            best_val, best = v, net.get_params()
    net.set_params(best)
    # data aggregation: samples on the corrected solver's own states, then
    # more training on everything (the held-out discs stay held out)
    report["rollout"] = []
    ntrain_disc = args.train_discs - args.val_discs
    for rnd in range(args.rollout_rounds):
        t2 = time.perf_counter()
        first_new = slot
        for d, draw in enumerate(draws[:ntrain_disc]):
            draw = dict(draw)
            draw.pop("Nrad"), draw.pop("Nsec")
            fine, coarse = disc_pair(draw, wd, "roll%02d_%02d" % (rnd, d), args.coarse_nr, args.factor)
            for _ in range(args.spinup_dt):
                fine.step()
            try:
                slot = record_rollout_samples(net, fine, coarse, slot, args.samples_per_disc, args.every,
                                              args.rollout_horizon)
            except FbError as exc:  # a corrected run that fails contributes no samples
                print("rollout disc", d, "failed:", exc, flush=True)
            fine.close()
            coarse.close()
        # the new samples go behind the validation block: train on both ranges
        for it in range(0, args.iters, chunk):
            n = min(chunk, args.iters - it)
            losses.extend(net.train(0, ntrain, (n + 1) // 2, lr=args.lr, seed=100 * rnd + it).tolist())
            if slot > first_new:
                losses.extend(net.train(first_new, slot - first_new, n // 2, lr=args.lr,
                                        seed=100 * rnd + it + 1).tolist())
            v = val_loss()
            curve.append([len(losses), float(np.mean(losses[-chunk:])), v])
            if v < best_val:
                best_val, best = v, net.get_params()
        net.set_params(best)
        report["rollout"].append({"round": rnd, "samples": slot - first_new, "t_s": time.perf_counter() - t2,
                                  "loss_val_best": best_val})
        print("rollout round", rnd, report["rollout"][-1], flush=True)
    report["t_train_s"] = time.perf_counter() - t1
    report["loss_train_first"], report["loss_train_last"] = float(losses[0]), float(np.mean(losses[-50:]))
    report["loss_val_best"] = best_val
    report["curve_iter_train_val"] = curve
    print("training", report, flush=True)
    evals = []
    for d, draw in enumerate(sweep.draw_discs(args.eval_discs, seed=4)):
        draw = dict(draw)
        draw.pop("Nrad"), draw.pop("Nsec")
        r = evaluate(net, draw, wd, "eval%02d" % d, args.coarse_nr, args.factor, args.eval_dt,
                     gains=[float(g) for g in args.gains.split(",")])
        evals.append(r)
        print("eval", d, r, flush=True)
    report["evaluations"] = evals
    if args.out:
        net.save(args.out, meta={k: v for k, v in report.items() if k != "evaluations"})
    if args.report:
        with open(args.report, "w") as f:
            json.dump(report, f, indent=1)
    net.close()


if __name__ == "__main__":
    main()
