"""Training and evaluation of the learned bracket network.

Pairs come from the uneven-batch generator (lognormal lengths, median 2,000 points, sigma 1,
clipped to [100, 50,000]; 2D/3D and walk/spline shapes 50/50).  Each pair is labelled by the
plain method on the GPU (endpoint bound, DFD, VE-FD, bisection to 2^-33), its bracket
features come from rfd_features (the same device code the solver uses), and the target is
y = log10(FD / VEFD - 1 + 1e-13).  The network is trained on the GPU by its own forward and
backward kernels (rfd_model_train_step: pinball loss of the 5% / 95% quantiles, Adam).

VE-FD is a lower bound that equals FD within the 2^-33 stop tolerance for most pairs (97% of
this generator's), and the search always tries the threshold probe VE-FD (1 + 0.999 2^-33)
first when it has the network's bracket: those pairs end in one probe whatever the network
says.  The network's bracket is used only after that probe fails, so it is trained on the
pairs above the threshold (their y is also the only part of the label the plain method's
stop rule resolves: below it, y is the search's stopping noise).

Training runs on standardised inputs and targets; afterwards both affine maps are folded into
the first and last layers, so the saved parameters take the solver's raw features.

    python -m robotfd_b200.train_bracket [--pairs 200000] [--seed 3] [--eval-pairs 4096]
        [--eval-seed 4] [--epochs 150] [--out robotfd_b200/bracket_model.npy]
    python -m robotfd_b200.train_bracket --eval-only robotfd_b200/bracket_model.npy

prints one JSON object: training set, loss curve, and the held-out evaluation (probes with
and without the network, verification failures, solves/s, largest deviation from plain).
"""
import argparse
import json
import os
import sys
import time

import numpy as np

if __package__ in (None, ""):
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import robotfd_b200 as rfd  # noqa: E402

CONFIG = 3          # uneven-batch generator (training and held-out pairs differ by seed)
CHUNK = 4096        # pairs per labelling call
TOL = 2.0 ** -33    # precise stop rule: ub - lb <= 2^-33 ub
THRESHOLD_Y = float(np.log10(0.999 * TOL))  # y of the threshold probe
DEFAULT_OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "bracket_model.npy")


def target(res):
    """y = log10(FD/VEFD - 1 + 1e-13); NaN where VE-FD is missing (degenerate pairs)."""
    fd, ve = res["distance"], res["vefd"]
    if not (ve > 0 and fd == fd) or res["flags"] & rfd.FLAG_DEGENERATE:
        return np.nan
    return float(np.log10(max(fd / ve - 1.0, 0.0) + 1e-13))


def pairs_of(npairs, seed, start, stop):
    """Pairs start..stop-1 of the npairs-pair set (the generator runs in C, GIL released)."""
    from concurrent.futures import ThreadPoolExecutor
    dims, n1, n2, styles, scales, noises = rfd.gen_batch_spec(CONFIG, npairs, seed)

    def one(k):
        return rfd.gen_pair(int(styles[k]), int(dims[k]), int(n1[k]), int(n2[k]),
                            float(scales[k]), float(noises[k]), seed, k)
    with ThreadPoolExecutor(max(1, min(32, os.cpu_count() or 1))) as ex:
        return list(ex.map(one, range(start, stop)))


def label(ctx, npairs, seed, log=None):
    """Features [npairs][400] (float32), targets [npairs] and the plain results' probes."""
    X = np.zeros((npairs, rfd.FEATURE_WIDTH), np.float32)
    y = np.full(npairs, np.nan)
    probes = np.zeros(npairs, np.int32)
    t0 = time.perf_counter()
    for s in range(0, npairs, CHUNK):
        e = min(npairs, s + CHUNK)
        pairs = pairs_of(npairs, seed, s, e)
        Ps, Qs = [p for p, _ in pairs], [q for _, q in pairs]
        res = ctx.distance_batch(Ps, Qs, precise=True)
        ep = np.array([r["endpoint"] for r in res])
        ve = np.array([r["vefd"] for r in res])
        ok = ve > 0
        if ok.any():
            idx = np.nonzero(ok)[0]
            X[s + idx] = ctx.features([Ps[i] for i in idx], [Qs[i] for i in idx], ep[idx], ve[idx])
        y[s:e] = [target(r) for r in res]
        probes[s:e] = [r["probes"] for r in res]
        if log:
            log(f"labelled {e}/{npairs} pairs, {time.perf_counter() - t0:.1f} s")
    return X, y, probes


def fold(params, mu, sd, ymu, ysd):
    """Folds x -> (x - mu) / sd into layer 1 and y -> y * ysd + ymu into layer 4."""
    p = params.astype(np.float64).copy()
    n_in, h = rfd.FEATURE_WIDTH, 256
    W1 = p[: h * n_in].reshape(h, n_in)
    b1 = p[h * n_in: h * n_in + h]
    b1 -= W1 @ (mu / sd)
    W1 /= sd[None, :]
    o4 = len(p) - (2 * h + 2)
    W4 = p[o4: o4 + 2 * h].reshape(2, h)
    b4 = p[o4 + 2 * h:]
    W4 *= ysd
    b4[:] = b4 * ysd + ymu
    return p.astype(np.float32)


def train(X, y, epochs=150, batch=512, lr=2e-3, seed=0, device=0, log=None, val_frac=0.2,
          patience=15):
    """Trains a fresh network on the pairs of (X, y) above the threshold; returns it with
    the normalisations folded in, and the per-epoch loss.  A fixed fifth of the pairs is held
    out: the parameters kept are those of the epoch with the lowest held-out pinball loss, and
    training stops after `patience` epochs without improvement (a few thousand tail pairs
    for 234k parameters overfit otherwise, and the quantiles collapse onto each other)."""
    import torch
    ok = np.isfinite(y) & (y > THRESHOLD_Y)
    X, y = X[ok], y[ok]
    perm0 = np.random.default_rng(seed).permutation(len(y))
    nval = int(len(y) * val_frac)
    Xv, yv = X[perm0[:nval]], y[perm0[:nval]]
    X, y = X[perm0[nval:]], y[perm0[nval:]]
    mu = X.mean(0).astype(np.float64)
    sd = X.std(0).astype(np.float64)
    sd[sd < 1e-6] = 1.0
    mu[sd == 1.0] = 0.0
    ymu, ysd = float(np.median(y)), float(max(y.std(), 1e-3))
    Xn = ((X - mu) / sd).astype(np.float32)
    yn = ((y - ymu) / ysd).astype(np.float32)
    dX = torch.from_numpy(Xn).to(f"cuda:{device}")
    dy = torch.from_numpy(yn).to(f"cuda:{device}")
    dXv = torch.from_numpy(((Xv - mu) / sd).astype(np.float32)).to(f"cuda:{device}")
    dyv = torch.from_numpy(((yv - ymu) / ysd).astype(np.float32)).to(f"cuda:{device}")
    model = rfd.Model(device, seed=seed)
    gen = torch.Generator(device=f"cuda:{device}").manual_seed(seed)
    n = len(y)
    batch = min(batch, n)
    steps_per_epoch = max(1, n // batch)
    total = epochs * steps_per_epoch
    losses, val_losses, step = [], [], 0
    best, best_params, since = np.inf, model.get_params(), 0
    for ep in range(epochs):
        perm = torch.randperm(n, generator=gen, device=dX.device)
        acc = 0.0
        for k in range(steps_per_epoch):
            idx = perm[k * batch:(k + 1) * batch]
            xb, yb = dX[idx].contiguous(), dy[idx].contiguous()
            # the network runs on its own stream: the gathers must be complete first
            torch.cuda.current_stream().synchronize()
            cur = lr * 0.5 * (1 + np.cos(np.pi * step / total)) + 1e-5
            acc += model.train_step(xb.data_ptr(), yb.data_ptr(), len(idx), cur)
            step += 1
        losses.append(acc / steps_per_epoch * ysd)
        torch.cuda.current_stream().synchronize()
        _, vl = model.gradients(dXv.data_ptr(), dyv.data_ptr(), len(yv)) if len(yv) else (0, 0.0)
        val_losses.append(vl * ysd)
        if vl < best:
            best, best_params, since = vl, model.get_params(), 0
        else:
            since += 1
        if log and (ep + 1) % 10 == 0:
            log(f"epoch {ep + 1}/{epochs}: pinball loss {losses[-1]:.4f}, held out {val_losses[-1]:.4f}")
        if since >= patience:
            break
    model.set_params(fold(best_params, mu, sd, ymu, ysd))
    return model, (losses, val_losses)


def coverage(ctx, model, Ps, Qs, plain):
    """Per pair above the threshold: whether y lies inside the predicted [q05, q95], the
    bracket's width and the distance of y from its middle, in decades."""
    import torch
    ep = np.array([r["endpoint"] for r in plain])
    ve = np.array([r["vefd"] for r in plain])
    y = np.array([target(r) for r in plain])
    idx = np.nonzero(np.isfinite(y) & (y > THRESHOLD_Y) & (ve > 0))[0]
    if len(idx) == 0:
        return [], [], []
    X = ctx.features([Ps[i] for i in idx], [Qs[i] for i in idx], ep[idx], ve[idx])
    dX = torch.from_numpy(X).cuda(model.device)
    dY = torch.empty((len(idx), 2), dtype=torch.float32, device=dX.device)
    torch.cuda.synchronize()
    model.forward(dX.data_ptr(), len(idx), dY.data_ptr())
    q = dY.cpu().numpy().astype(np.float64)
    lo, hi = np.minimum(q[:, 0], q[:, 1]), np.maximum(q[:, 0], q[:, 1])
    yt = y[idx]
    return (list((yt >= lo) & (yt <= hi)), list(hi - lo), list(np.abs(yt - 0.5 * (lo + hi))))


def evaluate(ctx, model, npairs, seed, log=None):
    """Held-out pairs solved plainly, with the network, and with the threshold probe alone."""
    st = {k: 0 for k in ("plain_probes", "learned_probes", "tol_probes", "widened", "tol_widened",
                         "one_probe", "plain_rounds", "learned_rounds", "tol_rounds", "tail",
                         "tail_plain", "tail_learned", "tail_tol")}
    st.update(plain_s=0.0, learned_s=0.0, tol_s=0.0, max_rel_dev=0.0, max_rel_gap=0.0)
    cover, width, resid = [], [], []
    for s in range(0, npairs, CHUNK):
        e = min(npairs, s + CHUNK)
        pairs = pairs_of(npairs, seed, s, e)
        Ps, Qs = [p for p, _ in pairs], [q for _, q in pairs]
        ctx.distance_batch(Ps[:8], Qs[:8], precise=True)  # workspace sized, kernels loaded
        t0 = time.perf_counter()
        plain = ctx.distance_batch(Ps, Qs, precise=True)
        t1 = time.perf_counter()
        got = ctx.distance_batch(Ps, Qs, precise=True, model=model)
        t2 = time.perf_counter()
        # no network: a bracket at the VE-FD bound itself, i.e. the threshold probe and,
        # when it fails, plain bisection above it
        br = np.array([[r["vefd"] * (1 - 1e-15), r["vefd"]] for r in plain])
        t3 = time.perf_counter()
        tol_only = ctx.distance_batch(Ps, Qs, precise=True, brackets=br)
        t4 = time.perf_counter()
        st["plain_s"] += t1 - t0
        st["learned_s"] += t2 - t1
        st["tol_s"] += t4 - t3
        cov = coverage(ctx, model, Ps, Qs, plain)
        cover += cov[0]
        width += cov[1]
        resid += cov[2]
        st["plain_rounds"] += max(a["probes"] for a in plain)
        st["learned_rounds"] += max(b["probes"] for b in got)
        st["tol_rounds"] += max(c["probes"] for c in tol_only)
        for a, b, c in zip(plain, got, tol_only):
            st["plain_probes"] += a["probes"]
            st["learned_probes"] += b["probes"]
            st["tol_probes"] += c["probes"]
            st["widened"] += bool(b["flags"] & rfd.FLAG_BRACKET_WIDENED)
            st["tol_widened"] += bool(c["flags"] & rfd.FLAG_BRACKET_WIDENED)
            st["one_probe"] += b["probes"] <= 1
            if c["probes"] > 1:  # the threshold probe failed: a tail pair
                st["tail"] += 1
                st["tail_plain"] += a["probes"]
                st["tail_learned"] += b["probes"]
                st["tail_tol"] += c["probes"]
            if a["distance"] > 0:
                st["max_rel_dev"] = max(st["max_rel_dev"],
                                        abs(a["distance"] - b["distance"]) / a["distance"])
                st["max_rel_gap"] = max(st["max_rel_gap"], (b["ub"] - b["lb"]) / b["ub"])
        if log:
            log(f"evaluated {e}/{npairs} pairs")
    n = npairs
    return {
        "pairs": n,
        "mean_probes_plain": st["plain_probes"] / n,
        "mean_probes_learned": st["learned_probes"] / n,
        "probes_saved_fraction": 1 - st["learned_probes"] / max(st["plain_probes"], 1),
        "bracket_verification_failure_rate": st["widened"] / n,
        "one_probe_fraction": st["one_probe"] / n,
        "solves_per_s_plain": n / st["plain_s"],
        "solves_per_s_learned": n / st["learned_s"],
        "probe_rounds_plain": st["plain_rounds"],
        "probe_rounds_learned": st["learned_rounds"],
        "no_network_bracket": {
            "mean_probes": st["tol_probes"] / n,
            "failure_rate": st["tol_widened"] / n,
            "probe_rounds": st["tol_rounds"],
            "solves_per_s": n / st["tol_s"]},
        "tail_pairs": st["tail"],
        "tail_mean_probes": {k: st["tail_" + k] / max(st["tail"], 1)
                             for k in ("plain", "learned", "tol")},
        "tail_quantile_coverage": float(np.mean(cover)) if cover else None,
        "tail_bracket_width_decades_median": float(np.median(width)) if width else None,
        "tail_median_abs_error_decades": float(np.median(resid)) if resid else None,
        "max_rel_deviation_from_plain": st["max_rel_dev"],
        "max_rel_final_gap": st["max_rel_gap"],
    }


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--pairs", type=int, default=200000)
    ap.add_argument("--seed", type=int, default=3)
    ap.add_argument("--eval-pairs", type=int, default=4096)
    ap.add_argument("--eval-seed", type=int, default=4)
    ap.add_argument("--epochs", type=int, default=150)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--out", default=DEFAULT_OUT)
    ap.add_argument("--eval-only", metavar="MODEL", help="evaluate saved parameters, no training")
    ap.add_argument("--save-dataset", metavar="NPZ", help="write the labelled pairs above the "
                    "threshold (features, targets) and the set's statistics")
    ap.add_argument("--dataset", metavar="NPZ", help="train on a file written by --save-dataset "
                    "instead of labelling pairs")
    args = ap.parse_args(argv)

    def log(m):
        print(m, file=sys.stderr, flush=True)

    ctx = rfd.Context(args.device)
    if args.eval_only:
        model = rfd.Model.load(args.eval_only, device=args.device)
        print(json.dumps({"eval": evaluate(ctx, model, args.eval_pairs, args.eval_seed, log),
                          "model": args.eval_only}), flush=True)
        model.close()
        ctx.close()
        return
    t0 = time.perf_counter()
    if args.dataset:
        z = np.load(args.dataset)
        X, y, probes = z["X"], z["y"], z["probes"]
        stats = {k: float(z[k]) for k in ("usable", "mean_plain_probes")}
    else:
        X, y, probes = label(ctx, args.pairs, args.seed, log)
        fin = y[np.isfinite(y)]
        stats = {"usable": float(fin.size), "mean_plain_probes": float(probes.mean())}
        keep = np.isfinite(y) & (y > THRESHOLD_Y)
        X, y, probes = X[keep], y[keep], probes[keep]
        if args.save_dataset:
            np.savez(args.save_dataset, X=X, y=y, probes=probes, **stats)
    t_label = time.perf_counter() - t0
    t0 = time.perf_counter()
    model, losses = train(X, y, args.epochs, lr=args.lr, device=args.device, log=log)
    t_train = time.perf_counter() - t0
    model.save(args.out)
    out = {
        "train": {"pairs": args.pairs, "seed": args.seed, "usable": int(stats["usable"]),
                  "above_threshold": int(len(y)), "label_s": t_label, "train_s": t_train,
                  "epochs": args.epochs, "lr": args.lr,
                  "mean_plain_probes": stats["mean_plain_probes"],
                  "y_quantiles_above": {q: float(np.quantile(y, q)) for q in (0.05, 0.5, 0.95)},
                  "loss_first": losses[0][0], "loss_last": losses[0][-1],
                  "epochs_run": len(losses[0]),
                  "held_out_loss_best": float(min(losses[1])) if losses[1] else None},
        "eval": evaluate(ctx, model, args.eval_pairs, args.eval_seed, log),
        "out": os.path.relpath(args.out),
    }
    print(json.dumps(out), flush=True)
    model.close()
    ctx.close()


if __name__ == "__main__":
    main()
