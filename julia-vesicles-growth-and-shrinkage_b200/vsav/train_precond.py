"""Trains the learned psi preconditioner on the GPU from pairs the solver
itself generates.

    python julia-vesicles-growth-and-shrinkage_b200/vsav/train_precond.py [--out PATH] [--crops 20480]

1. Harvest: seeded 512^2 runs with 4 vesicles (the multi2d_512x4 workload,
   dt = 1e-6) advance on the FP64 reference-form solver; during every Step-1
   psi solve the iterates x_k and preconditioned residuals r_k = D^-1 (b - A x_k)
   of the BiCGSTAB are kept (vsav_psi_harvest).  With x* the converged
   solution, e_k = x* - x_k solves A e_k = b - A x_k, so (r_k, e_k) is a
   residual/error pair of the diagonal preconditioner: the network must map
   y = Re IFFT(r_k) (and M_psi) to the part of e = Re IFFT(e_k) that y misses.
2. Crops: 74x74 windows (periodic) of (y / s, (M_psi - 0.075) / 0.025), s the
   RMS of y over the field, with targets (e - y) / s on the central 64x64
   (five valid 3x3 convolutions).  Three in four windows are centred on the
   vesicle interfaces (M_psi < 0.0875), one in four anywhere.
3. Training: Adam on the library's own GPU forward/backward kernels
   (vsav_net_train) on the residual the corrected preconditioner leaves:
   sum |L(out - t)|^2 / sum |L t|^2 with L the psi operator in grid units
   (c0 - div_h(M grad_h), c0 = (a/dt) dx^2 / S4), because Krylov convergence
   follows the residual, which weighs the preconditioner's error by the
   operator (an error small in L2 but rough at the grid scale leaves a large
   residual).  Every crop is weighted by the inverse mean square residual of
   its field's target (each field counts by its relative residual: smooth
   first residuals, where the diagonal is already close, as much as rough late
   ones), random sign flips of (y, target) make the map odd in the residual,
   and a held-out tenth of the crops validates.

Writes an .npz with theta and the training record (default: the package's
precond_weights.npz, which the bench and the tests load).
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
if PKG not in sys.path:
    sys.path.insert(0, PKG)

from vsav import Handle, ics  # noqa: E402
from vsav.net import Net, init_params  # noqa: E402

S_IN, S_OUT = 74, 64
DEFAULT_OUT = os.path.join(HERE, "precond_weights.npz")


class _Cfg:
    def __init__(self, **kw):
        self.__dict__.update(kw)
        self.Nz = kw.get("Nz", 0)
        self.Lz = kw.get("Lz", 0.0)


def op_field(u, m, c0):
    """L u = c0 u - div_h(M grad_h u) on a periodic field (grid units; the
    stencil of the training loss)."""
    def face(d, ax):
        return 0.5 * (m + np.roll(m, -d, axis=ax))
    out = c0 * u
    for ax in (0, 1):
        for d in (1, -1):
            out = out - face(d, ax) * (np.roll(u, -d, axis=ax) - u)
    return out


def crops_of(y, e, m, rng, n, c0, interface_frac=0.75):
    """n crops of one field: inputs [n][2][74][74], targets [n][64][64], and
    the crops' loss weight: the inverse mean square residual of the whole
    field's target, so every field counts by its relative residual."""
    H, W = y.shape
    s = float(np.sqrt(np.mean(y * y)))
    if s == 0.0:
        return None, None, None
    tms = float(np.mean(op_field((e - y) / s, m, c0) ** 2))
    if tms == 0.0:
        return None, None, None
    mt = (m - 0.075) / 0.025
    iface = np.argwhere(m < 0.0875)
    X = np.empty((n, 2, S_IN, S_IN), np.float32)
    T = np.empty((n, S_OUT, S_OUT), np.float32)
    h = S_IN // 2
    for k in range(n):
        if len(iface) and rng.random() < interface_frac:
            cy, cx = iface[rng.integers(len(iface))]
        else:
            cy, cx = rng.integers(H), rng.integers(W)
        iy = (np.arange(S_IN) + cy - h) % H
        ix = (np.arange(S_IN) + cx - h) % W
        X[k, 0] = y[np.ix_(iy, ix)] / s
        X[k, 1] = mt[np.ix_(iy, ix)]
        c = slice(5, 5 + S_OUT)
        T[k] = ((e[np.ix_(iy, ix)] - y[np.ix_(iy, ix)]) / s)[c, c]
    return X, T, np.full(n, 1.0 / tms, np.float32)


def harvest(ncrops, seeds, steps_per_run, per_field, rng, log, c0):
    Xs, Ts, Ws = [], [], []
    total = 0
    for seed in seeds:
        kw, phi, psi, _ = ics.workload("multi2d_512x4", seed=seed)
        kw["dt"] = 1e-6
        h = Handle(_Cfg(**kw), precision="fp64", psi_itmax=40, psi_rtol=1e-13)
        h.init_state(phi, psi)
        h.harvest(12)
        V = h.V
        for n in range(1, steps_per_run + 1):
            h.run(n, 1)
            xk, rk, xs, M = h.harvest_read()
            for k in range(xk.shape[0]):
                for f in range(3 * V):
                    e = xs[f] - xk[k, f]
                    # the converged x* is accurate to ~1e-12 relative: keep errors well above that
                    if np.linalg.norm(e) < 1e-7 * np.linalg.norm(xs[f]):
                        continue
                    X, T, Wt = crops_of(rk[k, f], e, M[f % V], rng, per_field, c0)
                    if X is None:
                        continue
                    Xs.append(X)
                    Ts.append(T)
                    Ws.append(Wt)
                    total += len(X)
            log(f"seed {seed} step {n}: {xk.shape[0]} iterates, {total} crops")
            if total >= ncrops:
                break
        h.close()
        if total >= ncrops:
            break
    X = np.concatenate(Xs)[:ncrops]
    T = np.concatenate(Ts)[:ncrops]
    Wt = np.concatenate(Ws)[:ncrops]
    return X, T, (Wt / Wt.mean()).astype(np.float32)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=DEFAULT_OUT)
    ap.add_argument("--crops", type=int, default=20480)
    ap.add_argument("--steps", type=int, default=8000)
    ap.add_argument("--batch", type=int, default=64)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--seed", type=int, default=0)
    args = ap.parse_args()
    import torch
    t0 = time.time()
    rng = np.random.default_rng(args.seed)
    logs = []

    def log(msg):
        logs.append(msg)
        print(msg, flush=True)

    # psi operator a/dt - S4 div(M grad) in grid units: c0 = (a/dt) dx^2 / S4 (BDF2 a = 1.5)
    kw0 = ics.workload("multi2d_512x4", seed=100)[0]
    c0 = 1.5 / 1e-6 * (kw0["Lx"] / kw0["Nx"]) ** 2 / kw0["S4"]
    X, T, Wt = harvest(args.crops, seeds=range(100, 140), steps_per_run=4, per_field=4, rng=rng, log=log, c0=c0)
    log(f"harvest: {len(X)} crops in {time.time() - t0:.1f} s")
    perm = rng.permutation(len(X))
    nval = len(X) // 10
    val, tr = perm[:nval], perm[nval:]
    dev = torch.device("cuda")
    Xtr = torch.from_numpy(X[tr]).to(dev).contiguous()
    Ttr = torch.from_numpy(T[tr]).to(dev).contiguous()
    Xva = torch.from_numpy(X[val]).to(dev).contiguous()
    Tva = torch.from_numpy(T[val]).to(dev).contiguous()
    Wtr = torch.from_numpy(Wt[tr]).to(dev).contiguous()
    Wva = torch.from_numpy(Wt[val]).to(dev).contiguous()
    net = Net(args.batch * S_IN * S_IN)
    net.set_params(init_params(args.seed))
    # loss of the diagonal preconditioner alone (network output 0) is 1 by construction
    v0 = net.eval(Xva.data_ptr(), Tva.data_ptr(), nval, S_IN, args.batch, w_dev=Wva.data_ptr(), residual_c0=c0)
    log(f"validation loss at init {v0:.4f}")
    record = []
    chunk = 500
    t1 = time.time()
    done = 0
    while done < args.steps:
        nst = min(chunk, args.steps - done)
        # cosine decay of the learning rate, per chunk
        lr = args.lr * 0.5 * (1 + np.cos(np.pi * done / args.steps))
        losses = net.train(Xtr.data_ptr(), Ttr.data_ptr(), len(tr), S_IN, args.batch, nst, lr, seed=args.seed + done,
                           w_dev=Wtr.data_ptr(), flip=True, residual_c0=c0)
        done += nst
        v = net.eval(Xva.data_ptr(), Tva.data_ptr(), nval, S_IN, args.batch, w_dev=Wva.data_ptr(), residual_c0=c0)
        record.append((done, float(lr), float(np.mean(losses)), float(v)))
        log(f"step {done}: lr {lr:.2e} train {np.mean(losses):.4f} val {v:.4f}")
    log(f"training: {args.steps} steps in {time.time() - t1:.1f} s")
    theta = net.get_params()
    meta = {"crops": int(len(X)), "train": int(len(tr)), "val": int(nval), "steps": args.steps,
            "batch": args.batch, "lr": args.lr, "val_loss_init": float(v0), "val_loss": record[-1][3],
            "record": record, "source": "multi2d_512x4 FP64 reference-form psi solves, dt 1e-6",
            "crop": [S_IN, S_OUT], "loss": "residual norm", "c0": c0, "log": logs}
    np.savez(args.out, theta=theta, meta=json.dumps(meta))
    log(f"wrote {args.out}")


if __name__ == "__main__":
    main()
