"""Learned opening criterion: the MLP, its training data and its training.

For a 32-body group of the walk and a relative-criterion budget alpha (one of
the ladder of bh_mac_ladder()), the MLP predicts log10 of the group's RMS
relative force error against the FP64 direct sum.  A learned walk (macMode 2)
gives every group the largest budget whose prediction meets the target.

Training data are made by the engine itself: seeded snapshots (disk galaxies
and mergers, evolved a few steps), a sample of whole groups per snapshot, one
walk per ladder budget, and FP64 direct-sum labels of the sampled bodies
(bh_direct_sum_f64).  Training runs on the GPU with the library's BF16
tensor-core forward/backward kernels and Adam (bh_mlp_train_epoch).

    python -m cudagravitydemo_b200.learned --out cudagravitydemo_b200/data/mac_mlp.f32
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import time
from pathlib import Path

import numpy as np

from . import _native as N
from . import _check, _ptr, lib

DATA_DIR = Path(__file__).resolve().parent / "data"
DEFAULT_WEIGHTS = DATA_DIR / "mac_mlp.f32"

# parameter block layout (bh_api.h): W1[8][32] b1[32] W2[32][32] b2[32] W3[32] b3 mean[8] inv_std[8]
OFF = {"W1": (0, (8, 32)), "b1": (256, (32,)), "W2": (288, (32, 32)), "b2": (1312, (32,)), "W3": (1344, (32,)),
       "b3": (1376, (1,)), "mean": (1377, (8,)), "inv_std": (1385, (8,))}
assert OFF["inv_std"][0] + 8 == N.MLP_PARAMS and OFF["mean"][0] == N.MLP_TRAINED


def unpack(params: np.ndarray) -> dict:
    """Views of the named blocks of a parameter vector."""
    return {k: params[o:o + int(np.prod(s))].reshape(s) for k, (o, s) in OFF.items()}


def init_params(mean: np.ndarray, std: np.ndarray, seed: int = 0) -> np.ndarray:
    """He-initialised weights, zero biases and the given input normalisation."""
    rng = np.random.default_rng(seed)
    p = np.zeros(N.MLP_PARAMS, np.float32)
    u = unpack(p)
    u["W1"][:] = rng.normal(0, np.sqrt(2 / 8), (8, 32))
    u["W2"][:] = rng.normal(0, np.sqrt(2 / 32), (32, 32))
    u["W3"][:] = rng.normal(0, np.sqrt(1 / 32), 32)
    u["mean"][:] = mean
    u["inv_std"][:] = 1.0 / np.maximum(std, 1e-6)
    return p


def mac_ladder() -> np.ndarray:
    a = np.zeros(N.MAC_CANDIDATES, np.float32)
    _check(lib().bh_mac_ladder(a.ctypes.data), "bh_mac_ladder")
    return a


def load_weights(path: Path | str | None = None) -> np.ndarray:
    path = Path(path) if path else DEFAULT_WEIGHTS
    if not path.exists():
        raise FileNotFoundError(f"{path}: no trained MLP (python -m cudagravitydemo_b200.learned)")
    p = np.fromfile(path, dtype="<f4")
    if p.size != N.MLP_PARAMS or not np.all(np.isfinite(p)):
        raise ValueError(f"{path}: expected {N.MLP_PARAMS} finite float32 values")
    return p


def save_weights(params: np.ndarray, path: Path | str, meta: dict) -> None:
    path = Path(path)
    path.parent.mkdir(parents=True, exist_ok=True)
    np.asarray(params, "<f4").tofile(path)
    path.with_suffix(".json").write_text(json.dumps(meta, indent=1, sort_keys=True) + "\n")


# -------------------------------------------------------------- kernels
def forward(params_dev, X_dev, stream=None):
    """MLP outputs of the rows of X (device tensors)."""
    import torch
    rows = int(X_dev.shape[0])
    Y = torch.empty(rows, dtype=torch.float32, device=X_dev.device)
    _check(lib().bh_mlp_forward(_ptr(params_dev), _ptr(X_dev), rows, _ptr(Y), stream), "bh_mlp_forward")
    return Y


def loss_grad(params_dev, X_dev, Y_dev, stream=None):
    """(gradient of the mean squared error, sum of squared errors)."""
    import torch
    grad = torch.empty(N.MLP_TRAINED, dtype=torch.float32, device=X_dev.device)
    loss = torch.empty(1, dtype=torch.float32, device=X_dev.device)
    _check(lib().bh_mlp_loss_grad(_ptr(params_dev), _ptr(X_dev), _ptr(Y_dev), int(X_dev.shape[0]), _ptr(grad),
                                  _ptr(loss), stream), "bh_mlp_loss_grad")
    return grad, loss


class Trainer:
    """Adam over device-resident training rows (bh_mlp_train_epoch)."""

    def __init__(self, params: np.ndarray, device="cuda"):
        import torch
        self.torch = torch
        self.P = torch.from_numpy(np.asarray(params, np.float32).copy()).to(device)
        self.grad = torch.zeros(N.MLP_TRAINED, dtype=torch.float32, device=device)
        self.m = torch.zeros_like(self.grad)
        self.v = torch.zeros_like(self.grad)
        self.loss = torch.zeros(1, dtype=torch.float32, device=device)
        self.step = C.c_int(0)

    def epoch(self, X_dev, Y_dev, batch: int, lr: float) -> float:
        """One pass; returns the mean squared error seen during it."""
        self.loss.zero_()
        rows = int(X_dev.shape[0])
        _check(lib().bh_mlp_train_epoch(_ptr(self.P), _ptr(X_dev), _ptr(Y_dev), rows, _ptr(self.grad),
                                        _ptr(self.m), _ptr(self.v), batch, C.byref(self.step), lr, _ptr(self.loss),
                                        None), "bh_mlp_train_epoch")
        return float(self.loss.item()) / rows

    def params(self) -> np.ndarray:
        return self.P.cpu().numpy().copy()


# ------------------------------------------------------- training data
def snapshot_rows(sim, groups_per_snapshot: int, rng, theta_cap: float, eps: float, G: float):
    """Rows (X [k*8, 8], Y [k*8]) of one snapshot: sampled whole groups, one
    row per ladder budget, labels from the FP64 direct sum."""
    import torch
    from .accuracy import direct_sum
    from . import Params
    n = sim.n
    feat, ids = sim.group_features()
    full = n // 32
    k = min(groups_per_snapshot, full)
    groups = np.sort(rng.choice(full, size=k, replace=False))
    targets = ids.reshape(-1)[: full * 32].reshape(full, 32)[groups].reshape(-1).astype(np.int32)
    pos, _ = sim.store()
    exact = direct_sum(torch.from_numpy(pos).cuda(), torch.from_numpy(targets).cuda(), eps, G).cpu().numpy()
    exact_mag = np.maximum(np.linalg.norm(exact, axis=1), 1e-300)
    ladder = mac_ladder()
    base = sim.params
    X = np.zeros((k * len(ladder), 8), np.float32)
    Y = np.zeros(k * len(ladder), np.float32)
    for c, a in enumerate(ladder):
        sim.set_params(Params(**{**base.__dict__, "mac_mode": 1, "alpha": float(a), "theta": theta_cap}))
        acc = sim.accelerations()[targets].astype(np.float64)
        rel = np.linalg.norm(acc - exact, axis=1) / exact_mag
        rms = np.sqrt(np.mean(rel.reshape(k, 32) ** 2, axis=1))
        X[c::len(ladder), 0] = np.log10(a)
        X[c::len(ladder), 1:] = feat[groups]
        Y[c::len(ladder)] = np.log10(np.maximum(rms, 1e-12))
    sim.set_params(base)
    return X, Y


def generate(n: int = 1 << 20, snapshots: int = 64, groups_per_snapshot: int = 2048, theta_cap: float = 0.9,
             seed: int = 1000, merger_n: int = 1 << 22, log=print):
    """Training rows from `snapshots` seeded snapshots, in a cycle of four:
    two disk galaxies of n bodies, a two-disk merger of n bodies and one of
    merger_n bodies (eps 0.005, dt 5e-4; mergers at separations 2.5-20 with
    pericentre 2, so that some are in close passage).  Snapshot s is evolved
    1 + 20 * ((s // 4) % 8) steps with the relative criterion (alpha 1e-3) so
    that the last step's |a| exists.  Every fourth holdout snapshot is of each
    kind."""
    from . import Params, Simulation, disk_galaxy, merger
    rng = np.random.default_rng(seed)
    Xs, Ys, snap = [], [], []
    sim = None
    kinds = ("disk", "disk", "merger", "merger-large")
    for s in range(snapshots):
        t0 = time.time()
        kind = kinds[s % 4]
        if kind == "disk":
            pos, vel = disk_galaxy(n, seed=seed + s)
        else:
            sep = float(rng.uniform(2.5, 20.0))
            incl = float(rng.uniform(0.0, 60.0))
            pos, vel = merger(merger_n if kind == "merger-large" else n, separation=sep, inclination=incl,
                              seed=seed + s)
        prm = Params(theta=theta_cap, eps=0.005, G=1.0, dt=5e-4, mac_mode=1, alpha=1e-3)
        if sim is None:
            sim = Simulation(max(n, merger_n), prm)
        sim.set_params(prm)
        sim.load(pos, vel)
        sim.step(1 + 20 * ((s // 4) % 8))
        X, Y = snapshot_rows(sim, groups_per_snapshot, rng, theta_cap, prm.eps, prm.G)
        Xs.append(X)
        Ys.append(Y)
        snap.append(np.full(len(Y), s, np.int32))
        log(f"snapshot {s}: {kind} n {pos.shape[0]} rows {len(Y)} label mean {Y.mean():.3f} "
            f"({time.time() - t0:.1f} s)")
    if sim is not None:
        sim.close()
    return np.concatenate(Xs), np.concatenate(Ys), np.concatenate(snap)


def train(X: np.ndarray, Y: np.ndarray, snap: np.ndarray, epochs: int = 60, batch: int = 4096, lr: float = 3e-3,
          holdout: int = 8, seed: int = 0, log=print):
    """Trains on all snapshots but the last `holdout`; returns (params, meta)."""
    import torch
    val = snap >= snap.max() + 1 - holdout
    Xt, Yt, Xv, Yv = X[~val], Y[~val], X[val], Y[val]
    mean, std = Xt.mean(axis=0), Xt.std(axis=0)
    tr = Trainer(init_params(mean, std, seed))
    rng = np.random.default_rng(seed)
    Xv_d, Yv_d = torch.from_numpy(Xv).cuda(), torch.from_numpy(Yv).cuda()
    hist = []
    for e in range(epochs):
        order = rng.permutation(len(Yt))
        Xd = torch.from_numpy(np.ascontiguousarray(Xt[order])).cuda()
        Yd = torch.from_numpy(np.ascontiguousarray(Yt[order])).cuda()
        lr_e = lr * 0.5 * (1 + np.cos(np.pi * e / epochs))
        tl = tr.epoch(Xd, Yd, batch, lr_e)
        pv = forward(tr.P, Xv_d).cpu().numpy()
        vl = float(np.mean((pv - Yv) ** 2))
        hist.append((tl, vl))
        if e % 10 == 0 or e == epochs - 1:
            log(f"epoch {e}: train mse {tl:.4f}  holdout mse {vl:.4f}")
    params = tr.params()
    pv = forward(tr.P, Xv_d).cpu().numpy()
    meta = {"rows_train": int(len(Yt)), "rows_holdout": int(len(Yv)), "epochs": epochs, "batch": batch, "lr": lr,
            "train_mse": hist[-1][0], "holdout_mse": hist[-1][1],
            "holdout_mse_of_mean": float(np.mean((Yv - Yt.mean()) ** 2)),
            "holdout_mae_dex": float(np.mean(np.abs(pv - Yv))), "ladder": [float(a) for a in mac_ladder()]}
    return params, meta


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--out", default=str(DEFAULT_WEIGHTS))
    ap.add_argument("--n", type=int, default=1 << 20)
    ap.add_argument("--snapshots", type=int, default=64)
    ap.add_argument("--groups", type=int, default=2048)
    ap.add_argument("--epochs", type=int, default=60)
    ap.add_argument("--batch", type=int, default=4096)
    ap.add_argument("--lr", type=float, default=3e-3)
    ap.add_argument("--seed", type=int, default=1000)
    ap.add_argument("--merger-n", type=int, default=1 << 22, help="bodies of the large merger snapshots")
    ap.add_argument("--save-rows", default=None, help="also save the training rows (.npz)")
    a = ap.parse_args(argv)
    t0 = time.time()
    X, Y, snap = generate(a.n, a.snapshots, a.groups, seed=a.seed, merger_n=a.merger_n)
    t1 = time.time()
    if a.save_rows:
        np.savez_compressed(a.save_rows, X=X, Y=Y, snap=snap)
    params, meta = train(X, Y, snap, a.epochs, a.batch, a.lr)
    t2 = time.time()
    meta.update({"n": a.n, "merger_n": a.merger_n, "snapshots": a.snapshots, "groups_per_snapshot": a.groups,
                 "seed": a.seed, "kinds": "cycle of four: disk, disk, merger (n), merger (merger_n)",
                 "generate_s": round(t1 - t0, 1), "train_s": round(t2 - t1, 1)})
    save_weights(params, a.out, meta)
    print(json.dumps(meta))


if __name__ == "__main__":
    main()
