"""CPU oracle of the learned opening criterion (test infrastructure only).

The learned criterion is an extension of the engine with no counterpart in
the reference, so this restates the engine's own specification:

* the MLP 8 -> 32 -> 32 -> 1 with ReLU on the packed parameter block of
  bh_api.h (W1[8][32] b1 W2[32][32] b2 W3[32] b3 mean[8] inv_std[8]);
* its BF16 form as the tensor-core kernels compute it: normalised inputs,
  weights and hidden activations rounded to bfloat16 (round to nearest even),
  products accumulated in FP32, biases added in FP32;
* the gradient of the mean squared error through that network (the backward
  product through W2 takes bf16 operands, the weight gradients are FP32 sums);
* an FP64 form without rounding, whose analytic gradient is checked against
  central finite differences;
* the group features and the per-group choice of the budget.
"""
from __future__ import annotations

import numpy as np

OFF = {"W1": (0, (8, 32)), "b1": (256, (32,)), "W2": (288, (32, 32)), "b2": (1312, (32,)), "W3": (1344, (32,)),
       "b3": (1376, (1,)), "mean": (1377, (8,)), "inv_std": (1385, (8,))}
TRAINED = 1377
TOTAL = 1393


def blocks(p: np.ndarray) -> dict:
    return {k: p[o:o + int(np.prod(s))].reshape(s) for k, (o, s) in OFF.items()}


def bf16(x) -> np.ndarray:
    """float32 -> nearest bfloat16 (ties to even), returned as float32."""
    u = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def _mm(a, b):
    """FP32 result of a product of FP32-exact operands (float64 sum, rounded)."""
    return (a.astype(np.float64) @ b.astype(np.float64)).astype(np.float32)


def forward_bf16(p: np.ndarray, X: np.ndarray):
    """Outputs and intermediates of the BF16 tensor-core network."""
    w = blocks(np.asarray(p, np.float32))
    X = np.asarray(X, np.float32)
    xn = bf16((X - w["mean"]) * w["inv_std"])
    z1 = _mm(xn, bf16(w["W1"])) + w["b1"]
    h1 = bf16(np.maximum(z1, 0))
    z2 = _mm(h1, bf16(w["W2"])) + w["b2"]
    h2 = bf16(np.maximum(z2, 0))
    y = _mm(h2, bf16(w["W3"])[:, None])[:, 0] + w["b3"][0]
    return y, dict(xn=xn, z1=z1, h1=h1, z2=z2, h2=h2)


def grad_bf16(p: np.ndarray, X: np.ndarray, Y: np.ndarray):
    """(gradient of sum (y - Y)^2 / rows over the trained parameters, sum of
    squared errors) as the training kernel computes them."""
    w = blocks(np.asarray(p, np.float32))
    y, a = forward_bf16(p, X)
    rows = len(Y)
    d = (y - np.asarray(Y, np.float32)).astype(np.float32)
    dy = (2.0 * d / rows).astype(np.float32)
    w3 = bf16(w["W3"])
    dh2 = np.where(a["z2"] > 0, dy[:, None] * w3[None, :], 0).astype(np.float32)
    dh1 = np.where(a["z1"] > 0, _mm(bf16(dh2), bf16(w["W2"]).T), 0).astype(np.float32)
    g = np.zeros(TRAINED, np.float64)
    gb = blocks(np.concatenate([g, np.zeros(TOTAL - TRAINED)]))
    gb["W1"][:] = a["xn"].T.astype(np.float64) @ dh1
    gb["b1"][:] = dh1.sum(axis=0, dtype=np.float64)
    gb["W2"][:] = a["h1"].T.astype(np.float64) @ dh2
    gb["b2"][:] = dh2.sum(axis=0, dtype=np.float64)
    gb["W3"][:] = a["h2"].T.astype(np.float64) @ dy
    gb["b3"][:] = dy.sum(dtype=np.float64)
    flat = np.concatenate([gb[k].reshape(-1) for k in ("W1", "b1", "W2", "b2", "W3", "b3")])
    return flat, float(np.sum(d.astype(np.float64) ** 2))


def forward_f64(p: np.ndarray, X: np.ndarray):
    w = {k: v.astype(np.float64) for k, v in blocks(np.asarray(p, np.float64)).items()}
    xn = (np.asarray(X, np.float64) - w["mean"]) * w["inv_std"]
    z1 = xn @ w["W1"] + w["b1"]
    h1 = np.maximum(z1, 0)
    z2 = h1 @ w["W2"] + w["b2"]
    h2 = np.maximum(z2, 0)
    return h2 @ w["W3"] + w["b3"][0], dict(xn=xn, z1=z1, h1=h1, z2=z2, h2=h2)


def loss_f64(p, X, Y) -> float:
    y, _ = forward_f64(p, X)
    return float(np.mean((y - Y) ** 2))


def grad_f64(p: np.ndarray, X: np.ndarray, Y: np.ndarray) -> np.ndarray:
    """Analytic gradient of the mean squared error of the FP64 network."""
    w = {k: v.astype(np.float64) for k, v in blocks(np.asarray(p, np.float64)).items()}
    y, a = forward_f64(p, X)
    dy = 2.0 * (y - Y) / len(Y)
    dh2 = np.where(a["z2"] > 0, dy[:, None] * w["W3"][None, :], 0)
    dh1 = np.where(a["z1"] > 0, dh2 @ w["W2"].T, 0)
    parts = [a["xn"].T @ dh1, dh1.sum(0), a["h1"].T @ dh2, dh2.sum(0), a["h2"].T @ dy, [dy.sum()]]
    return np.concatenate([np.asarray(q, np.float64).reshape(-1) for q in parts])


# ---------------------------------------------------------- features
def root_f64(pos) -> np.ndarray:
    """The system's centre of mass and total mass summed in FP64: (x, y, z, M)."""
    p = np.asarray(pos, np.float64)
    M = p[:, 3].sum()
    return np.array([*(p[:, :3] * p[:, 3:4]).sum(axis=0) / M, M], np.float64)


def group_features(sorted_pos, amag, sorted_keys, bits: int, extent: float, root_com, G: float):
    """The seven features of every 32-body group (engine order), FP32.
    root_com = the system's FP64 centre of mass and mass (root_f64): the
    distance of a group's centre from it is taken in FP64, then rounded."""
    f32 = np.float32
    n = sorted_pos.shape[0]
    groups = (n + 31) // 32
    out = np.zeros((groups, 7), f32)
    ext = max(f32(extent), f32(1e-30))
    root_com = np.asarray(root_com, np.float64)
    M = max(f32(root_com[3]), f32(1e-30))
    for g in range(groups):
        s, e = 32 * g, min(32 * g + 32, n)
        p = sorted_pos[s:e].astype(f32)
        a = amag[s:e].astype(f32)
        lo, hi = p[:, :3].min(axis=0), p[:, :3].max(axis=0)
        h = f32(0.5) * (hi - lo)
        R = np.sqrt(f32(h[0] * h[0] + h[1] * h[1] + h[2] * h[2]))
        c = ((f32(0.5) * (lo + hi)).astype(np.float64) - root_com[:3]).astype(f32)
        D = np.sqrt(f32(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]))
        cnt = e - s
        a_mean = f32(a.sum(dtype=np.float64)) / f32(cnt)
        a_scale = f32(G) * M / (ext * ext)
        x = int(sorted_keys[s]) ^ int(sorted_keys[e - 1])
        depth = bits if x == 0 else bits - 1 - (x.bit_length() - 1) // 3
        vol = max(f32(8) * h[0] * h[1] * h[2], f32(1e-30) * ext * ext * ext)
        m_sum = f32(p[:, 3].sum(dtype=np.float64))
        hmin, hmax = h.min(), h.max()
        out[g] = [np.log10(R / ext + f32(1e-7)), np.log10(a_mean / a_scale + f32(1e-12)),
                  np.log10((a.max() + f32(1e-30)) / (a.min() + f32(1e-30))), np.log10(D / ext + f32(1e-4)),
                  f32(depth) / f32(bits), np.log10(m_sum / M * ext * ext * ext / vol),
                  np.log10((hmin + f32(1e-7) * ext) / (hmax + f32(1e-7) * ext))]
    return out


def select(p: np.ndarray, feat: np.ndarray, ladder: np.ndarray, err_target: float, theta_cap: float):
    """(theta, alpha) per group and the predictions [groups, candidates].

    Restates k_mac_select (csrc/mlp.cu): c = the largest candidate whose
    prediction meets the target; alpha is interpolated in log alpha between
    candidates c and c+1 to where the prediction crosses the target."""
    groups, nc = feat.shape[0], len(ladder)
    X = np.zeros((groups * nc, 8), np.float32)
    X[:, 0] = np.tile(np.log10(ladder.astype(np.float32)), groups)
    X[:, 1:] = np.repeat(feat, nc, axis=0)
    y, _ = forward_bf16(p, X)
    y = y.reshape(groups, nc)
    lt = np.float32(np.log10(np.float32(err_target)))
    gp = np.zeros((groups, 2), np.float32)
    for g in range(groups):
        if not np.all(np.isfinite(y[g])):
            gp[g] = (0.5, 1e30)
            continue
        ok = np.nonzero(y[g] <= lt)[0]
        if not len(ok):
            gp[g] = (theta_cap, ladder[0])
            continue
        c = ok.max()
        alpha = np.float32(ladder[c])
        # interpolate in log alpha up to where the predicted curve meets the target
        if c + 1 < nc and y[g, c + 1] > lt and y[g, c + 1] > y[g, c]:
            frac = np.float32(np.float32(lt - y[g, c]) / np.float32(y[g, c + 1] - y[g, c]))
            alpha = np.float32(alpha * np.exp2(frac, dtype=np.float32))
        gp[g] = (theta_cap, alpha)
    return gp, y
