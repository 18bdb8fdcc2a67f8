"""Force accuracy against an FP64 direct sum, computed on the GPU.

Every Barnes-Hut result of the engine can be stated against the exact
softened sum a_t = sum_j G m_j (x_j - x_t) / (|x_j - x_t|^2 + eps^2)^{3/2},
evaluated in double precision by bh_direct_sum_f64 for a sample of target
bodies.  The relative error of a body is |a - a_exact| / |a_exact|; a run is
summarised by the RMS of that over the sample (and its percentiles).
"""
from __future__ import annotations

import numpy as np

from . import _check, _ptr, lib


def direct_sum(pos, targets, eps: float, G: float = 1.0, stream=None):
    """FP64 accelerations (torch float64 [nt,3], device) of bodies `targets`
    (torch int32, device) of the device positions `pos` (torch float32 [n,4])."""
    import torch
    nt = int(targets.shape[0])
    out = torch.empty((nt, 3), dtype=torch.float64, device=pos.device)
    _check(lib().bh_direct_sum_f64(_ptr(pos), int(pos.shape[0]), _ptr(targets), nt, float(eps), float(G), _ptr(out),
                                   stream), "bh_direct_sum_f64")
    return out


def sample_targets(n: int, nsample: int, seed: int = 0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    if nsample >= n:
        return np.arange(n, dtype=np.int32)
    return np.sort(rng.choice(n, size=nsample, replace=False)).astype(np.int32)


def force_error(sim, nsample: int = 65536, seed: int = 0) -> dict:
    """Relative force error of sim's current accelerations on a body sample."""
    import torch
    pos, _ = sim.store()
    acc = sim.accelerations()
    tgt = sample_targets(pos.shape[0], nsample, seed)
    exact = direct_sum(torch.from_numpy(pos).cuda(), torch.from_numpy(tgt).cuda(), sim.params.eps,
                       sim.params.G).cpu().numpy()
    got = acc[tgt].astype(np.float64)
    rel = np.linalg.norm(got - exact, axis=1) / np.maximum(np.linalg.norm(exact, axis=1), 1e-300)
    return {"rms": float(np.sqrt(np.mean(rel ** 2))), "median": float(np.median(rel)),
            "p99": float(np.percentile(rel, 99)), "max": float(rel.max()), "nsample": int(len(tgt)),
            "targets": tgt, "rel": rel}
