"""Generate the golden fixtures under tests/golden/ from the reference itself.

Runs the reference's own buildTree / calculateAcceleration / positionUpdater
(compiled from its sources into oracle/_ref/libref.so by oracle/build.py) on a
CUDA GPU, one step per case, and stores inputs and outputs:

    python tests/golden/make_golden.py [outdir]

Each case file ref_<name>.npz holds: pos, vel (inputs), eps, G, theta, dt,
keys (Morton keys of the inputs), skeys, perm (sorted keys, permutation),
nodes (the tree, reference layout, as raw bytes), level_offsets,
level_count, deepest, acc (sorted order), pos_out, vel_out (after the step).
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import cudagravitydemo_b200 as bh  # noqa: E402  (initial conditions only)
from oracle import cpu  # noqa: E402


def cases():
    p, v = bh.plummer(2048, seed=0)
    yield "plummer2048", p, v, dict(eps=0.01, G=1.0, theta=0.5, dt=1e-3)
    p, v = bh.disk_galaxy(3000, seed=1)
    yield "disk3000", p, v, dict(eps=0.005, G=1.0, theta=0.5, dt=5e-4)
    p, v = bh.plummer(1024, seed=7)
    p[1::16, :3] = p[0::16, :3]  # coincident pairs -> multi-body leaves at level 21
    p[200:203, :3] = p[200, :3]  # and a triple
    yield "coincident1024", p, v, dict(eps=0.02, G=1.0, theta=0.7, dt=1e-3)
    p = np.array([[0, 0, 0, 1], [1, 0.5, 0.25, 2], [-0.5, 0.125, 2, 0.5]], np.float32)
    v = np.zeros((3, 3), np.float32)
    yield "three_bodies", p, v, dict(eps=0.01, G=1.0, theta=0.5, dt=1e-3)


def main(outdir: Path) -> None:
    outdir.mkdir(parents=True, exist_ok=True)
    for name, p, v, prm in cases():
        r = cpu.ref_run(p, v, prm["eps"], prm["G"], prm["theta"], prm["dt"], steps=1)
        np.savez_compressed(outdir / f"ref_{name}.npz", pos=p, vel=v, **{k: np.float32(x) for k, x in prm.items()},
                            keys=r["keys"], skeys=r["skeys"], perm=r["perm"], nodes=r["nodes"].view(np.uint8),
                            level_offsets=r["level_offsets"], level_count=r["level_count"],
                            deepest=np.int32(r["deepest"]), acc=r["acc"], pos_out=r["pos"], vel_out=r["vel"])
        print(name, p.shape[0], "nodes", r["count"], "deepest", r["deepest"])


if __name__ == "__main__":
    main(Path(sys.argv[1]) if len(sys.argv) > 1 else Path(__file__).resolve().parent)
