"""Generates tests/golden/rmse_refs.npz: converged FP64 oracle renders of the time-to-RMSE batch.

Each of the 16 scenes of phosphor_b200.rmse.rmse_batch() is rendered by the CPU oracle in double
precision (oracle/phx_oracle.hpp instantiated with R = double, RGBE/octahedral quantisation kept)
for RMSE_REF_ROUNDS rounds with an independent seed (scene seed + RMSE_REF_SEED_OFFSET), then
passed through the reference display transform (output.cpp:40-83, exposure 0.66, no ACES).
Images are stored as uint16 fixed point (value * 65535, max error 7.6e-6).

    python tests/golden/make_rmse_refs.py [--threads N]
"""
import argparse
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import oracle as O  # noqa: E402
from phosphor_b200 import rmse as R  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--threads", type=int, default=0)
    a = ap.parse_args()
    specs = R.rmse_batch()
    imgs = {}
    meta = []
    t_all = time.time()
    for i, s in enumerate(specs):
        t = time.time()
        scene = s.scene()
        orc = O.Oracle(scene)
        args = s.args(seed=s.seed + R.RMSE_REF_SEED_OFFSET)
        st = orc.render(args.params(), R.RMSE_REF_ROUNDS, prec=1, threads=a.threads or None)
        img = O.image(st["flux"], st["radiance"], 1, 0.66, False, st["total"], R.RMSE_REF_ROUNDS)
        imgs[f"scene{i}"] = np.round(np.clip(img, 0, 1) * 65535).astype(np.uint16).reshape(s.height, s.width, 3)
        meta.append(vars(s))
        print(f"scene {i}: {s.width}x{s.height} kind {s.kind} {s.photons} photons -> {time.time() - t:.1f}s",
              flush=True)
    out = Path(__file__).with_name("rmse_refs.npz")
    np.savez_compressed(out, rounds=R.RMSE_REF_ROUNDS, **imgs)
    print(f"wrote {out} in {time.time() - t_all:.0f}s")


if __name__ == "__main__":
    main()
