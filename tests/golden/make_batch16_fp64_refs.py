"""Generates tests/golden/batch16_fp64_refs.npz: FP64 oracle renders of 1/8-scale copies of the 16
scenes of the uneven batch (phosphor_b200.rmse.uneven_batch_specs), the calibration of the time-to-RMSE
study's references.

At full size (256^2..1024^2 pixels, up to 2^21 photons per round) a converged CPU FP64 render of
the 16 scenes is out of reach, so the study's references are long fp32 renders on the GPU with an
independent seed.  To bound their error, each scene is also rendered here at 1/8 scale
(phosphor_b200.rmse.scaled: resolution / 8 per side, photons / 64, the same grid, alpha and
generator seed) by the CPU oracle in double precision (oracle/phx_oracle.hpp with R = double,
RGBE/octahedral quantisation kept) for RMSE_REF_ROUNDS rounds with the seed scene seed +
RMSE_REF_SEED_OFFSET, through the reference display transform (output.cpp:40-83, exposure 0.66,
no ACES).  The bench renders the same 1/8-scale copies with its reference procedure (fp32, GPU,
another seed) and reports their RMSE to these images.  Images are uint16 fixed point.

    python tests/golden/make_batch16_fp64_refs.py [--threads N]
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
    ap.add_argument("--rounds", type=int, default=R.RMSE_REF_ROUNDS)
    a = ap.parse_args()
    imgs = {}
    t_all = time.time()
    for i, full in enumerate(R.uneven_batch_specs()):
        s = R.scaled(full, R.BATCH_CAL_SCALE)
        t = time.time()
        scene = O.GeneratedScene(s.kind, seed=s.seed, width=s.width, height=s.height, detail=s.detail)
        orc = O.Oracle(scene)
        args = s.args(seed=s.seed + R.RMSE_REF_SEED_OFFSET)
        st = orc.render(args.params(), a.rounds, prec=1, threads=a.threads or None)
        img = O.image(st["flux"], st["radiance"], 1, 0.66, False, st["total"], a.rounds)
        imgs[f"scene{i}"] = np.round(np.clip(img, 0, 1) * 65535).astype(np.uint16).reshape(s.height, s.width, 3)
        print(f"scene {i}: {s.width}x{s.height} kind {s.kind} {s.photons} photons -> {time.time() - t:.1f}s",
              flush=True)
    out = Path(__file__).with_name("batch16_fp64_refs.npz")
    np.savez_compressed(out, rounds=a.rounds, scale=R.BATCH_CAL_SCALE, **imgs)
    print(f"wrote {out} in {time.time() - t_all:.0f}s")


if __name__ == "__main__":
    main()
