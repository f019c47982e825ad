#!/usr/bin/env python
"""Train the learned seed proposal network on the GPU and write its weights.

    python semper-dic-engine_b200/train_proposal.py --out weights.npy [--steps N] [--seconds S]

Training pairs are made on the device from a seeded 4096x4096 speckle image
(the same Gaussian-blob recipe as the benchmark workloads, another seed):
each pair is two 64x64 patches, box-averaged by 4 (a 256-pixel square), the
second under a random rotation in [0, 360) deg, stretch and shear up to 3 % and
2 %, a translation up to 64 px and noise of 2 gray levels. Adam, batch 256,
learning rate 1e-3 then 3e-4 and 1e-4 over the last 40 % and 15 % of the
steps. The weights are written as one float32 vector in the library's
parameter layout (semper_b200_proposal_set_params). A held-out set reports the
rotation and translation errors of the trained network.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
import semper_b200 as sb  # noqa: E402

CFG = [2 * np.pi, 0.03, 0.02, 64.0, 2.0, 4]
BOX = 4


def affine_errors(out, target):
    """Rotation error (deg) and translation error (full-resolution px) of
    predicted affine maps against their targets."""
    def rot(o):
        a00, a01, a10, a11 = 1 + o[:, 0], o[:, 1], o[:, 2], 1 + o[:, 3]
        return np.degrees(np.arctan2(a10 - a01, a00 + a11))

    dr = np.abs((rot(out) - rot(target) + 180.0) % 360.0 - 180.0)
    dt = BOX * 16.0 * np.hypot(out[:, 4] - target[:, 4], out[:, 5] - target[:, 5])
    return dr, dt


def evaluate(net, speckle, n=1024, seed=999):
    outs, tgts = [], []
    for k in range(0, n, 256):
        x, t = net.synth(speckle, CFG, seed=seed + k, batch=256)
        outs.append(net.forward(x))
        tgts.append(t)
    dr, dt = affine_errors(np.concatenate(outs), np.concatenate(tgts))
    return {"rot_deg_median": float(np.median(dr)), "rot_deg_p90": float(np.percentile(dr, 90)),
            "shift_px_median": float(np.median(dt)), "shift_px_p90": float(np.percentile(dt, 90))}


def train(steps: int, seconds: float, seed: int = 1, log=print):
    speckle = sb.speckle(4096, 4096, 4321)
    net = sb.Proposal(256)
    chunk = 100
    done, t0, curve = 0, time.time(), []
    while done < steps and time.time() - t0 < seconds:
        frac = done / max(steps, 1)
        lr = 1e-3 if frac < 0.6 else (3e-4 if frac < 0.85 else 1e-4)
        losses = net.train(speckle, CFG, steps=min(chunk, steps - done), batch=256, lr=lr, seed=seed * 100003 + done)
        done += len(losses)
        curve.append(float(losses.mean()))
        if len(curve) % 10 == 1:
            log(f"step {done}: loss {curve[-1]:.2f} (lr {lr:g}, {time.time() - t0:.0f} s)")
    return net, speckle, done, curve, time.time() - t0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    ap.add_argument("--steps", type=int, default=6000)
    ap.add_argument("--seconds", type=float, default=600.0)
    ap.add_argument("--report", default=None, help="write a JSON summary here")
    args = ap.parse_args()
    net, speckle, done, curve, secs = train(args.steps, args.seconds)
    np.save(args.out, net.get_params())
    ev = evaluate(net, speckle)
    rep = {"steps": done, "seconds": round(secs, 1), "pairs_seen": done * 256, "loss_first": curve[0],
           "loss_last": curve[-1], "heldout": ev, "cfg": CFG}
    print(json.dumps(rep))
    if args.report:
        with open(args.report, "w") as f:
            json.dump(rep, f, indent=1)


if __name__ == "__main__":
    main()
