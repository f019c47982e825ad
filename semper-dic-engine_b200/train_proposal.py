#!/usr/bin/env python
"""Train the learned seed proposal network on the GPU and write its weights.

    python semper-dic-engine_b200/train_proposal.py --out weights.npy [--minutes M]

The shipped weights (weights/proposal.npy) come from this script with its
defaults (10 minutes on one B200, about 170,000 Adam steps).

Training pairs are made on the device from a seeded 4096x4096 speckle image
(the same Gaussian-blob recipe as the benchmark workloads, another seed):
each pair is two 64x64 patches box-averaged by a factor f, the second under a
random rotation, stretch and shear up to 3 % and 2 %, a translation and noise
of 2 gray levels. One network serves the three stages of learned seeding, so
the batches cycle, 100 steps each, through
- f = 4, rotation in [0, R) with R growing from 30 to 360 deg over the first
  40 % of the time, translation up to 64 px (the coarse stage);
- f = 2, rotation up to 15 deg, translation up to 24 px;
- f = 1, rotation up to 8 deg, translation up to 10 px (the refinements).
Adam, batch 256, learning rate 1e-3, then 3e-4 from 70 % and 1e-4 from 90 % of
the time. The weights are written as one float32 vector in the library's
parameter layout (semper_b200_proposal_set_params). A held-out set reports the
rotation and translation errors per stage.
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

STAGES = {"f4": [2 * np.pi, 0.03, 0.02, 64.0, 2.0, 4], "f2": [np.radians(15.0), 0.03, 0.02, 24.0, 2.0, 2],
          "f1": [np.radians(8.0), 0.03, 0.02, 10.0, 2.0, 1]}


def stage_cfgs(frac: float):
    """The three stages' synthetic-pair settings at a fraction of the time."""
    rot = np.radians(30.0 + 330.0 * min(1.0, frac / 0.4))
    return [[rot] + STAGES["f4"][1:], STAGES["f2"], STAGES["f1"]]


def affine_errors(out, target, f):
    """Rotation error (deg) and translation error (full-resolution px) of
    predicted affine maps against their targets at box factor f."""
    def rot(o):
        a00, a01, a10, a11 = 1 + o[:, 0], o[:, 1], o[:, 2], 1 + o[:, 3]
        return np.degrees(np.arctan2(a10 - a01, a00 + a11))

    dr = np.abs((rot(out) - rot(target) + 180.0) % 360.0 - 180.0)
    dt = f * 16.0 * np.hypot(out[:, 4] - target[:, 4], out[:, 5] - target[:, 5])
    return dr, dt


def evaluate(net, speckle, n=1024, seed=999):
    rep = {}
    for name, cfg in STAGES.items():
        outs, tgts = [], []
        for k in range(0, n, 256):
            x, t = net.synth(speckle, cfg, seed=seed + k, batch=256)
            outs.append(net.forward(x))
            tgts.append(t)
        dr, dt = affine_errors(np.concatenate(outs), np.concatenate(tgts), cfg[5])
        rep[name] = {"rot_deg_median": float(np.median(dr)), "rot_deg_p90": float(np.percentile(dr, 90)),
                     "shift_px_median": float(np.median(dt)), "shift_px_p90": float(np.percentile(dt, 90))}
    return rep


def train(minutes: float, seed: int = 1000, log=print):
    speckle = sb.speckle(4096, 4096, 4321)
    net = sb.Proposal(256)
    total = 60.0 * minutes
    done, k, t0, curve = 0, 0, time.time(), []
    while time.time() - t0 < total:
        frac = (time.time() - t0) / total
        lr = 1e-3 if frac < 0.7 else (3e-4 if frac < 0.9 else 1e-4)
        cfg = stage_cfgs(frac)[k % 3]
        losses = net.train(speckle, cfg, steps=100, batch=256, lr=lr, seed=seed + done)
        done += len(losses)
        k += 1
        curve.append(float(losses.mean()))
        if k % 60 == 1:
            log(f"step {done}: f={cfg[5]} loss {curve[-1]:.2f} (lr {lr:g}, {time.time() - t0:.0f} s)")
    return net, speckle, done, curve, time.time() - t0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    ap.add_argument("--minutes", type=float, default=10.0)
    ap.add_argument("--report", default=None, help="write a JSON summary here")
    args = ap.parse_args()
    net, speckle, done, curve, secs = train(args.minutes)
    np.save(args.out, net.get_params())
    ev = evaluate(net, speckle)
    rep = {"steps": done, "seconds": round(secs, 1), "pairs_seen": done * 256, "heldout": ev}
    print(json.dumps(rep))
    if args.report:
        with open(args.report, "w") as f:
            json.dump(rep, f, indent=1)


if __name__ == "__main__":
    main()
