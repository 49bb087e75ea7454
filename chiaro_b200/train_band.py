"""Train and evaluate the band proposal network (no counterpart in the reference).

    python -m chiaro_b200.train_band --out chiaro_b200/weights/bandnet.bin \\
        [--train 2000] [--eval 200] [--steps 3000] [--batch 64] [--resume PATH]

Training scenes are seeded 1040x780 renderings of the five-view structure (a reference
and 4 sources at 2-6 cm, 12 slanted planes and 3 spheres, 192 planes over 0.4-50 m),
ray cast on the GPU. For each, the network's inputs are the coarse search's pre-pass
(16 sampled labels, ``coarse.band_prepass``) and its targets the tile medians of the
exact plain search's winners over the tested nodes. Training runs Adam over minibatches
of images, on the GPU through the library's kernels. The held-out evaluation renders
full-resolution five-view scenes (4160x3120, 4 sources, 192 planes) and scores the
learned-band search against the plain search (within one plane over tested nodes,
fallback rate, time) beside the naive band. The checkpoint (``BandNet.save``: a
versioned binary of the parameters and optimiser state, with a JSON of the training
set-up and results) can be resumed with ``--resume``.
"""
from __future__ import annotations

import argparse
import json
import time
from pathlib import Path

import numpy as np

from . import bandnet
from .depth import DeviceStage


def render(name: str, seeds, device, **overrides):
    from . import scenes
    for seed in seeds:
        yield scenes.workload(name, seed=seed, cache=False, render_device=device, **overrides)


def prepare(ctx, seeds, device, tile: int, options=dict(planes=192)):
    """Training samples of the seeded 1040x780 scenes: device tensors of the pre-pass rows
    and guidance, host tile-median targets and masks."""
    import torch
    from .coarse import PREPASS_SLOTS, band_prepass, coarse_depth
    out = []
    for sc in render("band", seeds, device, options=options):
        stage = DeviceStage(sc.inputs(), 0, sc.alignments(), sc.options, context=ctx)
        costs, guidance, _ = band_prepass(stage)
        plain = coarse_depth(stage)
        sample = bandnet.Sample(costs.reshape(-1).clone(), guidance.clone(), plain.winner.cpu().numpy(),
                                plain.tested.cpu().numpy(), plain.columns, plain.rows, plain.labels, PREPASS_SLOTS)
        target = bandnet.tile_targets(sample, tile, "median")
        target.winners = torch.from_numpy(target.winners).to(device)
        target.mask = torch.from_numpy(target.mask).to(device)
        out.append(target)
        del stage
    return out


def train(net, samples, steps: int, batch: int, lr: float, seed: int = 0):
    """Minibatch Adam: each step draws `batch` images; the learning rate drops 4x for the last third."""
    rng = np.random.default_rng(seed)
    losses = []
    for k in range(steps):
        pick = rng.choice(len(samples), size=min(batch, len(samples)), replace=False)
        rate = lr if k < 2 * steps // 3 else lr / 4
        losses.append(float(net.train([samples[i] for i in pick], 1, rate)[0]))
    return losses


def evaluate(ctx, net, seeds, device, tile: int, band: int, margin: int, fraction: float):
    """The learned-band and naive searches against the plain search on held-out
    full-resolution scenes, rendered one at a time (one scene's planes resident)."""
    stages = (DeviceStage(sc.inputs(), 0, sc.alignments(), sc.options, context=ctx)
              for sc in render("five_view", seeds, device, options=dict(planes=192)))
    return bandnet.evaluate_search(stages, {"learned": net}, tile, band, margin, fraction)


def main(argv=None):
    import torch
    from .runtime import DepthContext
    p = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    p.add_argument("--out", required=True)
    p.add_argument("--train", type=int, default=2000)
    p.add_argument("--eval", type=int, default=200)
    p.add_argument("--steps", type=int, default=3000)
    p.add_argument("--batch", type=int, default=64)
    p.add_argument("--lr", type=float, default=2e-3)
    p.add_argument("--tile", type=int, default=4)
    p.add_argument("--band", type=int, default=24)
    p.add_argument("--margin", type=int, default=8)
    p.add_argument("--fraction", type=float, default=0.5)
    p.add_argument("--resume", default=None)
    p.add_argument("--seed", type=int, default=0)
    args = p.parse_args(argv)
    device = torch.device("cuda", 0)
    ctx = DepthContext(0)
    net = bandnet.BandNet(ctx, seed=args.seed)
    if args.resume:
        net.load(args.resume)
    t0 = time.perf_counter()
    samples = prepare(ctx, range(10000, 10000 + args.train), device, args.tile)
    prepare_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    losses = train(net, samples, args.steps, args.batch, args.lr, args.seed)
    torch.cuda.synchronize()
    train_s = time.perf_counter() - t0
    del samples
    torch.cuda.empty_cache()
    t0 = time.perf_counter()
    scores = evaluate(ctx, net, range(20000, 20000 + args.eval), device, args.tile, args.band, args.margin,
                      args.fraction) if args.eval else None
    eval_s = time.perf_counter() - t0
    meta = {"training": {"scenes": args.train, "workload": "band: 1040x780, reference + 4 sources, 192 planes",
                         "scene_seeds": [10000, 10000 + args.train], "steps": args.steps, "batch": args.batch,
                         "learning_rate": args.lr, "targets": "tile medians (4x4 nodes) of the plain search's "
                         "winners over tested nodes", "inputs": "pre-pass: guidance and 16 sampled labels",
                         "loss_first": losses[0] if losses else None, "loss_last": losses[-1] if losses else None,
                         "prepare_s": round(prepare_s, 1), "train_s": round(train_s, 1)},
            "evaluation": {"scenes": args.eval, "workload": "five_view at 4160x3120, 192 planes",
                           "scene_seeds": [20000, 20000 + args.eval], "tile": args.tile, "band": args.band,
                           "margin": args.margin, "contradicted_fraction": args.fraction,
                           "eval_s": round(eval_s, 1), "scores": scores}}
    Path(args.out).parent.mkdir(parents=True, exist_ok=True)
    net.save(args.out, meta)
    print(json.dumps(meta, indent=1))
    ctx.close()


if __name__ == "__main__":
    main()
