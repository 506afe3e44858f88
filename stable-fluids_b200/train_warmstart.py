"""Trains the learned pressure warm start with the config-2 protocol and
saves its weights.

Protocol (the pressure warm start's training set):
  - pairs generated by the solver itself at 128^3: seeded plume scenes with
    1-4 Gaussian sources of radius U[4, 12] cells and upward forces U[1, 10]
    (scenes.training_scene), config-0 coefficients;
  - each pair: the pressure right-hand side (pre-projection divergence) and
    the previous step's pressure as inputs, the pressure after 1000 Jacobi
    sweeps from the previous pressure as the target; the target's own FP64
    relative residual is recorded for every pair;
  - 2000 pairs by default (scenes x steps per scene), a held-out tail for
    validation, Adam on the rest; the weights of the epoch with the best
    held-out error are kept.
Everything runs in the library's own kernels (stencils for the pairs, the
network's forward / backward / Adam on the tensor cores); torch only holds
device buffers.

Usage: python stable-fluids_b200/train_warmstart.py [--pairs 2000] [--out PATH]
Writes PATH (FP32 parameters, .npy) and PATH with suffix .json (protocol,
target residuals, losses, SHA-256 of the parameters).
"""

from __future__ import annotations

import argparse
import hashlib
import importlib
import json
import pathlib
import sys
import time

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
DEFAULT_WEIGHTS = HERE / "weights" / "warmstart_128.npy"


def parse(argv=None):
    p = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    p.add_argument("--pairs", type=int, default=2000)
    p.add_argument("--size", type=int, default=128)
    p.add_argument("--steps-per-scene", type=int, default=50)
    p.add_argument("--skip", type=int, default=2, help="plain steps before a scene's first pair")
    p.add_argument("--sweeps", type=int, default=1000, help="Jacobi sweeps of each target solve")
    p.add_argument("--holdout", type=int, default=100, help="pairs kept out of training for validation")
    p.add_argument("--epochs", type=int, default=4)
    p.add_argument("--learning-rate", type=float, default=3e-4)
    p.add_argument("--seconds", type=float, default=1800.0, help="training time budget")
    p.add_argument("--seed", type=int, default=0)
    p.add_argument("--out", type=pathlib.Path, default=DEFAULT_WEIGHTS)
    return p.parse_args(argv)


def sha256_of(params: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(params, np.float32).tobytes()).hexdigest()


def generate(sf, args):
    """The pairs on the device, with each target's relative residual."""
    pairs, target_res = [], []
    scenes = (args.pairs + args.steps_per_scene - 1) // args.steps_per_scene
    for k in range(scenes):
        scene = sf.scenes.training_scene(k, n=args.size, pressure_iterations=args.sweeps)
        o = sf.default_options()
        o.scheme = sf.SCHEME_JACOBI
        o.warm_start = sf.WARM_START_PREVIOUS
        o.compute_residual = 1
        sim = sf.Simulation(scene.config, scene.scalars, scene.vectors, options=o)
        sf.scenes.apply_inputs(sim, scene, 0)
        sim.step(args.skip)
        for _ in range(min(args.steps_per_scene, args.pairs - len(pairs))):
            pairs.append(sf.warmstart.step_with_snapshot(sim))
            target_res.append(sim.stats().rel_residual)  # measured by the projection stage
        sim.close()
    return pairs, np.asarray(target_res)


def held_out_error(net, pairs, h):
    """Mean over the pairs of ||pred - target|| / ||p_prev - target||: the
    fraction of the previous pressure's error the prediction leaves."""
    import torch

    errs = []
    for b, p, t in pairs:
        pred = net.predict(b, p, h)
        errs.append(float(torch.linalg.vector_norm(pred - t) / torch.clamp(torch.linalg.vector_norm(p - t), min=1e-30)))
    return float(np.mean(errs))


def main(argv=None):
    args = parse(argv)
    sys.path.insert(0, str(HERE.parent))
    sf = importlib.import_module("stable-fluids_b200")
    t0 = time.perf_counter()
    pairs, target_res = generate(sf, args)
    t_pairs = time.perf_counter() - t0
    print(json.dumps({"pairs": len(pairs), "pair_generation_s": t_pairs, "target_rel_residual_median": float(np.median(target_res))}), flush=True)
    h = float(sf.scenes.training_scene(0, n=args.size).config.cell_size)
    train = pairs[:-args.holdout] if args.holdout else pairs
    valid = pairs[-args.holdout:] if args.holdout else []
    net = sf.WarmStartNetwork(seed=args.seed)
    best = (held_out_error(net, valid, h) if valid else float("inf"), net.parameters())
    history, deadline = [], time.perf_counter() + args.seconds
    rng = np.random.default_rng(args.seed)
    for epoch in range(args.epochs):
        losses = []
        for k in rng.permutation(len(train)):
            b, p, t = train[k]
            losses.append(net.train_step(b, p, t, h, args.learning_rate))
            if time.perf_counter() > deadline:
                break
        err = held_out_error(net, valid, h) if valid else float("nan")
        history.append({"epoch": epoch + 1, "train_loss": float(np.mean(losses)), "held_out_error": err, "steps": len(losses), "elapsed_s": time.perf_counter() - t0})
        print(json.dumps(history[-1]), flush=True)
        if valid and err < best[0]:
            best = (err, net.parameters())
        if time.perf_counter() > deadline:
            break
    params = best[1] if valid else net.parameters()
    args.out.parent.mkdir(parents=True, exist_ok=True)
    np.save(args.out, params)
    info = {
        "protocol": {"pairs": len(pairs), "grid": [args.size] * 3, "scenes": (args.pairs + args.steps_per_scene - 1) // args.steps_per_scene, "steps_per_scene": args.steps_per_scene,
                     "skip": args.skip, "target": f"{args.sweeps} Jacobi sweeps from the previous pressure", "held_out": len(valid), "epochs": args.epochs, "learning_rate": args.learning_rate, "seed": args.seed},
        "target_rel_residual": {"mean": float(target_res.mean()), "median": float(np.median(target_res)), "min": float(target_res.min()), "max": float(target_res.max())},
        "history": history, "best_held_out_error": best[0] if valid else None,
        "pair_generation_s": t_pairs, "training_s": time.perf_counter() - t0 - t_pairs, "sha256": sha256_of(params),
    }
    args.out.with_suffix(".json").write_text(json.dumps(info, indent=1) + "\n")
    print(json.dumps({k: info[k] for k in ("target_rel_residual", "best_held_out_error", "pair_generation_s", "training_s", "sha256")}))
    net.close()


if __name__ == "__main__":
    main()
