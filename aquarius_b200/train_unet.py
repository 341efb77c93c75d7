"""Trains the learned pressure warm start and writes its weights file.

    python -m aquarius_b200.train_unet --size 64 --scenes 500 --train-steps 12000 --calibrate-scale \
        --out aquarius_b200/weights/unet_64.bin
    python -m aquarius_b200.train_unet --size 128 --scenes 500 --init aquarius_b200/weights/unet_64.bin \
        --train-steps 6000 --lr 2e-4 --residual-weight 1.0 --select-every 500 --calibrate-scale \
        --out aquarius_b200/weights/unet_128.bin
    python -m aquarius_b200.train_unet --size 256 --scenes 25 --init aquarius_b200/weights/unet_128.bin \
        --train-steps 1500 --lr 1e-4 --residual-weight 1.0 --select-every 250 --calibrate-scale \
        --out aquarius_b200/weights/unet_256.bin
    python -m aquarius_b200.train_unet --size 128 --scenes 250 --every 5 --init aquarius_b200/weights/unet_128.bin \
        --train-steps 4000 --lr 1e-4 --residual-weight 1.0 --select-every 500 --calibrate-scale \
        --out aquarius_b200/weights/unet_128.bin

Training pairs: seeded ball-drop scenes (a pool of random depth 0.1-0.4 under
1-3 spheres of radius 0.08-0.2 at random positions, 8 particles per cell),
simulated by this library with a plain zero-init Jacobi solve; every
`--every` steps over `--steps-per-scene` steps the pressure system of the
next step (rhs = -divergence x density, fluid mark) is labelled by the FP64
PCG to relative residual 1e-10 and stored on the device.  The network is then
trained by the library's own kernels (Adam, cosine learning rate) on 90% of
the pairs and evaluated on the rest (mean relative L2 pressure error over
fluid cells).  `--adopt` skips training and takes a trained network as it is
(the fully convolutional network applies to any grid size divisible by 4).
`--init` starts from a trained network (fine-tuning); `--select-every` then
trains in chunks and keeps the chunk's weights, the starting ones included,
whose held-out 20-sweep residual ratio (the fallback rule's quantity) is
lowest.
`--calibrate-scale` then picks the network's output scale, among multiples
of its current one, that minimises the mean ratio of the residuals after 20
Jacobi sweeps from the prediction and from zero on the held-out pairs (all
pairs with --adopt): the quantity the warm start's fallback rule compares.
Everything runs on one GPU; a JSON summary goes to stdout.
"""
from __future__ import annotations

import argparse
import json
import math
import pathlib
import tempfile
import time

import numpy as np

from . import Dataset, Fluid, UNet, _abi

WEIGHTS_DIR = pathlib.Path(__file__).resolve().parent / "weights"


def scene_config(size: int, rng: np.random.RandomState, seed: int, sweeps: int) -> _abi.Config:
    depth = float(rng.uniform(0.1, 0.4))
    vols = [dict(shape="box", min=(0.0, 0.0, 0.0), max=(1.0, depth, 1.0), phase=0)]
    for _ in range(int(rng.randint(1, 4))):
        r = float(rng.uniform(0.08, 0.2))
        c = (float(rng.uniform(0.15, 0.85)), float(rng.uniform(min(depth + r, 0.9), 0.9)), float(rng.uniform(0.15, 0.85)))
        vols.append(dict(shape="sphere", center=c, radius=r, phase=0))
    return _abi.make_config((size, size, size), vols, timestep=0.64 / size, flip_coeff=0.95,
                            particle_jitter=0.05, seed=seed, pressure_init=_abi.PRESSURE_ZERO,
                            solve_mode=_abi.SOLVE_FIXED, pressure_iterations=sweeps)


def generate(size: int, scenes: int, steps_per_scene: int, every: int, seed: int, sweeps: int,
             device: int = 0) -> tuple[Dataset, dict]:
    per_scene = len(range(every, steps_per_scene + 1, every))
    ds = Dataset((size, size, size), capacity=scenes * per_scene, device=device)
    rng = np.random.RandomState(seed)
    t0 = time.perf_counter()
    pcg_its = []
    for k in range(scenes):
        cfg = scene_config(size, rng, seed * 100003 + k, sweeps)
        cfg.device = device
        with Fluid(cfg) as f:
            done = 0
            for s in range(every, steps_per_scene + 1, every):
                f.step(s - done)
                for stage in range(1, 5):  # the next step's pressure system
                    f.run_stage(stage)
                pcg_its.append(ds.add_fluid(f, 1e-10))
                for stage in range(5, 9):
                    f.run_stage(stage)
                done = s + 1
    info = {"pairs": len(ds), "scenes": scenes, "generate_s": time.perf_counter() - t0,
            "pcg_iterations_mean": float(np.mean(pcg_its)) if pcg_its else 0.0}
    return ds, info


def check_warm(net: UNet, size: int, device: int, steps: int = 4) -> list:
    """Residuals after 20 sweeps from the prediction and from zero on the
    ball-drop scene (pool y < 0.3, sphere r 0.12 at (0.5, 0.7, 0.5))."""
    vols = [dict(shape="box", min=(0, 0, 0), max=(1, 0.3, 1), phase=0),
            dict(shape="sphere", center=(0.5, 0.7, 0.5), radius=0.12, phase=0)]
    cfg = _abi.make_config((size, size, size), vols, timestep=0.64 / size, pressure_init=_abi.PRESSURE_LEARNED,
                           solve_mode=_abi.SOLVE_FIXED, pressure_iterations=200, device=device)
    out = []
    with Fluid(cfg) as f:
        f.set_warm_start(net)
        for _ in range(steps):
            f.step(1)
            s = f.solve_stats()
            out.append([s["warm_rel_residual"], s["zero_rel_residual"]])
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--size", type=int, default=64)
    ap.add_argument("--scenes", type=int, default=500)
    ap.add_argument("--steps-per-scene", type=int, default=80)
    ap.add_argument("--every", type=int, default=10)
    ap.add_argument("--sim-sweeps", type=int, default=200, help="Jacobi sweeps of the data-generating simulation")
    ap.add_argument("--train-steps", type=int, default=6000)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--residual-weight", type=float, default=0.3,
                    help="weight of (residual after --residual-sweeps sweeps from the prediction / from zero)^2 "
                         "in the loss")
    ap.add_argument("--residual-sweeps", type=int, default=20)
    ap.add_argument("--check-warm", action="store_true",
                    help="after training, step a 128^3-style test scene with the warm start and report "
                         "the residuals after 20 sweeps from the prediction and from zero")
    ap.add_argument("--seed", type=int, default=7)
    ap.add_argument("--init", type=str, default=None, help="weights file to start from (fine-tuning)")
    ap.add_argument("--adopt", type=str, default=None, help="weights file to use as it is (no training)")
    ap.add_argument("--calibrate-scale", action="store_true",
                    help="choose the output scale by the 20-sweep residual ratio on held-out pairs")
    ap.add_argument("--select-every", type=int, default=0,
                    help="train in chunks of this many steps (learning rate on one cosine over all steps) and "
                         "keep the weights, the starting ones included, with the lowest held-out 20-sweep "
                         "residual ratio")
    ap.add_argument("--out", type=str, default=None)
    ap.add_argument("--device", type=int, default=0)
    args = ap.parse_args()

    ds, info = generate(args.size, args.scenes, args.steps_per_scene, args.every, args.seed, args.sim_sweeps,
                        args.device)
    n = len(ds)
    net = UNet(device=args.device, seed=args.seed)
    t0 = time.perf_counter()
    selection = None
    if args.adopt:
        net.load(args.adopt)
        n_train, n_test = 0, n
        before = net.evaluate(ds, 0, n)
        loss, after, train_err = None, before, None
    else:
        n_train = max(1, int(round(0.9 * n)))
        n_test = n - n_train
        if args.init:
            net.load(args.init)
        net.train(ds, 0, n_train, steps=1, lr=0.0)  # output scale from the training targets
        before = net.evaluate(ds, n_train, n_test) if n_test else None
        if args.select_every > 0 and n_test:
            with tempfile.TemporaryDirectory() as tmp:
                best_path = pathlib.Path(tmp) / "best.bin"
                net.save(best_path)
                best = net.evaluate_warm(ds, n_train, n_test, args.residual_sweeps)
                selection = [[0, best]]
                done, loss = 0, None
                while done < args.train_steps:
                    k = min(args.select_every, args.train_steps - done)
                    lr_k = args.lr * 0.5 * (1.0 + math.cos(math.pi * done / args.train_steps))
                    loss = net.train(ds, 0, n_train, steps=k, lr=lr_k, seed=args.seed + done,
                                     out_scale=net.output_scale(), residual_weight=args.residual_weight,
                                     residual_sweeps=args.residual_sweeps)
                    done += k
                    r = net.evaluate_warm(ds, n_train, n_test, args.residual_sweeps)
                    selection.append([done, r])
                    if r < best:
                        best = r
                        net.save(best_path)
                net.load(best_path)
        else:
            loss = net.train(ds, 0, n_train, steps=args.train_steps, lr=args.lr, seed=args.seed,
                             out_scale=net.output_scale(), residual_weight=args.residual_weight,
                             residual_sweeps=args.residual_sweeps)
        after = net.evaluate(ds, n_train, n_test) if n_test else None
        train_err = net.evaluate(ds, 0, min(n_train, 64))
    train_s = time.perf_counter() - t0
    calibration = None
    if args.calibrate_scale and n_test:
        base = net.output_scale()
        calibration = []
        for k in (0.25, 0.35, 0.5, 0.7, 1.0, 1.4, 2.0):
            net.set_output_scale(base * k)
            calibration.append([base * k, net.evaluate_warm(ds, n_train, n_test, args.residual_sweeps)])
        best = min(calibration, key=lambda t: t[1])
        net.set_output_scale(best[0])
    out = pathlib.Path(args.out) if args.out else WEIGHTS_DIR / f"unet_{args.size}.bin"
    out.parent.mkdir(parents=True, exist_ok=True)
    net.save(out)
    warm = check_warm(net, args.size, args.device) if args.check_warm else None
    print(json.dumps(dict(info, size=args.size, train_pairs=n_train, test_pairs=n_test, warm_check=warm,
                          adopted=args.adopt, init=args.init, scale_calibration=calibration,
                          selection=selection,
                          residual_weight=args.residual_weight, residual_sweeps=args.residual_sweeps,
                          train_steps=args.train_steps, train_s=train_s, final_loss=loss,
                          test_rel_error_before=before, test_rel_error_after=after,
                          train_rel_error=train_err, output_scale=net.output_scale(), weights=str(out),
                          parameters=net.parameter_count())), flush=True)


if __name__ == "__main__":
    main()
