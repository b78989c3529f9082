"""Autotuners: the CTA size of each nao size class of the batched launch (`tune`), and the tile
configuration of the whole-GPU purification for one large molecule (`tune_grid`), by timing.

Each size class of `k_batch_scf` can run with CTAs of 128 (classes up to nao 64), 256 or 512
threads; smaller CTAs fit more molecules per SM, larger ones give each molecule more warps for
its products and Fock build.  `tune()` times a batch with every admissible choice for one class
at a time (coordinate descent from the defaults, classes in order of their share of the run),
keeps a choice only when it beats the current best by more than `min_gain`, and returns the
per-class CTA sizes; `Context.set_class_threads` applies them.  The measured times are device
times of the persistent launches (the library's own events), medians over `repeats` runs.

    python -m semigpu_b200.autotune --batch 4096 --out tuned.json
"""
from __future__ import annotations

import json
import statistics

import numpy as np

from . import Batch, Context, size_classes


def _time(ctx: Context, batch: Batch, threads, repeats: int, tol: float) -> float:
    ctx.set_class_threads(threads)
    batch.run(tol)
    batch.results()
    ms = []
    for _ in range(repeats):
        batch.run(tol)
        batch.results()
        ms.append(batch.last_ms())
    return statistics.median(ms)


def candidates(k: int, classes) -> list[int]:
    nmax, default = classes[k]
    if default == 512 and nmax > 160:  # the large-molecule classes stream from global memory
        return [512]
    return [128, 256, 512] if nmax <= 64 else [256, 512]


def tune(ctx: Context, mols, repeats: int = 3, tol: float = 1e-6, min_gain: float = 0.01) -> dict:
    """Per-class CTA sizes for `mols` on this context's GPU.  Returns {"class_threads": [...],
    "ms": best, "default_ms": ..., "trials": [(threads, ms), ...]}."""
    classes = size_classes()
    present = sorted({next(k for k, (nm, _) in enumerate(classes) if m.nao <= nm) for m in mols})
    best = [t for _, t in classes]
    batch = Batch(ctx, mols)
    try:
        default_ms = best_ms = _time(ctx, batch, best, repeats, tol)
        trials = [(list(best), default_ms)]
        # classes holding the most n^3 work first
        work = {k: sum(m.nao ** 3 for m in mols
                       if next(c for c, (nm, _) in enumerate(classes) if m.nao <= nm) == k)
                for k in present}
        for k in sorted(present, key=lambda c: -work[c]):
            for t in candidates(k, classes):
                if t == best[k]:
                    continue
                trial = list(best)
                trial[k] = t
                ms = _time(ctx, batch, trial, repeats, tol)
                trials.append((trial, ms))
                if ms < best_ms * (1.0 - min_gain):
                    best, best_ms = trial, ms
        ctx.set_class_threads(best)
    finally:
        batch.close()
    return {"class_threads": best, "ms": best_ms, "default_ms": default_ms, "trials": trials}


def main(argv=None):
    import argparse

    from . import geometry as geo

    ap = argparse.ArgumentParser(description="Pick the CTA size per nao size class by timing.")
    ap.add_argument("--batch", type=int, default=4096)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--repeats", type=int, default=3)
    ap.add_argument("--out", default=None, help="write the result as JSON here")
    args = ap.parse_args(argv)
    ctx = Context(0)
    try:
        res = tune(ctx, geo.batch_c3(args.batch, seed=args.seed), repeats=args.repeats)
    finally:
        ctx.close()
    text = json.dumps(res)
    if args.out:
        with open(args.out, "w") as fh:
            fh.write(text + "\n")
    print(text)


if __name__ == "__main__":
    main()


def tune_grid(ctx: Context, mol, repeats: int = 2, steps: int = 1, tol: float = 1e-6,
              min_gain: float = 0.01) -> dict:
    """Tile configuration of the whole-GPU purification for molecules like `mol` (a geometry
    above nao 160): times `steps` SCF steps of `mol` with every configuration of
    `grid_configs()` (the automatic choice first), keeps the fastest if it beats the automatic
    one by more than `min_gain`, and applies it to `ctx` (Context.set_grid_config).  Returns
    {"config": index or -1, "ms": ..., "auto_ms": ..., "trials": [(config, ms), ...]}."""
    import time

    from . import Molecule, grid_configs

    def run(cfg):
        ctx.set_grid_config(cfg)
        best = float("inf")
        for _ in range(repeats + 1):  # the first run also compiles nothing but warms the arenas
            m = Molecule(ctx, mol.Z, mol.xyz)
            m.set_path(2)  # PATH_GRID
            m.two_center()
            m.hcore()
            ctx.synchronize()
            t0 = time.perf_counter()
            m.scf(tol=tol, max_iter=steps)
            best = min(best, time.perf_counter() - t0)
            m.close()
        return 1e3 * best

    trials = [(-1, run(-1))]
    for k in range(len(grid_configs())):
        trials.append((k, run(k)))
    auto_ms = trials[0][1]
    cfg, ms = min(trials[1:], key=lambda t: t[1])
    if not ms < auto_ms * (1.0 - min_gain):
        cfg, ms = -1, auto_ms
    ctx.set_grid_config(cfg)
    return {"config": cfg, "ms": ms, "auto_ms": auto_ms, "trials": trials}
