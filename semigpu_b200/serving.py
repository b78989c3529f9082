"""Serving: molecules arrive one by one, results stream back, work overlaps on the device.

A `Server` owns `slots` workers on one GPU.  Each worker has its own engine context (its own
CUDA streams), so the persistent launches of different workers run concurrently on the device.
A free worker takes every request waiting in its queue -- up to `max_batch` molecules and up to
its share of the HBM budget, by each molecule's device footprint -- builds one device batch
(integrals, Hcore, P, F, density stay resident for the whole SCF) and runs it; requests that
arrive meanwhile wait for the next free worker, so batches form continuously from whatever has
arrived (continuous batching at launch granularity).

Requests are queued by size: molecules up to nao 160 (SCF matrices in shared memory, a few ms)
and larger ones (up to nao 1024 in the batch, seconds at the top of the range) have separate
queues, and `big_slots` of the workers serve only the large queue, so a small request never
waits for a batch that holds a large molecule.  Molecules above nao 1024 run through the
single-molecule grid path in the large-queue worker that picked them.

`solver` picks how each SCF step gets the density (SOLVER_PURIFY, the FP64 default, or
SOLVER_PURIFY_MIXED: TF32 tensor-core products with an FP64 finish, within 1e-4 eV of FP64).
`diis` (depth 2..8, default off) turns on Pulay DIIS in every worker: fewer SCF steps per
molecule, converged energies within the SCF tolerance of the plain loop's, step counts no longer
the reference's.

Latency of a request = completion time - arrival time (host clock); `stats()` reports p50/p99
and throughput.  `replay()` drives an open-loop arrival schedule (e.g. Poisson) in real time.
"""
from __future__ import annotations

import collections
import threading
import time
from dataclasses import dataclass, field

import numpy as np

from . import SOLVER_PURIFY, SOLVER_PURIFY_MIXED, Context, Molecule, run_molecules
from .geometry import Molecule as Geometry

CTA_MAX_NAO = 1024  # larger molecules take the grid path
SMEM_MAX_NAO = 160  # above this a batched molecule also holds its work matrices in global memory
# nao 129-160: the largest shared-memory class, one CTA of ~225 KB shared memory, which starts
# only on an SM with nothing else resident
WHOLE_SM_NAO = 128


def device_bytes(mol: Geometry, diis: int = 0) -> int:
    """Device memory a molecule occupies inside a batch (integral blocks, Hcore/P/F packed,
    eigenvectors + F full square (+ the work matrices above nao 160), eigenvalues, atom
    arrays, and with DIIS of depth `diis` its history of 2 diis + 1 squares)."""
    heavy = int(np.count_nonzero(mol.Z > 1))
    light = mol.natoms - heavy
    nblk = 100 * heavy * (heavy + 1) // 2 + 10 * heavy * light + light * (light + 1) // 2
    n = mol.nao
    squares = 2 * n * n
    if diis >= 2:
        squares += (2 * diis + 1) * n * n + 128
    if n > SMEM_MAX_NAO:  # work matrices X and Y of purification, n16 x (n16 + 8) each
        n16 = (n + 15) // 16 * 16
        squares += max(n * n, 2 * n16 * (n16 + 8))
    return 8 * (nblk + 3 * n * (n + 1) // 2 + squares + n) + 64 * mol.natoms + 256


@dataclass
class Request:
    rid: int
    mol: Geometry
    t_arrival: float
    t_submit: float = 0.0  # when submit() ran (replay() sets t_arrival to the scheduled time)
    t_start: float = 0.0
    t_done: float = 0.0
    result: dict = field(default_factory=dict)


class Server:
    def __init__(self, device: int = 0, slots: int = 3, max_batch: int = 4096,
                 hbm_budget: int = 16 << 30, tol: float = 1e-6, max_iter: int = 100,
                 batch_window_s: float = 0.0, engine=None, big_slots: int = 1,
                 big_sm_share: float = 0.95, solver: int | None = None, diis: int = 0,
                 mid_slots: int = 0):
        """engine(ctx, mols, tol, max_iter) -> dict of arrays (defaults to run_molecules);
        replaceable for host-only tests of the scheduling.  big_slots of the slots serve the
        queue of molecules above nao 160 (at least one slot stays with the small queue); their
        launches together use at most big_sm_share of the SMs, so the persistent large-molecule
        launches (seconds) always leave SMs to the small ones.  solver: the density solver of
        every worker context (None: the library default); diis: DIIS depth of every worker
        context (0: off).  mid_slots of the slots (taken from the small ones, at least one
        small slot stays) serve a third queue, molecules of nao 129-160: their CTA needs a whole
        SM, and while the large launches hold most SMs it can wait for one for as long as a
        large batch runs; in their own queue they no longer hold up the other small requests."""
        self.solver = solver
        self.diis = diis
        self.big_sm_share = big_sm_share
        self.tol, self.max_iter = tol, max_iter
        self.max_batch = max_batch
        self.slot_budget = hbm_budget // max(1, slots)
        self.window = batch_window_s
        self.engine = engine or run_molecules
        self._queues = (collections.deque(), collections.deque(), collections.deque())
        # small, large, whole-SM (nao 129-160)
        self.big_slots = max(0, min(big_slots, slots - 1))
        self.mid_slots = max(0, min(mid_slots, slots - self.big_slots - 1))
        self._cv = threading.Condition()
        self._done: list[Request] = []
        self._next = 0
        self._stop = False
        self._device = device
        # the last big_slots workers serve the large queue, the mid_slots before them the
        # whole-SM one
        def kind(i):
            if i >= slots - self.big_slots:
                return 1
            return 2 if i >= slots - self.big_slots - self.mid_slots else 0

        self._workers = [threading.Thread(target=self._work, args=(i, kind(i)), daemon=True)
                         for i in range(slots)]
        self.batches: list[tuple[int, int, float, float]] = []  # (worker, size, t0, t1)
        self._errors: list[BaseException] = []
        for w in self._workers:
            w.start()

    # -- client side -----------------------------------------------------------------------
    def submit(self, mol: Geometry, t_arrival: float | None = None) -> int:
        with self._cv:
            rid = self._next
            self._next += 1
            now = time.perf_counter()
            req = Request(rid, mol, now if t_arrival is None else t_arrival, t_submit=now)
            if self.big_slots > 0 and mol.nao > SMEM_MAX_NAO:
                q = 1
            elif self.mid_slots > 0 and mol.nao > WHOLE_SM_NAO:
                q = 2
            else:
                q = 0
            self._queues[q].append(req)
            self._cv.notify_all()
        return rid

    def drain(self, timeout: float = 600.0) -> list[Request]:
        """Waits until every submitted request has completed; returns them by request id."""
        t_end = time.perf_counter() + timeout
        with self._cv:
            while len(self._done) < self._next:
                if self._errors:
                    raise self._errors[0]
                left = t_end - time.perf_counter()
                if left <= 0:
                    raise TimeoutError(f"{self._next - len(self._done)} requests unfinished")
                self._cv.wait(min(left, 0.05))
            return sorted(self._done, key=lambda r: r.rid)

    def close(self):
        with self._cv:
            self._stop = True
            self._cv.notify_all()
        for w in self._workers:
            w.join(timeout=60)

    def replay(self, arrivals, time_scale: float = 1.0) -> list[Request]:
        """Submits (t, molecule) pairs at their arrival times (open loop), waits for all and
        returns this replay's requests (earlier ones, e.g. a warm-up, are left out)."""
        with self._cv:
            first = self._next
        t0 = time.perf_counter()
        for t, mol in arrivals:
            delay = t0 + t * time_scale - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
            self.submit(mol, t_arrival=t0 + t * time_scale)
        return [r for r in self.drain() if r.rid >= first]

    # -- worker side ------------------------------------------------------------------------
    def _take(self, queue) -> list[Request]:
        """Everything waiting in `queue`, up to max_batch molecules and this worker's HBM
        share."""
        out, used = [], 0
        while queue and len(out) < self.max_batch:
            need = device_bytes(queue[0].mol, self.diis)
            if out and used + need > self.slot_budget:
                break
            used += need
            out.append(queue.popleft())
        return out

    def _work(self, idx: int, kind: int = 0):
        queue = self._queues[kind]
        big = kind == 1
        ctx = None
        try:
            if self.engine is run_molecules:
                ctx = Context(self._device)
                if self.solver is not None:
                    ctx.set_density_solver(self.solver)
                if self.diis:
                    ctx.set_diis(self.diis)
                if big and self.big_slots:
                    ctx.set_sm_share(max(0.05, self.big_sm_share / self.big_slots))
                elif self.big_slots:
                    # small batches take freed SMs ahead of the large launches' waiting blocks
                    ctx.set_priority(True)
                # batches are built in a per-worker arena: no cudaMalloc/cudaFree per batch
                # (cudaFree would synchronise the device and stall the other workers)
                ctx.reserve(self.slot_budget + (64 << 20))
            while True:
                with self._cv:
                    while not queue and not self._stop:
                        self._cv.wait(0.05)
                    if self._stop and not queue:
                        return
                if self.window:
                    time.sleep(self.window)
                with self._cv:
                    reqs = self._take(queue)
                if not reqs:
                    continue
                t0 = time.perf_counter()
                for r in reqs:
                    r.t_start = t0
                small = [r for r in reqs if r.mol.nao <= CTA_MAX_NAO]
                large = [r for r in reqs if r.mol.nao > CTA_MAX_NAO]
                if small:
                    res = self.engine(ctx, [r.mol for r in small], self.tol, self.max_iter)
                    t1 = time.perf_counter()
                    for j, r in enumerate(small):
                        r.result = {k: (v[j].item() if hasattr(v[j], "item") else v[j])
                                    for k, v in res.items()}
                        r.t_done = t1
                for r in large:
                    if self.engine is run_molecules:
                        m = Molecule.from_geometry(ctx, r.mol)
                        res = m.run(tol=self.tol, max_iter=self.max_iter)
                        m.close()
                        r.result = {k: res[k] for k in ("E_el", "E_cc", "E_tot", "n_iter",
                                                        "converged", "status")}
                    else:
                        res = self.engine(ctx, [r.mol], self.tol, self.max_iter)
                        r.result = {k: (v[0].item() if hasattr(v[0], "item") else v[0])
                                    for k, v in res.items()}
                    r.t_done = time.perf_counter()
                with self._cv:
                    self.batches.append((idx, len(reqs), t0, time.perf_counter()))
                    self._done.extend(reqs)
                    self._cv.notify_all()
        except BaseException as exc:  # surfaced to drain()
            with self._cv:
                self._errors.append(exc)
                self._cv.notify_all()
        finally:
            if ctx is not None:
                ctx.close()


def stats(done: list[Request]) -> dict:
    """p50/p99 time-to-converged-energy (arrival -> result) and throughput (requests over the
    span from the first arrival to the last result, so the final drain counts against it).
    Whether the load is sustained shows in p50_ms_by_arrival_quarter: the p50 latency of the
    requests arriving in each quarter of the arrival span, flat when no backlog builds, and in
    drain_ms, the time from the last arrival to the last result."""
    if not done:
        return {}
    lat = np.array([r.t_done - r.t_arrival for r in done])
    arr = np.array([r.t_arrival for r in done])
    t_first, t_last_arrival = float(arr.min()), float(arr.max())
    t_last = max(r.t_done for r in done)
    span = max(t_last_arrival - t_first, 1e-9)
    quarter = np.minimum((4 * (arr - t_first) / span).astype(int), 3)
    return {"requests": len(done), "p50_ms": 1e3 * float(np.percentile(lat, 50)),
            "p99_ms": 1e3 * float(np.percentile(lat, 99)),
            "molecules_per_s": len(done) / (t_last - t_first) if t_last > t_first else float("nan"),
            "p50_ms_by_arrival_quarter": [
                1e3 * float(np.percentile(lat[quarter == k], 50)) if np.any(quarter == k) else None
                for k in range(4)],
            "drain_ms": 1e3 * (t_last - t_last_arrival),
            # how late the replay submitted requests against their schedule (host-side lag that
            # the latencies above include)
            "submit_lag_p99_ms": 1e3 * float(np.percentile(
                [max(0.0, r.t_submit - r.t_arrival) if r.t_submit else 0.0 for r in done], 99)),
            "all_converged": bool(all(r.result.get("converged", False) for r in done))}


def main(argv=None):
    """Replays seeded open-loop Poisson arrivals and prints latency and throughput, overall and
    for the small (nao <= 160) and large molecules:

        python -m semigpu_b200.serving --workload c5 --rate 2000 --duration 3
    """
    import argparse
    import json

    from . import geometry as geo

    ap = argparse.ArgumentParser(description=main.__doc__)
    ap.add_argument("--workload", choices=["c3", "c5"], default="c5",
                    help="c3: the 4096-batch composition; c5: alkanes extended to C150H302")
    ap.add_argument("--rate", type=float, default=2000.0, help="requests per second")
    ap.add_argument("--duration", type=float, default=3.0, help="seconds of arrivals")
    ap.add_argument("--slots", type=int, default=4)
    ap.add_argument("--big-slots", type=int, default=2)
    ap.add_argument("--mid-slots", type=int, default=0,
                    help="workers of their own for nao 129-160 (whole-SM CTAs)")
    ap.add_argument("--hbm-gb", type=float, default=40.0)
    ap.add_argument("--big-share", type=float, default=0.95,
                    help="fraction of the SMs the large-molecule workers' launches may use")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--mixed", action="store_true",
                    help="mixed precision (TF32 tensor-core products, FP64 finish)")
    ap.add_argument("--diis", type=int, default=0, help="DIIS depth (2..8; 0: off)")
    args = ap.parse_args(argv)
    if args.workload == "c5":
        arrivals = geo.serving_c5(rate=args.rate, duration_s=args.duration, seed=args.seed)
    else:
        rng = np.random.default_rng(args.seed + 1)
        t, times = 0.0, []
        while True:
            t += rng.exponential(1.0 / args.rate)
            if t >= args.duration:
                break
            times.append(t)
        arrivals = list(zip(times, geo.batch_c3(len(times), seed=args.seed)))
    srv = Server(slots=args.slots, big_slots=args.big_slots, mid_slots=args.mid_slots,
                 hbm_budget=int(args.hbm_gb * (1 << 30)),
                 big_sm_share=args.big_share,
                 solver=SOLVER_PURIFY_MIXED if args.mixed else SOLVER_PURIFY, diis=args.diis)
    try:
        srv.replay([(0.001 * i, m) for i, (_, m) in enumerate(arrivals[:40])])  # warm-up
        done = srv.replay(arrivals)
    finally:
        srv.close()
    out = {"workload": args.workload, "rate_per_s": args.rate, "duration_s": args.duration,
           "precision": "mixed" if args.mixed else "fp64", "big_share": args.big_share,
           "diis": args.diis,
           "all": stats(done),
           "small": stats([r for r in done if r.mol.nao <= SMEM_MAX_NAO]),
           "large": stats([r for r in done if r.mol.nao > SMEM_MAX_NAO]),
           "max_nao": max(r.mol.nao for r in done)}
    print(json.dumps(out))


if __name__ == "__main__":
    main()
