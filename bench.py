"""Benchmark: converged SCF molecules/s on the 4096-molecule uneven batch (FP64, tol 1e-6 eV).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With --gpus N > 1 and no torchrun around it, bench.py starts N ranks of itself under
torch.distributed.run; under torchrun, WORLD_SIZE must equal N.

A step is one persistent launch that takes every molecule of the batch from coordinates to
converged total energy (integrals, Hcore, SCF, core-core).  `value` is device-timed
(CUDA events recorded by the library around each launch, inputs resident in HBM);
`e2e` goes through the public C ABI (sgb_run_molecules) from pinned host arrays with the
coordinate upload and the result read-back inside the timed region.  Multi-GPU: one process
per GPU under torchrun, each rank runs its own seeded 4096-molecule batch (weak scaling, no
collective on the data path); time is the max over ranks.

--impl reference times the reference's own CPU build (oracle/_ref/ref_driver, the unmodified
LuisAlfredoNu/semiGPU sources compiled serially) on bounded samples of the same workload, one
molecule per process on all host cores; rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "converged SCF molecules/s + p50/p99 latency vs plain FP64 GPU, |ΔE|≤1e-4 eV"
UNIT = "molecules/s"
BATCH = 4096
TOL = 1e-6
WORKLOAD = ("uneven batch of 4096 seeded molecules per GPU: 50% CnH2n+2 (n=1..20), 30% all-trans "
            "CnHn+2 (n even 2..30), 20% aza-aromatic rings (0-3 N); coordinates jittered "
            "N(0,0.01 A); FP64; SCF to |dE| < 1e-6 eV")


def env_int(name, default):
    try:
        return int(os.environ.get(name, default))
    except ValueError:
        return default


# ------------------------------------------------------------------------------------------
# Clock sampling during the timed region

class ClockSampler:
    """nvidia-smi samples of the SM clock and throttle reasons of the given GPUs (every rank's
    GPU when rank 0 samples for the job), every 200 ms while the timed region runs."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, devices):
        self.devices = [devices] if isinstance(devices, int) else list(devices)
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", ",".join(str(d) for d in self.devices),
                 f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        rows = []
        try:
            for line in open(self.path):
                f = [x.strip() for x in line.split(",")]
                if len(f) >= 9:
                    rows.append(f)
        except OSError:
            pass
        finally:
            if self.path and os.path.exists(self.path):
                os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}

        def num(x):
            try:
                return float(x)
            except ValueError:
                return None
        sm = [num(r[1]) for r in rows if num(r[1]) is not None]
        mx = [num(r[2]) for r in rows if num(r[2]) is not None]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(rows), "gpus": sorted({r[0] for r in rows})}


# ------------------------------------------------------------------------------------------
# Algorithmic work (the roofline numerator)

def algorithmic_flops(mols, n_iter) -> float:
    """Per SCF step and molecule: eigensolve (10/3) N^3 (Householder tridiagonalisation +
    back-transform, independent of the algorithm run) + density 2 N^2 nocc; summed over the
    steps each molecule took."""
    tot = 0.0
    for m, it in zip(mols, n_iter):
        n, o = m.nao, m.nocc
        tot += float(it) * ((10.0 / 3.0) * n ** 3 + 2.0 * n * n * o)
    return tot


def fp64_peak_tflops(torch):
    """Measured cuBLAS DGEMM throughput (the FP64 peak the roofline is quoted against);
    cached in profiles/fp64_peak.json once measured on this pool."""
    path = os.path.join(ROOT, "profiles", "fp64_peak.json")
    if os.path.exists(path):
        with open(path) as fh:
            return json.load(fh)["dgemm_tflops"], "profiles/fp64_peak.json (measured cuBLAS DGEMM)"
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    for _ in range(2):
        a @ b
    torch.cuda.synchronize()
    best = 1e9
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(); a @ b; e1.record(); torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1) / 1e3)
    return 2 * n ** 3 / best / 1e12, "measured in this run (cuBLAS DGEMM 8192^3, best of 5)"


def load_traffic():
    path = os.path.join(ROOT, "profiles", "k_batch_scf_traffic.json")
    if os.path.exists(path):
        with open(path) as fh:
            return json.load(fh)
    return None


# ------------------------------------------------------------------------------------------
# CPU reference timing

def stratified_index(mols, k, offset=0):
    """Indices of k molecules at evenly spaced quantiles of nao, largest first (so a process
    pool schedules them longest-job-first)."""
    idx = np.argsort([m.nao for m in mols], kind="stable")
    pos = np.linspace(0, len(mols) - 1, k).round().astype(int)
    pos = np.clip(pos + offset, 0, len(mols) - 1)
    return [int(idx[p]) for p in pos[::-1]]


def stratified(mols, k, offset=0):
    return [mols[i] for i in stratified_index(mols, k, offset)]


def _ref_one(args):
    """One molecule through the reference build (single-threaded process, OpenBLAS on one
    thread); returns E_tot, steps, CPU-seconds and wall seconds of that process."""
    import resource

    Z, xyz = args
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    c0 = resource.getrusage(resource.RUSAGE_CHILDREN)
    t0 = time.perf_counter()
    r = oracle.run_reference(Z, xyz, tol=TOL, matrices=False)
    wall = time.perf_counter() - t0
    c1 = resource.getrusage(resource.RUSAGE_CHILDREN)
    cpu = (c1.ru_utime + c1.ru_stime) - (c0.ru_utime + c0.ru_stime)
    return r["E_tot"], r["n_iter"], cpu, wall


def _pool_ready(_):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle  # noqa: F401

    return os.getpid()


def cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as fh:
            for line in fh:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def reference_queue(sample, cores):
    """The reference build over `sample` as a work queue: one single-threaded reference process
    per core, molecules handed out longest first (the sample is ordered by decreasing nao, the
    cost being ~nao^4 per Fock build), each core taking the next molecule as soon as it is
    free.  The pool is started before the timed region.  Returns wall seconds, the summed
    CPU-seconds of the reference processes and the per-molecule results."""
    import multiprocessing as mp

    ctx = mp.get_context("spawn")
    workers = min(cores, len(sample))
    with ctx.Pool(workers) as pool:
        pool.map(_pool_ready, range(workers), chunksize=1)
        t0 = time.perf_counter()
        out = list(pool.imap(_ref_one, [(m.Z, m.xyz) for m in sample], chunksize=1))
        wall = time.perf_counter() - t0
    return wall, sum(o[2] for o in out), out


def cpu_baseline_record(sample, cores, wall, cpu_s, label):
    """The cpu_baseline object: whole-queue throughput on `cores` cores, with the CPU-seconds
    per molecule, the cores' busy fraction and the serial (one core) throughput beside it."""
    n = len(sample)
    return {"value": n / wall, "unit": UNIT, "cores": min(cores, n), "kind": "reference",
            "cpu_model": cpu_model(), "host_cores": os.cpu_count(),
            "cpu_s_per_molecule": cpu_s / n, "wall_s": wall,
            "utilization": cpu_s / (wall * min(cores, n)),
            "serial_1core": {"value": n / cpu_s, "unit": UNIT,
                             "how": "molecules / summed CPU-seconds of the single-threaded "
                                    "reference processes (OPENBLAS_NUM_THREADS=1)"},
            "sample": f"{n} molecules of {label}, stratified by nao, one work queue "
                      f"(longest first) over {min(cores, n)} single-threaded reference processes"}


def reference_kind():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    return "reference" if oracle.reference_available() else None


# ------------------------------------------------------------------------------------------

def run_reference_arm(args):
    from semigpu_b200 import geometry as geo

    rank = env_int("RANK", 0)
    if rank != 0:
        return
    if reference_kind() is None:
        print(json.dumps({"impl": "reference", "unavailable":
                          "oracle/_ref/ref_driver not built (the reference tree was absent when "
                          "oracle/Makefile ran)"}))
        return
    mols = geo.batch_c3(BATCH, seed=0)
    cores = os.cpu_count() or 1
    # one stratified sample of ~256 molecules (at least one per core and step), run as a single
    # work queue across the K timed steps so the cores stay busy; warm-up: a few small ones
    per_step = max(cores, -(-256 // max(1, args.steps)))
    sample = stratified(mols, per_step * args.steps)
    small = sorted(mols, key=lambda m: m.nao)[: len(mols) // 4]
    if args.warmup:
        reference_queue(stratified(small, max(1, min(cores, 2 * args.warmup))), cores)
    wall, cpu_s, _ = reference_queue(sample, cores)
    value = len(sample) / wall
    cpu = cpu_baseline_record(sample, cores, wall, cpu_s, "the seed-0 4096-molecule batch")
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * wall / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "impl": "reference",
        "config": {"workload": WORKLOAD, "sample_per_step": per_step,
                   "sample": f"{len(sample)} molecules stratified by nao over the seed-0 batch, "
                             f"one work queue over the {args.steps} steps"},
        "cpu_baseline": cpu,
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def run_ours(args):
    import torch
    import torch.distributed as dist

    import semigpu_b200 as sg
    from semigpu_b200 import geometry as geo

    world = env_int("WORLD_SIZE", 1)
    rank = env_int("RANK", 0)
    local = env_int("LOCAL_RANK", 0)
    if world > 1:
        torch.cuda.set_device(local)
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)

    nb = args.batch
    mols = geo.batch_c3(nb, seed=rank)
    ctx = sg.Context(local)
    tuned = None
    if not args.no_tune:
        # CTA size per nao size class, chosen by timing this batch (semigpu_b200/autotune.py);
        # untimed, before the warm-up
        from semigpu_b200 import autotune

        tuned = autotune.tune(ctx, mols, repeats=2)
    batch = sg.Batch(ctx, mols)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)  # > L2

    def barrier():
        torch.cuda.synchronize(dev)
        ctx.synchronize()
        if world > 1:
            dist.barrier()

    for _ in range(args.warmup):
        batch.run(TOL)
        res = batch.results()
    barrier()
    kernel_ms = []
    lat_p50, lat_p99 = [], []
    with ClockSampler(list(range(world)) if rank == 0 else [local]) as clocks:
        for _ in range(args.steps):
            flush.fill_(1.0)
            torch.cuda.synchronize(dev)
            batch.run(TOL)
            res = batch.results()
            kernel_ms.append(batch.last_ms())
            tb, te = batch.timestamps()
            lat = (te.astype(np.float64) - float(tb.min())) / 1e6
            lat_p50.append(float(np.percentile(lat, 50)))
            lat_p99.append(float(np.percentile(lat, 99)))
        barrier()
    clk = clocks.summary()
    my_ms = float(sum(kernel_ms))
    t = torch.tensor([my_ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    total_ms = float(t.item())
    ok = bool(np.all(res["status"] == 0) and np.all(res["converged"]))
    value = world * nb * args.steps / (total_ms / 1e3)
    if args.kernel_only:
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
                              "steps": args.steps, "warmup": args.warmup,
                              "ms_per_step": total_ms / args.steps, "kernel_only": True,
                              "molecules_per_gpu": nb, "all_converged": ok, "clocks": clk}))
        batch.close()
        ctx.close()
        if world > 1:
            dist.destroy_process_group()
        return

    # e2e through the C ABI from pinned host memory: upload coordinates, run, read results
    natoms = np.array([m.natoms for m in mols], np.int32)
    rng = np.random.default_rng(100 + rank)
    pinned = torch.empty(int(natoms.sum()) * 3, dtype=torch.float64).pin_memory().numpy()
    base = np.concatenate([m.xyz.reshape(-1) for m in mols])
    e2e_mols = [geo.Molecule(m.Z, m.xyz) for m in mols]
    sg.run_molecules(ctx, e2e_mols, tol=TOL)  # builds the cached device batch
    barrier()
    e2e_s = 0.0
    for _ in range(args.steps):
        pinned[:] = base + rng.normal(0.0, 1e-4, base.shape)
        off = 0
        for m in e2e_mols:
            k = m.natoms * 3
            m.xyz = pinned[off:off + k].reshape(-1, 3)
            off += k
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        r = sg.run_molecules(ctx, e2e_mols, tol=TOL)
        e2e_s += time.perf_counter() - t0
    te2e = torch.tensor([e2e_s], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(te2e, op=dist.ReduceOp.MAX)
    e2e_value = world * nb * args.steps / float(te2e.item())
    ok = ok and bool(np.all(r["status"] == 0))

    mixed = diis = None
    if rank == 0:
        # the mixed-precision form on the same batch (TF32 tensor-core products with an FP64
        # finish, sgb SOLVER_PURIFY_MIXED): its speed and its error against the FP64 run above
        ctx.set_density_solver(sg.SOLVER_PURIFY_MIXED)
        batch.run(TOL)
        batch.results()
        mms = []
        for _ in range(3):
            flush.fill_(1.0)
            torch.cuda.synchronize(dev)
            batch.run(TOL)
            rm = batch.results()
            mms.append(batch.last_ms())
        ctx.set_density_solver(sg.SOLVER_PURIFY)
        dE = np.abs(rm["E_tot"] - res["E_tot"])
        # optional Pulay DIIS (depth 6) on the same batch: fewer SCF steps than the reference's
        # plain loop, the same converged energies
        ctx.set_diis(6)
        batch.run(TOL)
        batch.results()
        dms = []
        for _ in range(3):
            flush.fill_(1.0)
            torch.cuda.synchronize(dev)
            batch.run(TOL)
            rd = batch.results()
            dms.append(batch.last_ms())
        ctx.set_diis(0)
        diis = {"value": nb / (statistics.median(dms) / 1e3), "unit": UNIT,
                "ms_per_step": statistics.median(dms), "depth": 6,
                "mean_n_iter": float(np.mean(rd["n_iter"])),
                "mean_n_iter_plain": float(np.mean(res["n_iter"])),
                "max_abs_dE_total_eV": float(np.max(np.abs(rd["E_tot"] - res["E_tot"]))),
                "all_converged": bool(np.all(rd["converged"]))}
        mixed = {"value": nb / (statistics.median(mms) / 1e3), "unit": UNIT,
                 "ms_per_step": statistics.median(mms),
                 "max_abs_dE_total_eV": float(dE.max()), "tolerance_eV": 1e-4,
                 "n_iter_changed": int(np.sum(rm["n_iter"] != res["n_iter"])),
                 "all_converged": bool(np.all(rm["converged"])),
                 "form": "TF32 tcgen05 products (3xTF32) above nao 64, FP64 below and for the "
                         "finish of every purification"}
    if rank == 0:
        peak, peak_src = fp64_peak_tflops(torch)
        flops = algorithmic_flops(mols, res["n_iter"])
        achieved = flops / (my_ms / args.steps / 1e3) / 1e12
        traffic = load_traffic()
        roof = {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                "frac": achieved / peak, "traffic": None,
                "kernel": "k_batch_scf (one persistent launch per nao size class; FP64 pipe)",
                "peak_source": peak_src,
                "numerator": "sum over molecules of n_iter*((10/3)N^3 + 2 N^2 nocc) FP64 flops"}
        if traffic:
            roof["traffic"] = traffic["dram_bytes_per_molecule"] * nb
            roof["traffic_source"] = traffic["source"]
        # plain FP64 GPU path: one molecule at a time through the stage API (same kernels,
        # one CTA per launch), on a stratified sample
        sample = stratified(mols, 48)
        warm = sg.Molecule.from_geometry(ctx, sample[0])  # first-call set-up stays untimed
        warm.run(tol=TOL)
        warm.close()
        tp = time.perf_counter()
        plain_lat = []
        for m in sample:
            t1 = time.perf_counter()
            one = sg.Molecule.from_geometry(ctx, m)
            one.run(tol=TOL)
            one.close()
            plain_lat.append(time.perf_counter() - t1)
        plain = len(sample) / (time.perf_counter() - tp)
        # serving: open-loop Poisson arrivals of the same composition, continuous batching over
        # three worker contexts (semigpu_b200.serving); warmed up first
        from semigpu_b200 import serving

        srate, sdur = 2000.0, 3.0
        srng = np.random.default_rng(11)
        smols = geo.batch_c3(int(srate * sdur * 1.3) + 64, seed=1000 + rank)
        arrivals, t_a = [], 0.0
        while True:
            t_a += srng.exponential(1.0 / srate)
            if t_a >= sdur:
                break
            arrivals.append((t_a, smols[len(arrivals)]))
        srv = serving.Server(device=local, slots=3, hbm_budget=12 << 30, tol=TOL)
        try:
            srv.replay([(0.001 * i, m) for i, m in enumerate(smols[-64:])])  # warm-up
            srv_done = srv.replay(arrivals)
        finally:
            srv.close()
        served = serving.stats(srv_done)
        served.update({"rate_per_s": srate, "duration_s": sdur, "slots": 3,
                       "composition": "as the batch (seeded), open-loop Poisson arrivals"})
        # the same stream served in mixed precision, each result against its FP64 one
        srv = serving.Server(device=local, slots=3, hbm_budget=12 << 30, tol=TOL,
                             solver=sg.SOLVER_PURIFY_MIXED)
        try:
            srv.replay([(0.001 * i, m) for i, m in enumerate(smols[-64:])])  # warm-up
            mix_done = srv.replay(arrivals)
        finally:
            srv.close()
        served_mixed = serving.stats(mix_done)
        served_mixed["max_abs_dE_total_eV"] = float(max(
            abs(a.result["E_tot"] - b.result["E_tot"]) for a, b in zip(mix_done, srv_done)))
        served_mixed["precision"] = "TF32 tcgen05 products for nao above 64, FP64 finish"
        # config-5 stream: 2000 requests/s of the batch composition with alkanes to C150H302
        # (nao <= 902) for the configuration's 60 s (10 s while other ranks' GPUs wait), mixed
        # precision, split by small (nao <= 160) and large requests; each request's error
        # against the FP64 result of the same molecule on a sample
        c5_dur = 60.0 if world == 1 else 10.0
        c5 = geo.serving_c5(rate=2000.0, duration_s=c5_dur, seed=0)
        srv = serving.Server(device=local, slots=4, big_slots=2, hbm_budget=40 << 30, tol=TOL,
                             solver=sg.SOLVER_PURIFY_MIXED, big_sm_share=0.95)
        try:
            srv.replay([(0.001 * i, m) for i, (_, m) in enumerate(c5[:40])])  # warm-up
            c5_done = srv.replay(c5)
        finally:
            srv.close()
        small_r = [r for r in c5_done if r.mol.nao <= serving.SMEM_MAX_NAO]
        large_r = [r for r in c5_done if r.mol.nao > serving.SMEM_MAX_NAO]
        pick = stratified_index([r.mol for r in c5_done], 256)
        ref64 = sg.run_molecules(ctx, [c5_done[i].mol for i in pick], tol=TOL)
        dE5 = np.abs(np.array([c5_done[i].result["E_tot"] for i in pick]) - ref64["E_tot"])
        serving_c5 = {
            "rate_per_s": 2000.0, "duration_s": c5_dur, "precision": "mixed",
            "composition": "config 5: batch composition with alkanes CnH2n+2 n=1..150 "
                           "(nao <= 902), seeded Poisson arrivals",
            "all": serving.stats(c5_done), "small_nao_le_160": serving.stats(small_r),
            "large_nao_gt_160": serving.stats(large_r),
            "large_arrival_rate_per_s": len(large_r) / c5_dur,
            "max_abs_dE_total_eV_vs_fp64": float(dE5.max()),
            "dE_sample": f"{len(pick)} requests stratified by nao, against an FP64 batch run",
            "slots": 4, "big_slots": 2, "big_sm_share": 0.95}
        # CPU baseline: the reference build on the host cores, bounded sample
        cpu = None
        if reference_kind():
            cores = os.cpu_count() or 1
            cidx = stratified_index(mols, max(cores, 160))
            csample = [mols[i] for i in cidx]
            dt, cpu_s, ref_out = reference_queue(csample, cores)
            cpu = cpu_baseline_record(csample, cores, dt, cpu_s, "the same batch")
            # the reference's own energies for these molecules: the error of the FP64 and of the
            # mixed-precision batch results against them
            e_ref = np.array([o[0] for o in ref_out])
            it_ref = np.array([o[1] for o in ref_out])
            d64 = np.abs(res["E_tot"][cidx] - e_ref)
            cpu["parity_on_sample"] = {
                "molecules": len(cidx), "max_abs_dE_total_eV_fp64": float(d64.max()),
                "n_iter_equal_fp64": int(np.sum(res["n_iter"][cidx] == it_ref))}
            if mixed is not None:
                dmx = np.abs(rm["E_tot"][cidx] - e_ref)
                mixed["vs_reference_sample"] = {
                    "molecules": len(cidx), "max_abs_dE_total_eV": float(dmx.max()),
                    "median_abs_dE_total_eV": float(np.median(dmx)),
                    "within_tolerance": bool(dmx.max() <= 1e-4),
                    "reference": "the reference build's E_tot (cpu_baseline leg)"}
        nat_total = int(natoms.sum())
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "molecules_per_gpu": nb, "tol_eV": TOL,
                       "class_threads": tuned["class_threads"] if tuned else
                       [t for _, t in sg.size_classes()],
                       "autotuned": tuned is not None,
                       "precision": "fp64", "parallelism": f"replicas x{world}",
                       "l2": "working set > L2 (integrals + eigenvector arenas); a 256 MB "
                             "buffer is written between timed steps"},
            "latency_ms": {"p50": statistics.median(lat_p50), "p99": statistics.median(lat_p99),
                           "definition": "per-molecule time from launch start to its converged "
                                         "energy, device clock"},
            "mixed_precision": mixed,
            "serving_mixed": served_mixed,
            "serving_c5": serving_c5,
            "diis": diis,
            "plain_fp64_gpu": {"value": plain, "unit": UNIT,
                               "p50_ms": 1e3 * statistics.median(plain_lat),
                               "p99_ms": 1e3 * float(np.percentile(plain_lat, 99)),
                               "sample": "48 molecules stratified by nao, one molecule per call "
                                         "through the stage API"},
            "speedup_vs_plain_fp64_gpu": value / plain,
            "serving": served,
            "all_converged": ok,
            "roofline": roof,
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 24 * nat_total,
                    "d2h_bytes_per_step": nb * (8 + 8 + 4 + 4 + 4)},
            "clocks": clk,
            "gpu_launches": args.steps * batch.launches(),
        }
        print(json.dumps(line))
    batch.close()
    ctx.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--batch", type=int, default=BATCH,
                    help="molecules per GPU (default: the 4096-molecule workload)")
    ap.add_argument("--no-tune", action="store_true",
                    help="keep the default CTA size per size class (skip the autotuner)")
    ap.add_argument("--kernel-only", action="store_true",
                    help="device-timed launches only (no e2e, plain-path or CPU legs); used "
                         "for profiler captures of a smaller batch")
    ap.add_argument("--probe-ranks", action="store_true",
                    help="print this process's rank and world size as JSON and exit (no GPU "
                         "work): shows how `--gpus N` lays out its processes")
    args = ap.parse_args()
    if args.gpus < 1:
        ap.error("--gpus must be >= 1")
    rc = launch_ranks(args)
    if rc is not None:
        sys.exit(rc)
    if args.probe_ranks:
        # one write per line: the ranks share the launcher's stdout, and a line written in one
        # call below the pipe's atomic size never interleaves with another rank's
        line = json.dumps({"rank": env_int("RANK", 0), "world": env_int("WORLD_SIZE", 1),
                           "local_rank": env_int("LOCAL_RANK", 0), "gpus": args.gpus}) + "\n"
        sys.stdout.flush()
        os.write(sys.stdout.fileno(), line.encode())
        return
    if args.impl == "reference":
        run_reference_arm(args)
    else:
        run_ours(args)


def _free_port() -> int:
    import socket

    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        return sk.getsockname()[1]


def launch_ranks(args):
    """One process per GPU.  Under torchrun (WORLD_SIZE set) the world must be --gpus and this
    process carries on (None); launched plainly with --gpus N > 1, bench.py starts N ranks of
    itself under torch.distributed.run on 127.0.0.1 and returns their exit status."""
    world = os.environ.get("WORLD_SIZE")
    if world is not None:
        if int(world) != args.gpus:
            print(f"bench.py: --gpus {args.gpus} but WORLD_SIZE={world}", file=sys.stderr)
            return 2
        return None
    if args.gpus == 1:
        return None
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
           f"--nproc-per-node={args.gpus}", "--master-addr=127.0.0.1",
           f"--master-port={_free_port()}", os.path.abspath(__file__), *sys.argv[1:]]
    return subprocess.run(cmd).returncode


if __name__ == "__main__":
    main()
