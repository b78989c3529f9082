"""Generate the golden fixtures from the UNMODIFIED reference build (oracle/_ref/ref_driver).

Run in a container that has the reference tree (it reads the reference's XYZ fixtures and
runs the reference); the fixtures it writes travel with the repository so the GPU-side tests
never need the reference.

    python tests/golden/make_golden.py --reference-src <reference>/src
                                      # every fixture and synthetic case but C100H202
    python tests/golden/make_golden.py --c2   # C100H202 alone (serial reference: ~2 h)

The reference source tree is given by --reference-src or the SEMIGPU_REF_SRC environment
variable (the directory holding common/, App/ and Geometries4Test/).

Outputs (next to this script):
  reference_cases.json   per case: Z, xyz (Angstrom, as parsed by the reference reader), tol,
                         per-step energies, n_iter, converged, E_el / E_cc / E_tot, nao,
                         nocc, and checksums of the final H, F, P (sum, sum of squares);
  reference_matrices.npz element-level arrays for the small cases: integral blocks in the
                         reference's ragged [A][B<=A] order, Hcore, the guess P0 and its
                         Fock F0, the final P and F (packed lower triangles), eigenvalues.
  reference_c100h202.npz (--c2) the all-trans C100H202 workload (302 atoms, 602 AOs, seed 0)
                         at 1e-6 eV: geometry, per-step energies, step count, E_el / E_cc /
                         E_tot, the final F and P (packed lower triangles) and eigenvalues.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import glob
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import oracle  # noqa: E402
from semigpu_b200 import geometry as geo  # noqa: E402

MATRIX_NAO_MAX = 40
FIXTURE_DIR = None  # <reference>/src/Geometries4Test, set by main()


def run_case(name, Z, xyz, tol, matrices, timeout=None):
    t = time.time()
    r = oracle.run_reference(Z, xyz, tol=tol, matrices=True, timeout=timeout)
    r["wall_s"] = time.time() - t
    return name, tol, matrices, r


def summarize(name, tol, r):
    out = {k: r[k] for k in ("natoms", "nao", "nocc", "Z", "xyz", "energies", "n_iter",
                             "converged", "E_el", "E_cc", "E_tot", "lapack_info")}
    out["tol"] = tol
    for key in ("H", "F", "P"):
        a = np.asarray(r[key])
        out[f"{key}_sum"] = float(a.sum())
        out[f"{key}_sumsq"] = float((a * a).sum())
    out["blocks_sum"] = float(np.sum(r["blocks"]))
    out["blocks_sumsq"] = float(np.sum(np.square(r["blocks"])))
    out["t_fock_s"], out["t_scf_s"], out["wall_s"] = r["t_fock_s"], r["t_scf_s"], r["wall_s"]
    return out


def cases():
    out = []
    for path in sorted(glob.glob(os.path.join(FIXTURE_DIR, "*.xyz"))):
        base = os.path.basename(path)[:-4]
        if base.startswith("filetest_"):
            continue
        m = geo.read_xyz(path)
        tols = (5e-3,) if m.nao > 160 else (5e-3, 1e-6)
        for tol in tols:
            out.append((f"fixture/{base}", m.Z, m.xyz, tol, m.nao <= MATRIX_NAO_MAX and tol == 1e-6))
    c1 = geo.ring_c1()
    out.append(("config/ring_C5H5N", c1.Z, c1.xyz, 1e-6, True))
    for i, m in enumerate(geo.batch_c3(32, seed=0)):
        out.append((f"batch/{i:02d}_{m.name}", m.Z, m.xyz, 1e-6, m.nao <= MATRIX_NAO_MAX))
    rng = np.random.default_rng(7)
    for name, m in (("alkane/C20H42", geo.alkane(20, rng)), ("polyene/C10H12", geo.polyene(10, rng)),
                    ("polyene/C30H32", geo.polyene(30, rng)),
                    ("ring/C3H3N3", geo.aza_ring((0, 2, 4), rng))):
        out.append((name, m.Z, m.xyz, 1e-6, m.nao <= MATRIX_NAO_MAX))
    return out


def c2_golden():
    """C100H202 (the single-large-molecule workload) through the reference build, once."""
    m = geo.alkane_c2(0)
    t = time.time()
    r = oracle.run_reference(m.Z, m.xyz, tol=1e-6, matrices=True)
    wall = time.time() - t
    print(f"C100H202 N={r['nao']} it={r['n_iter']} E_tot={r['E_tot']:.10f} {wall:.0f}s", flush=True)
    np.savez_compressed(
        os.path.join(HERE, "reference_c100h202.npz"),
        Z=np.asarray(r["Z"], np.int32), xyz=np.asarray(r["xyz"], np.float64).reshape(-1, 3),
        energies=np.asarray(r["energies"]), n_iter=np.int32(r["n_iter"]),
        converged=np.bool_(r["converged"]), E_el=np.float64(r["E_el"]),
        E_cc=np.float64(r["E_cc"]), E_tot=np.float64(r["E_tot"]),
        F=np.asarray(r["F"], np.float64), P=np.asarray(r["P"], np.float64),
        eig=np.asarray(r["eig"], np.float64), wall_s=np.float64(wall),
        t_fock_s=np.float64(r["t_fock_s"]), t_eig_s=np.float64(r["t_eig_s"]))


def readers():
    """The reference reader's fixtures: raw text plus what the reference parsed from it."""
    import subprocess

    res = {}
    for path in sorted(glob.glob(os.path.join(FIXTURE_DIR, "*.xyz"))):
        with open(path) as fh:
            text = fh.read()
        out = subprocess.run([oracle.REF_DRIVER, path, "--max-iter", "0", "--no-matrices"],
                             capture_output=True, text=True, check=True)
        r = json.loads(out.stdout)
        res[os.path.basename(path)] = {"text": text, "Z": r["Z"], "xyz": r["xyz"]}
    return res


CLI_FIXTURES = ("04_pyridine", "03_formaldehyde", "02_benzene", "01_h2")


def cli_outputs():
    """The unmodified reference CLI's printout (oracle/_ref/semiGPU) on a few fixtures."""
    import subprocess

    out = {}
    for base in CLI_FIXTURES:
        path = os.path.join(FIXTURE_DIR, base + ".xyz")
        r = subprocess.run([oracle.REF_CLI, path], capture_output=True, text=True, check=True,
                           env=dict(os.environ, OPENBLAS_NUM_THREADS="1"))
        out[base] = {"xyz": open(path).read(), "stdout": r.stdout}
    with open(os.path.join(HERE, "reference_cli.json"), "w") as fh:
        json.dump(out, fh, indent=0)


def main():
    global FIXTURE_DIR
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference-src", default=os.environ.get("SEMIGPU_REF_SRC"),
                    help="the reference's src/ directory (or set SEMIGPU_REF_SRC)")
    ap.add_argument("--c2", action="store_true", help="only the C100H202 golden")
    ap.add_argument("--cli-only", action="store_true")
    ap.add_argument("--jobs", type=int, default=os.cpu_count())
    args = ap.parse_args()
    if not args.reference_src:
        ap.error("the reference source tree is required: --reference-src or SEMIGPU_REF_SRC")
    FIXTURE_DIR = os.path.join(args.reference_src, "Geometries4Test")
    os.environ["SEMIGPU_REF_SRC"] = args.reference_src
    oracle.build()
    if args.c2:
        c2_golden()
        return
    cli_outputs()
    if args.cli_only:
        return
    todo = cases()
    todo.sort(key=lambda c: -len(c[1]))
    summaries, mats = {}, {}
    with cf.ProcessPoolExecutor(args.jobs) as ex:
        futs = [ex.submit(run_case, *c) for c in todo]
        for f in cf.as_completed(futs):
            name, tol, matrices, r = f.result()
            key = f"{name}@{tol:g}"
            summaries[key] = summarize(name, tol, r)
            print(f"{key:48s} N={r['nao']:4d} it={r['n_iter']:3d} E_tot={r['E_tot']:.10f} "
                  f"{r['wall_s']:.1f}s", flush=True)
            if matrices:
                for k in ("blocks", "H", "P0", "F0", "P", "F", "eig"):
                    mats[f"{key}/{k}"] = np.asarray(r[k], dtype=np.float64)
    with open(os.path.join(HERE, "reference_cases.json"), "w") as fh:
        json.dump({"generator": "tests/golden/make_golden.py",
                   "reference": "LuisAlfredoNu/semiGPU src/common, serial g++ -O2 build",
                   "cases": dict(sorted(summaries.items())),
                   "xyz_reader_fixtures": readers()}, fh, indent=0)
    np.savez_compressed(os.path.join(HERE, "reference_matrices.npz"), **mats)


if __name__ == "__main__":
    main()
