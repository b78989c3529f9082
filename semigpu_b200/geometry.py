"""Molecule input: XYZ files and the seeded synthetic workloads.

XYZ parsing follows the reference reader (``src/common/readxyzfile.cpp:27-133``): the first
token is the atom count, the second line is a comment, then one line per atom holding either
an element symbol or an atomic number (decided from the first data line, ``:106-125``) and
three Cartesian coordinates in Angstrom.  Only H, C, N and O have MNDO parameters in the
reference (``src/common/MNDO_parameters.cpp:47-122``); other elements are rejected here
instead of silently getting zero parameters.

The generators build the synthetic molecules the engine is measured on.  None of them reads
a dataset: every geometry comes from bond lengths, angles and a seeded Gaussian jitter.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

SYMBOLS = {1: "H", 6: "C", 7: "N", 8: "O"}
NUMBERS = {v: k for k, v in SYMBOLS.items()}
SUPPORTED = frozenset(SYMBOLS)


class UnsupportedElement(ValueError):
    pass


@dataclass
class Molecule:
    """Atomic numbers and Cartesian coordinates in Angstrom (natoms x 3)."""

    Z: np.ndarray
    xyz: np.ndarray
    name: str = ""
    meta: dict = field(default_factory=dict)

    def __post_init__(self):
        self.Z = np.ascontiguousarray(self.Z, dtype=np.int32)
        self.xyz = np.ascontiguousarray(self.xyz, dtype=np.float64).reshape(-1, 3)
        if self.Z.shape[0] != self.xyz.shape[0]:
            raise ValueError("Z and xyz disagree on the atom count")

    @property
    def natoms(self) -> int:
        return int(self.Z.shape[0])

    @property
    def nao(self) -> int:
        return int(sum(1 if z == 1 else 4 for z in self.Z))

    @property
    def nocc(self) -> int:
        return int(sum(int(z) if z < 2 else int(z) - 2 for z in self.Z)) // 2

    def check(self) -> "Molecule":
        bad = sorted({int(z) for z in self.Z} - SUPPORTED)
        if bad:
            raise UnsupportedElement(f"no MNDO parameters for Z={bad}; supported: H, C, N, O")
        return self


# ----------------------------------------------------------------------------------------
# XYZ I/O


def parse_xyz(text: str, name: str = "") -> Molecule:
    """One XYZ frame.  Raises ValueError on a malformed file."""
    lines = text.splitlines()
    if not lines:
        raise ValueError("empty XYZ")
    try:
        n = int(lines[0].split()[0])
    except (ValueError, IndexError) as exc:
        raise ValueError("XYZ: first line must hold the atom count") from exc
    if n <= 0:
        raise ValueError("XYZ: atom count must be positive")
    toks = " ".join(lines[2:]).split()
    if len(toks) < 4 * n:
        raise ValueError(f"XYZ: expected {n} atoms, found {len(toks) // 4}")
    Z = np.empty(n, np.int32)
    xyz = np.empty((n, 3))
    numeric = toks[0].lstrip("+-").isdigit()
    for i in range(n):
        s, x, y, z = toks[4 * i : 4 * i + 4]
        if numeric:
            Z[i] = int(s)
        else:
            if s not in NUMBERS:
                raise UnsupportedElement(f"XYZ: unsupported or invalid element symbol {s!r}")
            Z[i] = NUMBERS[s]
        xyz[i] = float(x), float(y), float(z)
    return Molecule(Z, xyz, name=name).check()


def read_xyz(path: str) -> Molecule:
    with open(path) as fh:
        return parse_xyz(fh.read(), name=path)


def read_xyz_frames(path: str) -> list[Molecule]:
    """Multi-frame XYZ (concatenated frames) for batch and serving input."""
    with open(path) as fh:
        lines = fh.read().splitlines()
    out, i = [], 0
    while i < len(lines):
        if not lines[i].strip():
            i += 1
            continue
        n = int(lines[i].split()[0])
        out.append(parse_xyz("\n".join(lines[i : i + n + 2]), name=f"{path}#{len(out)}"))
        i += n + 2
    return out


def format_xyz(mol: Molecule, comment: str = "") -> str:
    rows = [str(mol.natoms), comment or mol.name]
    for z, (x, y, w) in zip(mol.Z, mol.xyz):
        rows.append(f"{SYMBOLS.get(int(z), str(int(z)))} {float(x)!r} {float(y)!r} {float(w)!r}")
    return "\n".join(rows) + "\n"


def write_xyz(path: str, mols) -> None:
    if isinstance(mols, Molecule):
        mols = [mols]
    with open(path, "w") as fh:
        for m in mols:
            fh.write(format_xyz(m))


# ----------------------------------------------------------------------------------------
# Geometry builders


def _unit(v):
    return v / np.linalg.norm(v)


def _zigzag(n: int, bonds, angle_deg: float) -> np.ndarray:
    """Planar (z=0) zigzag chain of n backbone atoms; bond i joins atoms i and i+1."""
    half = math.radians(180.0 - angle_deg) / 2.0
    pts = [np.zeros(3)]
    for i in range(n - 1):
        a = half if i % 2 == 0 else -half
        pts.append(pts[-1] + bonds[i] * np.array([math.cos(a), math.sin(a), 0.0]))
    return np.array(pts)


def _virtual_neighbours(bb: np.ndarray, n: int, bond: float, angle_deg: float):
    """Backbone extended by one virtual atom on each end (continuing the zigzag)."""
    half = math.radians(180.0 - angle_deg) / 2.0
    if n == 1:
        return None, None
    a_first = -half  # bond (-1 -> 0) mirrors bond (0 -> 1), which has angle +half
    prev = bb[0] - bond * np.array([math.cos(a_first), math.sin(a_first), 0.0])
    a_last = half if (n - 1) % 2 == 0 else -half
    nxt = bb[-1] + bond * np.array([math.cos(a_last), math.sin(a_last), 0.0])
    return prev, nxt


def _tetra_h(c, n1, n2, r_ch, hch_deg=109.47):
    """Two H on a tetrahedral carbon c with backbone neighbours n1, n2 (out of plane)."""
    u1, u2 = _unit(n1 - c), _unit(n2 - c)
    bis = _unit(-(u1 + u2))
    nrm = _unit(np.cross(u1, u2))
    h = math.radians(hch_deg) / 2.0
    return [c + r_ch * (math.cos(h) * bis + s * math.sin(h) * nrm) for s in (1.0, -1.0)]


def alkane(n: int, rng: np.random.Generator | None = None, jitter: float = 0.01,
           r_cc: float = 1.54, r_ch: float = 1.09, angle: float = 109.47) -> Molecule:
    """All-trans CnH2n+2, planar zigzag backbone, tetrahedral CH2/CH3 groups."""
    if n < 1:
        raise ValueError("alkane needs n >= 1")
    if n == 1:
        t = r_ch / math.sqrt(3.0)
        xyz = [np.zeros(3)] + [t * np.array(v, float) for v in
                               ((1, 1, 1), (1, -1, -1), (-1, 1, -1), (-1, -1, 1))]
        Z = [6, 1, 1, 1, 1]
    else:
        bb = _zigzag(n, [r_cc] * (n - 1), angle)
        prev, nxt = _virtual_neighbours(bb, n, r_cc, angle)
        ext = np.vstack([prev, bb, nxt])
        hs = []
        for i in range(n):
            c, a, b = ext[i + 1], ext[i], ext[i + 2]
            hs += _tetra_h(c, a, b, r_ch)
            if i == 0:
                hs.append(c + r_ch * _unit(a - c))
            if i == n - 1:
                hs.append(c + r_ch * _unit(b - c))
        xyz = list(bb) + hs
        Z = [6] * n + [1] * len(hs)
    xyz = np.array(xyz)
    if rng is not None and jitter:
        xyz = xyz + rng.normal(0.0, jitter, xyz.shape)
    return Molecule(Z, xyz, name=f"C{n}H{2 * n + 2}", meta={"kind": "alkane", "n": n})


def polyene(n: int, rng: np.random.Generator | None = None, jitter: float = 0.01,
            r_double: float = 1.34, r_single: float = 1.46, r_ch: float = 1.08,
            angle: float = 120.0) -> Molecule:
    """All-trans CnHn+2 (n even), planar, alternating C=C / C-C, =CH2 ends."""
    if n < 2 or n % 2:
        raise ValueError("polyene needs an even n >= 2")
    bonds = [r_double if i % 2 == 0 else r_single for i in range(n - 1)]
    bb = _zigzag(n, bonds, angle)
    prev, nxt = _virtual_neighbours(bb, n, r_single, angle)
    ext = np.vstack([prev, bb, nxt])
    hs = []
    for i in range(n):
        c, a, b = ext[i + 1], ext[i], ext[i + 2]
        bis = _unit(-(_unit(a - c) + _unit(b - c)))
        if i == 0:
            hs.append(c + r_ch * _unit(a - c))
        hs.append(c + r_ch * bis)
        if i == n - 1:
            hs.append(c + r_ch * _unit(b - c))
    xyz = np.array(list(bb) + hs)
    if rng is not None and jitter:
        xyz = xyz + rng.normal(0.0, jitter, xyz.shape)
    return Molecule([6] * n + [1] * len(hs), xyz, name=f"C{n}H{n + 2}",
                    meta={"kind": "polyene", "n": n})


def aza_ring(n_positions=(0,), rng: np.random.Generator | None = None, jitter: float = 0.01,
             r_ring: float = 1.39, r_ch: float = 1.08) -> Molecule:
    """Planar regular hexagon (side = circumradius = r_ring) in z=0; N at the listed ring
    positions, C elsewhere, one H radially outward on every carbon."""
    npos = set(int(k) for k in n_positions)
    ring, hs, Z = [], [], []
    for k in range(6):
        a = math.radians(180.0 + 60.0 * k)
        d = np.array([math.cos(a), math.sin(a), 0.0])
        ring.append(r_ring * d)
        Z.append(7 if k in npos else 6)
        if k not in npos:
            hs.append((r_ring + r_ch) * d)
    xyz = np.array(ring + hs)
    if rng is not None and jitter:
        xyz = xyz + rng.normal(0.0, jitter, xyz.shape)
    nn = len(npos)
    return Molecule(Z + [1] * len(hs), xyz, name=f"C{6 - nn}H{6 - nn}N{nn}",
                    meta={"kind": "ring", "n_N": nn, "positions": sorted(npos)})


# ----------------------------------------------------------------------------------------
# The named workloads


def ring_c1() -> Molecule:
    """Single planar aza-aromatic ring: 1 N + 5 C at 1.39 A, 5 H at 1.08 A, no jitter.
    11 atoms, 29 AOs, 15 occupied orbitals."""
    m = aza_ring((0,), rng=None, jitter=0.0)
    m.name = "ring_C5H5N"
    return m


def alkane_c2(seed: int = 0) -> Molecule:
    """All-trans C100H202 with N(0, 0.01 A) jitter (302 atoms, 602 AOs, 301 occupied)."""
    return alkane(100, np.random.default_rng(seed))


def polyene_c4(seed: int = 0, n: int = 2000) -> Molecule:
    """All-trans C2000H2002 with jitter (4002 atoms, 10002 AOs, 5001 occupied)."""
    return polyene(n, np.random.default_rng(seed))


def batch_c3(count: int = 4096, seed: int = 0, alkane_max: int = 20) -> list[Molecule]:
    """The uneven batch: 50 % alkanes CnH2n+2 (n ~ U{1..alkane_max}), 30 % all-trans polyenes
    CnHn+2 (n even in 2..30), 20 % aza-aromatic rings with 0-3 N at random positions; every
    coordinate jittered by N(0, 0.01 A).  Kinds are drawn per molecule from the seed."""
    rng = np.random.default_rng(seed)
    kinds = rng.choice(3, size=count, p=[0.5, 0.3, 0.2])
    out = []
    for k in kinds:
        if k == 0:
            out.append(alkane(int(rng.integers(1, alkane_max + 1)), rng))
        elif k == 1:
            out.append(polyene(2 * int(rng.integers(1, 16)), rng))
        else:
            nn = int(rng.integers(0, 4))
            pos = rng.choice(6, size=nn, replace=False) if nn else ()
            out.append(aza_ring(tuple(int(p) for p in pos), rng))
    return out


def serving_c5(rate: float = 2000.0, duration_s: float = 60.0, seed: int = 0):
    """Open-loop Poisson arrivals (seeded): list of (arrival_time_s, Molecule) with the batch
    composition and alkane n extended to 1..150."""
    rng = np.random.default_rng(seed + 1)
    t, times = 0.0, []
    while True:
        t += rng.exponential(1.0 / rate)
        if t >= duration_s:
            break
        times.append(t)
    mols = batch_c3(len(times), seed=seed, alkane_max=150)
    return list(zip(times, mols))
