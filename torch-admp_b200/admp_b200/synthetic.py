"""Seeded synthetic systems with the shapes of the benchmark workloads.

The reference ships no dataset; these generators reproduce the workload
shapes named for this path (random point charges, rigid three-site waters
on a jittered lattice, two fcc(111) metal slabs with an electrolyte gap and
a Poisson stream of mixed requests).  All randomness comes from
``numpy.random.default_rng(seed)``.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

# per-element QEq parameters of the water-like system (eV, eV, Angstrom)
WATER_PARAMS = {"O": (8.7, 13.4, 0.9), "H": (4.5, 13.9, 0.6)}
OH_BOND = 0.96
HOH_ANGLE = math.radians(104.5)


def random_charges_system(n: int, box_len: float, seed: int, balanced: bool = False):
    """Uniform positions in a cubic box; charges U[-1,1] shifted to sum zero
    (or +-1 balanced when ``balanced``)."""
    rng = np.random.default_rng(seed)
    pos = rng.random((n, 3)) * box_len
    if balanced:
        q = np.ones(n)
        q[n // 2:] = -1.0
        rng.shuffle(q)
        if n % 2:
            q[-1] = 0.0
    else:
        q = rng.uniform(-1.0, 1.0, n)
        q -= q.mean()
    return pos, np.diag([box_len] * 3).astype(np.float64), q


def _haar_rotations(rng, n):
    a = rng.standard_normal((n, 3, 3))
    qm, r = np.linalg.qr(a)
    d = np.sign(np.diagonal(r, axis1=1, axis2=2))
    return qm * d[:, None, :]


def water_system(n_mol: int, box_len: float, seed: int, jitter: float = 0.1,
                 lattice: Optional[int] = None):
    """Three-site waters: O on a jittered n^3 lattice (spacing box_len/n),
    H-O-H of 0.96 Angstrom / 104.5 degrees with Haar-random orientation,
    wrapped into the cubic box.  Returns pos, box, chi, hardness, eta, elements."""
    rng = np.random.default_rng(seed)
    side = lattice or int(math.ceil(n_mol ** (1.0 / 3.0) - 1e-9))
    spacing = box_len / side
    g = np.stack(np.meshgrid(np.arange(side), np.arange(side), np.arange(side), indexing="ij"), -1)
    sites = (g.reshape(-1, 3)[:n_mol] + 0.5) * spacing
    o = sites + rng.normal(0.0, jitter, sites.shape)
    h1 = np.array([OH_BOND, 0.0, 0.0])
    h2 = np.array([OH_BOND * math.cos(HOH_ANGLE), OH_BOND * math.sin(HOH_ANGLE), 0.0])
    R = _haar_rotations(rng, n_mol)
    pos = np.empty((n_mol, 3, 3))
    pos[:, 0] = o
    pos[:, 1] = o + R @ h1
    pos[:, 2] = o + R @ h2
    pos = np.mod(pos.reshape(-1, 3), box_len)
    elem = np.array(["O", "H", "H"] * n_mol)
    chi = np.where(elem == "O", WATER_PARAMS["O"][0], WATER_PARAMS["H"][0]).astype(np.float64)
    hard = np.where(elem == "O", WATER_PARAMS["O"][1], WATER_PARAMS["H"][1]).astype(np.float64)
    eta = np.where(elem == "O", WATER_PARAMS["O"][2], WATER_PARAMS["H"][2]).astype(np.float64)
    return pos, np.diag([box_len] * 3).astype(np.float64), chi, hard, eta, elem


def water_frames(nframes: int, seed: int, n_mol: int = 1000, box_len: float = 31.0, jitter: float = 0.05):
    """Frames of one water system (``water_system(n_mol, box_len, seed)``)
    with every position jittered by N(0, jitter); frame f draws its jitter
    from ``default_rng(seed + f)``.  Returns pos [nf, N, 3], box [nf, 3, 3],
    chi, hardness, eta [N] (shared by the frames) and the element labels."""
    pos0, box, chi, hard, eta, elem = water_system(n_mol, box_len, seed)
    pos = np.stack([pos0 + np.random.default_rng(seed + f).normal(0.0, jitter, pos0.shape) for f in range(nframes)])
    return pos, np.repeat(box[None], nframes, 0), chi, hard, eta, elem


def electrode_system(seed: int, n_side: int = 24, n_layers: int = 2, a: float = 4.08,
                     gap: float = 40.0, n_ions: int = 3000, min_sep: float = 1.0,
                     slab_factor: float = 3.0):
    """Two fcc(111) slabs (n_layers x n_side^2 atoms each) around an
    electrolyte gap holding n_ions +-1 charges with a minimum separation.
    Returns pos, box (z already multiplied by slab_factor), charges,
    electrode index arrays (top, bottom)."""
    rng = np.random.default_rng(seed)
    nn = a / math.sqrt(2.0)
    dz = a / math.sqrt(3.0)
    lx = n_side * nn
    ly = n_side * nn * math.sqrt(3.0) / 2.0
    base = []
    for j in range(n_side):
        for i in range(n_side):
            base.append([(i + 0.5 * (j % 2)) * nn, j * nn * math.sqrt(3.0) / 2.0])
    base = np.array(base)
    offs = [np.array([0.0, 0.0]), np.array([nn / 2.0, nn * math.sqrt(3.0) / 6.0]),
            np.array([nn, nn * math.sqrt(3.0) / 3.0])]

    def slab(z0, sign):
        layers = []
        for l in range(n_layers):
            xy = np.mod(base + offs[l % 3], [lx, ly])
            z = np.full((xy.shape[0], 1), z0 + sign * l * dz)
            layers.append(np.hstack([xy, z]))
        return np.vstack(layers)

    z_bot_top = (n_layers - 1) * dz + 1.0
    bottom = slab(z_bot_top, -1.0)
    z_top_bot = z_bot_top + gap
    top = slab(z_top_bot, 1.0)
    ions = []
    lo, hi = z_bot_top + 2.0, z_top_bot - 2.0
    cell = 3.0
    grid = {}
    tries = 0
    while len(ions) < n_ions and tries < 200 * n_ions:
        tries += 1
        p = np.array([rng.random() * lx, rng.random() * ly, lo + rng.random() * (hi - lo)])
        key = tuple((p // cell).astype(int))
        ok = True
        for dx in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for dzc in (-1, 0, 1):
                    for qx in grid.get((key[0] + dx, key[1] + dy, key[2] + dzc), []):
                        d = p - qx
                        d[0] -= lx * round(d[0] / lx)
                        d[1] -= ly * round(d[1] / ly)
                        if d @ d < min_sep * min_sep:
                            ok = False
                            break
                    if not ok:
                        break
                if not ok:
                    break
            if not ok:
                break
        if ok:
            grid.setdefault(key, []).append(p)
            ions.append(p)
    ions = np.array(ions)
    q_ions = np.ones(len(ions))
    q_ions[len(ions) // 2:] = -1.0
    rng.shuffle(q_ions)
    pos = np.vstack([top, bottom, ions])
    lz = (z_top_bot + (n_layers - 1) * dz + 1.0) * slab_factor
    box = np.diag([lx, ly, lz])
    q = np.concatenate([np.zeros(len(top) + len(bottom)), q_ions])
    top_idx = np.arange(len(top))
    bot_idx = np.arange(len(top), len(top) + len(bottom))
    return pos, box, q, top_idx, bot_idx


@dataclass
class Request:
    """One serving request: a PME energy+forces or a QEq solve."""
    rid: int
    kind: str            # "pme" or "qeq"
    arrival: float       # seconds from stream start
    pos: np.ndarray
    box: np.ndarray
    charges: Optional[np.ndarray] = None
    chi: Optional[np.ndarray] = None
    hardness: Optional[np.ndarray] = None
    eta: Optional[np.ndarray] = None
    meta: dict = field(default_factory=dict)

    @property
    def natoms(self) -> int:
        return self.pos.shape[0]


def serving_stream(n_req: int, seed: int, rate: float, nmin: int = 200, nmax: int = 20000,
                   density: float = 0.1, pme_frac: float = 0.6) -> List[Request]:
    """Poisson arrivals at ``rate`` per second; atom counts log-uniform in
    [nmin, nmax]; cubic boxes at ``density`` atoms per cubic Angstrom;
    60% PME requests (balanced +-1 charges, even N) and 40% QEq waters."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, n_req))
    reqs = []
    for r in range(n_req):
        n = int(round(math.exp(rng.uniform(math.log(nmin), math.log(nmax)))))
        s = int(rng.integers(0, 2 ** 31 - 1))
        if rng.random() < pme_frac:
            n += n % 2
            L = (n / density) ** (1.0 / 3.0)
            pos, box, q = random_charges_system(n, L, s, balanced=True)
            reqs.append(Request(r, "pme", float(t[r]), pos, box, charges=q))
        else:
            nmol = max(1, n // 3)
            L = (3 * nmol / density) ** (1.0 / 3.0)
            pos, box, chi, hard, eta, _ = water_system(nmol, L, s)
            reqs.append(Request(r, "qeq", float(t[r]), pos, box, chi=chi, hardness=hard, eta=eta))
    return reqs
