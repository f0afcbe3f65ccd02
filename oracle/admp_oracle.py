"""CPU FP64 oracle for the torch-admp electrostatics hot path.

TEST INFRASTRUCTURE ONLY.  This module is a NumPy restatement of the
reference algorithm (ChiahsinChu/torch-admp 1.1.5) and is imported by
``tests/``, by ``__graft_entry__.smoke()`` and by the ``cpu_baseline`` /
``--impl reference`` legs of ``bench.py`` -- always as the checker or as
the timed CPU baseline, never as part of the product path.  The product
(``admp_b200``) never imports it and fails loudly without its CUDA library.

Every function cites the reference file:line it restates.  Forces and
other gradients, which the reference obtains with ``torch.autograd``, are
written here analytically; the golden fixtures in ``tests/golden`` (made by
running the reference itself) pin both the values and the gradients.
"""
from __future__ import annotations

import math
from typing import Dict, Optional, Tuple

import numpy as np
from scipy import constants as _C
from scipy.special import erfc as _erfc

# utils.py:273-278  dielectric = 1/(4 pi eps0) in eV*Angstrom/e^2
EPSILON = _C.epsilon_0 / _C.elementary_charge * _C.angstrom
DIELECTRIC = 1.0 / (4.0 * np.pi * EPSILON)
SQRT_PI = np.sqrt(np.pi)
PME_ORDER = 6


# --------------------------------------------------------------------------
# geometry
# --------------------------------------------------------------------------
def pbc_shift(dr: np.ndarray, box: np.ndarray) -> np.ndarray:
    """Minimum image of row vectors ``dr`` -- spatial.py:15-36."""
    binv = np.linalg.inv(box)
    f = dr @ binv
    f = f - np.floor(f + 0.5)
    return f @ box


def pair_buffer_scales(pairs: np.ndarray) -> np.ndarray:
    """1 if i < j else 0 -- nblist.py:492-515, utils.py:21-41."""
    return (pairs[:, 0] - pairs[:, 1] < 0).astype(np.int64)


def pairs_ds(pos, pairs, box=None):
    """Pair distances -- nblist.py:517-551 (ds = |pbc_shift(r_i - r_j)|)."""
    ri = pos[pairs[:, 0]]
    rj = pos[pairs[:, 1]]
    if box is None:
        dr = rj - ri
    else:
        dr = pbc_shift(ri - rj, box)
    return np.linalg.norm(dr, axis=1)


def check_cutoff(box: np.ndarray, cutoff: float) -> None:
    """rc <= half the minimum box height -- nblist.py:620-660."""
    a1, a2, a3 = box
    normals = np.stack([np.cross(a2, a3), np.cross(a3, a1), np.cross(a1, a2)])
    unit = normals / np.linalg.norm(normals, axis=1, keepdims=True)
    heights = np.abs(np.einsum("ij,ij->i", box, unit))
    mh = heights.min() / 2
    if not cutoff <= mh:
        raise AssertionError(
            f"Cutoff {cutoff} is larger than half the minimum height {mh} of the box. "
            "This may lead to unphysical results."
        )


def nblist_pbc(pos: np.ndarray, box: np.ndarray, rc: float) -> np.ndarray:
    """Full pair list with 0.01 < r < rc under PBC -- nblist.py:335-445.

    The reference pads images and bins them into rc-sized cells; since it
    asserts rc <= half the minimum box height, every pair has at most one
    image inside rc, so the pair SET equals the minimum-image set computed
    here.  Pairs are returned sorted by (i, j).
    """
    check_cutoff(box, rc)
    n = pos.shape[0]
    binv = np.linalg.inv(box)
    f = pos @ binv
    out = []
    blk = max(1, 4_000_000 // max(n, 1))
    for s in range(0, n, blk):
        df = f[None, :, :] - f[s:s + blk, None, :]
        df -= np.floor(df + 0.5)
        d = np.linalg.norm(df @ box, axis=-1)
        ii, jj = np.nonzero((d < rc) & (d > 0.01))
        out.append(np.stack([ii + s, jj], axis=1))
    pairs = np.concatenate(out, axis=0) if out else np.zeros((0, 2), np.int64)
    return pairs.astype(np.int64)


def nblist_pbc_cells(pos: np.ndarray, box: np.ndarray, rc: float) -> np.ndarray:
    """Same pair set as ``nblist_pbc`` via a cell list (the reference's own
    strategy, nblist.py:382-445): atoms binned into cells at least rc high,
    candidate pairs from the 27 neighbouring cells, minimum-image test.
    Vectorised per cell pair; used where the O(N^2) form is too slow."""
    check_cutoff(box, rc)
    n = pos.shape[0]
    binv = np.linalg.inv(box)
    f = pos @ binv
    f -= np.floor(f)
    V = abs(np.linalg.det(box))
    h = np.array([V / np.linalg.norm(np.cross(box[(d + 1) % 3], box[(d + 2) % 3])) for d in range(3)])
    nc = np.maximum(np.floor(h / rc).astype(int), 1)
    c = np.minimum((f * nc).astype(int), nc - 1)
    cid = (c[:, 0] * nc[1] + c[:, 1]) * nc[2] + c[:, 2]
    order = np.argsort(cid, kind="stable")
    counts = np.bincount(cid, minlength=int(np.prod(nc)))
    start = np.concatenate([[0], np.cumsum(counts)])
    offs = []
    for d in range(3):
        offs.append([0] if nc[d] == 1 else ([0, 1] if nc[d] == 2 else [-1, 0, 1]))
    out = []
    for cx in range(nc[0]):
        for cy in range(nc[1]):
            for cz in range(nc[2]):
                a = order[start[(cx * nc[1] + cy) * nc[2] + cz]:start[(cx * nc[1] + cy) * nc[2] + cz + 1]]
                if a.size == 0:
                    continue
                nb = []
                for ox in offs[0]:
                    for oy in offs[1]:
                        for oz in offs[2]:
                            k = (((cx + ox) % nc[0]) * nc[1] + (cy + oy) % nc[1]) * nc[2] + (cz + oz) % nc[2]
                            nb.append(order[start[k]:start[k + 1]])
                b = np.concatenate(nb)
                df = f[b][None, :, :] - f[a][:, None, :]
                df -= np.floor(df + 0.5)
                d = np.linalg.norm(df @ box, axis=-1)
                ii, jj = np.nonzero((d < rc) & (d > 0.01))
                out.append(np.stack([a[ii], b[jj]], axis=1))
    pairs = np.concatenate(out, axis=0) if out else np.zeros((0, 2), np.int64)
    pairs = pairs[np.lexsort((pairs[:, 1], pairs[:, 0]))]
    return pairs.astype(np.int64)


def nblist_obc(pos: np.ndarray, rc: float) -> np.ndarray:
    """Open-boundary full list, r < rc, i != j -- nblist.py:472-490."""
    d = np.linalg.norm(pos[:, None, :] - pos[None, :, :], axis=-1)
    m = d < rc
    np.fill_diagonal(m, False)
    return np.argwhere(m).astype(np.int64)


def image_nblist(pos: np.ndarray, box: Optional[np.ndarray], rc: float, nnei: int):
    """dp_nblist's pair set for any cutoff -- nblist.py:33-93 with
    make_extended_pairs / make_local_pairs / make_ds (nblist.py:140-240).

    The per-atom list comes from deepmd-kit's (pt backend, not vendored with
    the reference and not pinned by it) extend_input_and_build_neighbor_list,
    whose published behaviour is restated here: coordinates are wrapped into
    the cell, ghost images are made within ceil(rc / h_d) cells along each
    axis d (h_d the cell height), each local atom's list holds every image
    (the atom itself excluded) with r <= rc, sorted by distance and cut to
    its first `nnei` entries (`sel`).  make_local_pairs then keeps the i < j
    entries (scale 1) followed by the self images i == j (scale 1/2), and
    make_ds takes |x_j' - x_i| from the extended coordinates.

    Returns (pairs [P,2] int64, shifts [P,3] int64 with
    ds = |r_j - r_i + shift.box| for the caller's unwrapped positions,
    ds [P], buffer_scales [P]).  Within each block the order here is (i, j,
    image); the reference orders by distance, so tests compare sorted sets.
    """
    pos = np.asarray(pos, np.float64).reshape(-1, 3)
    n = pos.shape[0]
    if box is None:
        bx = np.eye(3)
        f = pos.copy()
        k = np.zeros((n, 3), np.int64)
        m = np.zeros(3, np.int64)
    else:
        bx = np.asarray(box, np.float64).reshape(3, 3)
        x = pos @ np.linalg.inv(bx)
        k = np.floor(x).astype(np.int64)
        f = x - k
        V = abs(np.linalg.det(bx))
        h = np.array([V / np.linalg.norm(np.cross(bx[(d + 1) % 3], bx[(d + 2) % 3])) for d in range(3)])
        m = np.ceil(rc / h).astype(np.int64)
    imgs = np.stack(np.meshgrid(*[np.arange(-m[d], m[d] + 1) for d in range(3)], indexing="ij"), -1).reshape(-1, 3)
    rows_ij, rows_ii = [], []
    for i in range(n):
        df = f[None, :, :] - f[i][None, None, :] + imgs[:, None, :]          # [nimg, n, 3]
        r = np.linalg.norm(df @ bx, axis=-1)
        r[np.all(imgs == 0, axis=1), i] = np.inf
        ii, jj = np.nonzero(r <= rc)
        sel = np.argsort(r[ii, jj], kind="stable")
        if nnei >= 0 and sel.size > nnei:
            rth = r[ii, jj][sel[nnei - 1]] if nnei > 0 else -1.0
            keep = r[ii, jj] <= rth
            ii, jj = ii[keep], jj[keep]
        shift = imgs[ii] + k[i][None, :] - k[jj]
        for a, j, s in zip(ii, jj, shift):
            if j > i:
                rows_ij.append((i, j, *s, r[a, j]))
            elif j == i:
                rows_ii.append((i, j, *s, r[a, j]))
    rows_ij.sort(key=lambda t: t[:5])
    rows_ii.sort(key=lambda t: t[:5])
    rows = rows_ij + rows_ii
    if not rows:
        return (np.zeros((0, 2), np.int64), np.zeros((0, 3), np.int64), np.zeros(0), np.zeros(0))
    arr = np.array([t[:5] for t in rows], np.int64)
    ds = np.array([t[5] for t in rows])
    bs = np.concatenate([np.ones(len(rows_ij)), np.full(len(rows_ii), 0.5)])
    return arr[:, :2], arr[:, 2:5], ds, bs


# --------------------------------------------------------------------------
# Ewald parameters
# --------------------------------------------------------------------------
def ewald_kappa(rcut: float, ethresh: float) -> float:
    """pme.py:113-115."""
    return math.sqrt(-math.log(2 * ethresh)) / rcut


def auto_kmesh(box: np.ndarray, kappa: float, ethresh: float, spacing=None) -> np.ndarray:
    """pme.py:380-392 -- explicit spacing or ceil(2 kappa L / (3 ethresh^0.2))."""
    diag = np.diagonal(box)
    if spacing is not None:
        return np.ceil(diag / np.asarray(spacing, dtype=np.float64)).astype(np.int64)
    return np.ceil(2 * kappa * diag / (3.0 * ethresh ** (1.0 / 5.0))).astype(np.int64)


# --------------------------------------------------------------------------
# pair terms
# --------------------------------------------------------------------------
def _safe_inv(x, thr):
    """utils.py:66-82."""
    out = np.zeros_like(x)
    m = np.abs(x) > thr
    out[m] = 1.0 / x[m]
    return out, m


def pme_real(q, pairs, ds, bs, kappa):
    """Real-space Ewald sum -- pme.py:312-349.  Returns E, dE/dds, dE/dq."""
    qi, qj = q[pairs[:, 0]], q[pairs[:, 1]]
    inv, m = _safe_inv(ds, 1e-4)
    er = _erfc(kappa * ds)
    e = er * qi * qj * inv * bs * DIELECTRIC
    ddr = np.where(m, (-2 * kappa / SQRT_PI * np.exp(-(kappa * ds) ** 2) * inv - er * inv * inv), 0.0)
    dE_dds = ddr * qi * qj * bs * DIELECTRIC
    c = er * inv * bs * DIELECTRIC
    n = q.shape[0]
    dq = np.bincount(pairs[:, 0], c * qj, n) + np.bincount(pairs[:, 1], c * qi, n)
    return e.sum(), dE_dds, dq


def coulomb_obc(q, pairs, ds, bs):
    """Plain Coulomb, open boundaries -- pme.py:529-561 (safe_inverse 1e-8)."""
    qi, qj = q[pairs[:, 0]], q[pairs[:, 1]]
    inv, m = _safe_inv(ds, 1e-8)
    e = qi * qj * DIELECTRIC * inv * bs
    dE_dds = np.where(m, -qi * qj * DIELECTRIC * inv * inv * bs, 0.0)
    c = DIELECTRIC * inv * bs
    dq = np.zeros_like(q)
    np.add.at(dq, pairs[:, 0], c * qj)
    np.add.at(dq, pairs[:, 1], c * qi)
    return e.sum(), dE_dds, dq


def damping(q, eta, pairs, ds, bs):
    """Gaussian damping -- qeq.py:60-129.  Returns E, dE/dds, dE/dq, dE/deta."""
    i, j = pairs[:, 0], pairs[:, 1]
    ei, ej = eta[i], eta[j]
    eij = np.sqrt((ei ** 2 + ej ** 2) / 2)
    zero = eij == 0
    eij_s = np.where(zero, 1e-10, eij)
    x = ds / (2 * eij_s)
    pre = -_erfc(x)
    qi, qj = q[i], q[j]
    inv, m = _safe_inv(ds, 1e-4)
    e_pair = (pre * qi * qj * inv * bs).sum()
    einv, em = _safe_inv(eta, 1e-4)
    pre_self = einv / (2 * SQRT_PI)
    e_self = (pre_self * q * q).sum()
    E = (e_pair + e_self) * DIELECTRIC
    g = np.exp(-x * x) * 2 / SQRT_PI
    # d/dds [-erfc(x) inv] = g/(2 eij) * inv + erfc(x) inv^2
    dE_dds = np.where(m, (g / (2 * eij_s) * inv + _erfc(x) * inv * inv), 0.0) * qi * qj * bs * DIELECTRIC
    c = pre * inv * bs * DIELECTRIC
    n = q.shape[0]
    dq = np.bincount(i, c * qj, n) + np.bincount(j, c * qi, n)
    dq += 2 * pre_self * q * DIELECTRIC
    # d/deij [-erfc(ds/(2 eij))] = -g * ds / (2 eij^2)
    dpair_deij = np.where(zero, 0.0, -g * ds / (2 * eij_s ** 2) * qi * qj * inv * bs * DIELECTRIC)
    deij_dei = np.where(zero, 0.0, ei / (2 * eij_s))
    deij_dej = np.where(zero, 0.0, ej / (2 * eij_s))
    deta = np.bincount(i, dpair_deij * deij_dei, n) + np.bincount(j, dpair_deij * deij_dej, n)
    deta += np.where(em, -q * q / (2 * SQRT_PI) * einv * einv, 0.0) * DIELECTRIC
    return E, dE_dds, dq, deta


def site(q, chi, hardness):
    """Site energy chi q + hardness q^2 -- qeq.py:159-209."""
    return float((chi * q + hardness * q * q).sum()), chi + 2 * hardness * q


# --------------------------------------------------------------------------
# reciprocal space
# --------------------------------------------------------------------------
def bspline(u: np.ndarray) -> np.ndarray:
    """Cardinal B-spline M6 as piecewise quintics -- recip.py:102-143."""
    out = np.zeros_like(u)
    c = [
        (u >= 0.0) & (u < 1.0), (u >= 1.0) & (u < 2.0), (u >= 2.0) & (u < 3.0),
        (u >= 3.0) & (u < 4.0), (u >= 4.0) & (u < 5.0), (u >= 5.0) & (u < 6.0),
    ]
    out[c[0]] = (u ** 5 / 120)[c[0]]
    out[c[1]] = (u ** 5 / 120 - (u - 1) ** 5 / 20)[c[1]]
    out[c[2]] = (u ** 5 / 120 + (u - 2) ** 5 / 8 - (u - 1) ** 5 / 20)[c[2]]
    out[c[3]] = (u ** 5 / 120 - (u - 3) ** 5 / 6 + (u - 2) ** 5 / 8 - (u - 1) ** 5 / 20)[c[3]]
    out[c[4]] = (u ** 5 / 24 - u ** 4 + 19 * u ** 3 / 2 - 89 * u ** 2 / 2 + 409 * u / 4 - 1829 / 20)[c[4]]
    out[c[5]] = (-(u ** 5) / 120 + u ** 4 / 4 - 3 * u ** 3 + 18 * u ** 2 - 54 * u + 324 / 5)[c[5]]
    return out


def bspline_deriv(u: np.ndarray) -> np.ndarray:
    """d M6 / du of the same pieces (what autograd differentiates in recip.py:102-143)."""
    out = np.zeros_like(u)
    c = [
        (u >= 0.0) & (u < 1.0), (u >= 1.0) & (u < 2.0), (u >= 2.0) & (u < 3.0),
        (u >= 3.0) & (u < 4.0), (u >= 4.0) & (u < 5.0), (u >= 5.0) & (u < 6.0),
    ]
    out[c[0]] = (u ** 4 / 24)[c[0]]
    out[c[1]] = (u ** 4 / 24 - (u - 1) ** 4 / 4)[c[1]]
    out[c[2]] = (u ** 4 / 24 + 5 * (u - 2) ** 4 / 8 - (u - 1) ** 4 / 4)[c[2]]
    out[c[3]] = (u ** 4 / 24 - 5 * (u - 3) ** 4 / 6 + 5 * (u - 2) ** 4 / 8 - (u - 1) ** 4 / 4)[c[3]]
    out[c[4]] = (5 * u ** 4 / 24 - 4 * u ** 3 + 57 * u ** 2 / 2 - 89 * u + 409 / 4)[c[4]]
    out[c[5]] = (-(u ** 4) / 24 + u ** 3 - 9 * u ** 2 + 36 * u - 54)[c[5]]
    return out


def _stencil(pos, box_inv, kmesh):
    """u_reference + stencil weights -- recip.py:37-64, 67-99, 174-213."""
    K = np.asarray(kmesh, dtype=np.int64)
    x = (pos @ box_inv) * K[None, :]          # R_in_m_basis
    m0 = np.ceil(x).astype(np.int64)
    u0 = (m0 - x) + PME_ORDER / 2
    s = np.arange(-PME_ORDER // 2, PME_ORDER // 2)  # -3..2
    u = u0[:, :, None] + s[None, None, :]          # N,3,6
    w = bspline(u)
    dw = bspline_deriv(u)
    idx = np.mod(m0[:, :, None] + s[None, None, :], K[None, :, None])  # N,3,6
    flat = (idx[:, 0, :, None, None] * K[1] + idx[:, 1, None, :, None]) * K[2] + idx[:, 2, None, None, :]
    return x, w, dw, flat.reshape(pos.shape[0], -1)


def spread_charges(pos, box_inv, q, kmesh):
    """Charge spreading onto the mesh -- recip.py:216-252."""
    K = np.asarray(kmesh, dtype=np.int64)
    _, w, _, flat = _stencil(pos, box_inv, K)
    theta = (w[:, 0, :, None, None] * w[:, 1, None, :, None] * w[:, 2, None, None, :]).reshape(pos.shape[0], -1)
    Q = np.bincount(flat.ravel(), weights=(q[:, None] * theta).ravel(), minlength=int(np.prod(K)))
    return Q.reshape(tuple(K))


def kpts_integer(K: int) -> np.ndarray:
    """FFT-ordered integer k -- recip.py:255-285 (roll of arange)."""
    a = np.arange(-(K - 1) // 2, (K + 1) // 2)
    return np.roll(a, -(K - 1) // 2)


def theta_k_1d(K: int) -> np.ndarray:
    """sum_{m=-2..2} M6(m+3) cos(2 pi m k / K) -- pme.py:412-432 (per dimension)."""
    k = kpts_integer(K).astype(np.float64)
    m = np.arange(-2, 3, dtype=np.float64)
    return (bspline(m + 3.0)[:, None] * np.cos(2 * np.pi * m[:, None] * k[None, :] / K)).sum(0)


def _green(box, kappa, kmesh):
    K = [int(k) for k in kmesh]
    binv = np.linalg.inv(box)
    V = np.linalg.det(box)
    n0, n1, n2 = (kpts_integer(k).astype(np.float64) for k in K)
    n = np.stack(np.meshgrid(n0, n1, n2, indexing="ij"), axis=-1)   # K0,K1,K2,3
    kv = 2 * np.pi * (n @ binv)                                     # setup_kpts recip.py:288-308
    ksq = (kv ** 2).sum(-1)
    t0, t1, t2 = (theta_k_1d(k) for k in K)
    theta = t0[:, None, None] * t1[None, :, None] * t2[None, None, :]
    with np.errstate(divide="ignore", invalid="ignore"):
        coeff = 2 * np.pi / V / ksq * np.exp(-ksq / 4 / kappa ** 2)   # _coeff_k_1 pme.py:661-683
    coeff[0, 0, 0] = 0.0
    G = DIELECTRIC * coeff / theta ** 2
    return G, n, kv, ksq, V, binv


def pme_recip(pos, box, q, kappa, kmesh, want_grad=True):
    """Reciprocal-space PME energy -- pme.py:351-446 (one frame).

    Returns dict with E and (analytic) dE/dpos, dE/dq, dE/dbox.
    """
    K = np.asarray(kmesh, dtype=np.int64)
    G, n, kv, ksq, V, binv = _green(box, kappa, K)
    x, w, dw, flat = _stencil(pos, binv, K)
    theta = (w[:, 0, :, None, None] * w[:, 1, None, :, None] * w[:, 2, None, None, :]).reshape(pos.shape[0], -1)
    Q = np.bincount(flat.ravel(), weights=(q[:, None] * theta).ravel(), minlength=int(np.prod(K))).reshape(tuple(K))
    S = np.fft.fftn(Q)
    S2 = S.real ** 2 + S.imag ** 2
    E = float((G * S2).sum())
    out = {"E": E}
    if not want_grad:
        return out
    phi = (2.0 * np.prod(K)) * np.fft.ifftn(G * S).real
    phif = phi.ravel()[flat]                                  # N,216
    out["dq"] = (phif * theta).sum(1)
    # dtheta/du_d
    d0 = (dw[:, 0, :, None, None] * w[:, 1, None, :, None] * w[:, 2, None, None, :]).reshape(pos.shape[0], -1)
    d1 = (w[:, 0, :, None, None] * dw[:, 1, None, :, None] * w[:, 2, None, None, :]).reshape(pos.shape[0], -1)
    d2 = (w[:, 0, :, None, None] * w[:, 1, None, :, None] * dw[:, 2, None, None, :]).reshape(pos.shape[0], -1)
    Gu = np.stack([(phif * d0).sum(1), (phif * d1).sum(1), (phif * d2).sum(1)], axis=1) * q[:, None]  # dE/du
    # u = m0 - x + 3, x = K * (r @ binv)  ->  dE/dx = -dE/du
    dEdx = -Gu
    out["dpos"] = (dEdx * K[None, :]) @ binv.T
    # box: via binv in x, via V and k in G
    dE_dbinv = pos.T @ (dEdx * K[None, :])                         # [a][d]
    with np.errstate(divide="ignore", invalid="ignore"):
        fac = -(1.0 / (4 * kappa ** 2) + 1.0 / ksq)
    fac[0, 0, 0] = 0.0
    Ek = G * S2
    c = Ek * fac * 2                                                 # dE/d(k_b) = c * k_b
    dE_dbinv += 2 * np.pi * ((n * c[..., None]).reshape(-1, 3).T @ kv.reshape(-1, 3))
    dE_dV = -E / V
    dbox = -binv.T @ dE_dbinv @ binv.T + dE_dV * V * binv.T
    out["dbox"] = dbox
    out["phi"] = phi
    return out


def pme_self(q, kappa):
    """pme.py:448-461."""
    return float(-(kappa / SQRT_PI * q * q).sum() * DIELECTRIC), -2 * kappa / SQRT_PI * q * DIELECTRIC


def pme_non_neutral(q, box, kappa):
    """pme.py:463-493.  Returns E, dE/dq, dE/dbox."""
    V = np.linalg.det(box)
    Q = q.sum()
    coeff = -np.pi / (2 * V * kappa ** 2) * DIELECTRIC
    E = coeff * Q * Q
    dq = np.full_like(q, 2 * coeff * Q)
    dbox = (-E / V) * V * np.linalg.inv(box).T
    return float(E), dq, dbox


def slab_corr(q, pos, box, axis=2):
    """pme.py:495-527.  Returns E, dE/dq, dE/dpos, dE/dbox."""
    V = np.linalg.det(box)
    pre = 2 * np.pi / V * DIELECTRIC
    z = pos[:, axis]
    Mz = (q * z).sum()
    Q = q.sum()
    Lz = np.linalg.norm(box[axis])
    Sz2 = (q * z * z).sum()
    E = pre * (Mz ** 2 - Q * Sz2 - Q * Q * Lz * Lz / 12)
    dq = pre * (2 * Mz * z - Sz2 - Q * z * z - 2 * Q * Lz * Lz / 12)
    dpos = np.zeros_like(pos)
    dpos[:, axis] = pre * (2 * Mz * q - 2 * Q * q * z)
    dbox = (-E / V) * V * np.linalg.inv(box).T
    dbox[axis] += pre * (-Q * Q * 2 * Lz / 12) * box[axis] / Lz
    return float(E), dq, dpos, dbox


def coulomb(pos, box, pairs, ds, bs, q, rcut, ethresh=1e-5, kappa=None, kmesh=None,
            spacing=None, kspace=True, rspace=True, slab_corr_flag=False, slab_axis=2):
    """CoulombForceModule forward + analytic gradients (one frame) -- pme.py:24-561.

    Returns dict: E, terms, dq, dpos (explicit, not via ds), dbox (explicit),
    dds (gradient w.r.t. the caller's distances), kmesh, kappa.
    """
    N = pos.shape[0]
    out = {"dq": np.zeros(N), "dpos": np.zeros((N, 3)), "dbox": np.zeros((3, 3)),
           "dds": np.zeros(len(ds)), "terms": {}}
    if kappa is None:
        kappa = ewald_kappa(rcut, ethresh) if kspace else 0.0
    out["kappa"] = kappa
    if box is None:
        E, dds, dq = coulomb_obc(q, pairs, ds, bs)
        out.update(E=E, dds=dds, dq=dq)
        return out
    E = 0.0
    if rspace:
        e, dds, dq = pme_real(q, pairs, ds, bs, kappa)
        out["terms"]["real"] = e
        E += e
        out["dds"] += dds
        out["dq"] += dq
    if kspace:
        if kmesh is None:
            km = auto_kmesh(box, kappa, ethresh, spacing)
        else:
            km = np.broadcast_to(np.asarray(kmesh, dtype=np.int64), (3,)).copy()
        out["kmesh"] = km
        r = pme_recip(pos, box, q, kappa, km)
        out["terms"]["reciprocal"] = r["E"]
        E += r["E"]
        out["dq"] += r["dq"]
        out["dpos"] += r["dpos"]
        out["dbox"] += r["dbox"]
        e, dq = pme_self(q, kappa)
        out["terms"]["self"] = e
        E += e
        out["dq"] += dq
        e, dq, db = pme_non_neutral(q, box, kappa)
        out["terms"]["non_neutral"] = e
        E += e
        out["dq"] += dq
        out["dbox"] += db
    if slab_corr_flag:
        e, dq, dp, db = slab_corr(q, pos, box, slab_axis)
        out["terms"]["slab_corr"] = e
        E += e
        out["dq"] += dq
        out["dpos"] += dp
        out["dbox"] += db
    out["E"] = E
    return out


def ds_backward(pos, box, pairs, g):
    """Chain dE/dds into positions / box through ds = |pbc_shift(r_i - r_j)|."""
    ri, rj = pos[pairs[:, 0]], pos[pairs[:, 1]]
    dpos = np.zeros_like(pos)
    dbox = np.zeros((3, 3))
    if box is None:
        dr = rj - ri
        d = np.linalg.norm(dr, axis=1)
        v = (g / np.where(d > 0, d, 1.0))[:, None] * dr
        np.add.at(dpos, pairs[:, 1], v)
        np.add.at(dpos, pairs[:, 0], -v)
        return dpos, None
    binv = np.linalg.inv(box)
    dr0 = ri - rj
    f = dr0 @ binv
    nimg = np.floor(f + 0.5)
    dr = (f - nimg) @ box
    d = np.linalg.norm(dr, axis=1)
    v = (g / np.where(d > 0, d, 1.0))[:, None] * dr
    n = pos.shape[0]
    for e in range(3):
        dpos[:, e] += np.bincount(pairs[:, 0], v[:, e], n) - np.bincount(pairs[:, 1], v[:, e], n)
    dbox = -nimg.T @ v
    return dpos, dbox


def coulomb_forces(pos, box, pairs, bs, q, **kw):
    """Energy and total forces including the path through ds (autograd equivalent)."""
    ds = pairs_ds(pos, pairs, box)
    o = coulomb(pos, box, pairs, ds, bs, q, **kw)
    dp, db = ds_backward(pos, box, pairs, o["dds"])
    o["forces"] = -(o["dpos"] + dp)
    if box is not None:
        o["box_grad"] = o["dbox"] + db
    return o


# --------------------------------------------------------------------------
# QEq
# --------------------------------------------------------------------------
class QEqSystem:
    """Quadratic QEq objective E(q) = site + Coulomb(PME) + damping -- qeq.py:351-458.

    ``grad(q)`` is dE/dq, ``hvp(p)`` the Hessian-vector product (E is
    quadratic in q, so hvp(p) = grad(p) - grad(0)).
    """

    def __init__(self, pos, box, chi, hardness, eta, pairs, ds, bs, rcut, ethresh=1e-5,
                 kappa=None, kmesh=None, spacing=None, kspace=True, rspace=True,
                 slab_corr_flag=False, slab_axis=2, damping_flag=True):
        self.kw = dict(rcut=rcut, ethresh=ethresh, kappa=kappa, kmesh=kmesh, spacing=spacing,
                       kspace=kspace, rspace=rspace, slab_corr_flag=slab_corr_flag, slab_axis=slab_axis)
        self.pos, self.box, self.chi, self.hardness, self.eta = pos, box, chi, hardness, eta
        self.pairs, self.ds, self.bs = pairs, ds, bs
        self.damping_flag = damping_flag
        self.n_evals = 0

    def energy_grad(self, q):
        self.n_evals += 1
        o = coulomb(self.pos, self.box, self.pairs, self.ds, self.bs, q, **self.kw)
        E, g = o["E"], o["dq"].copy()
        e, gs = site(q, self.chi, self.hardness)
        E += e
        g += gs
        if self.damping_flag:
            e, _, dq, _ = damping(q, self.eta, self.pairs, self.ds, self.bs)
            E += e
            g += dq
        return E, g

    def hvp(self, p):
        _, g1 = self.energy_grad(p)
        _, g0 = self.energy_grad(np.zeros_like(p))
        return g1 - g0

    def hessian(self):
        n = self.pos.shape[0]
        _, g0 = self.energy_grad(np.zeros(n))
        H = np.zeros((n, n))
        for k in range(n):
            e = np.zeros(n)
            e[k] = 1.0
            H[:, k] = self.energy_grad(e)[1] - g0
        return 0.5 * (H + H.T)


def projection_coeff(C):
    """C^T (C C^T)^-1 -- utils.py:152-172."""
    return C.T @ np.linalg.inv(C @ C.T)


def vector_projection(x, C, b=None):
    """x + C^T (C C^T)^-1 (b - C x) -- utils.py:175-210."""
    if b is None:
        b = np.zeros(C.shape[0])
    return x + projection_coeff(C) @ (b - C @ x)


def project_grad(g, C, coeff):
    """calc_pgrads projection -- utils.py:116-149."""
    return g - coeff @ (C @ g)


def solve_quadratic(sys_: QEqSystem, q0, C, b, max_iter=20, eps=1e-4, reinit_q=True):
    """Projected nonlinear CG with parabolic line search -- qeq.py:1374-1527
    (Polak-Ribiere+ update, optimizer.py:378-407).  Returns q, converge_iter."""
    q = vector_projection(q0, C, b) if reinit_q else q0.copy()
    coeff = projection_coeff(C)
    n = q.shape[0]
    fk, g = sys_.energy_grad(q)
    gk = project_grad(g, C, coeff)
    pk = -gk / np.linalg.norm(gk)
    conv = -1
    for ii in range(max_iter):
        # line search: f at x, x+p, x+2p -> parabola (qeq.py:1427-1475)
        hf = [fk]
        xk = q.copy()
        g_ls = gk
        early = False
        for _ in range(2):
            if np.linalg.norm(g_ls) / n < eps:
                early = True
                break
            xk = xk + pk
            f, g = sys_.energy_grad(xk)
            g_ls = project_grad(g, C, coeff)
            hf.append(f)
        if early:
            x_new = xk
        else:
            A = np.array([[0.0, 0.0, 1.0], [1.0, 1.0, 1.0], [4.0, 2.0, 1.0]])
            a2, a1, _ = np.linalg.solve(A, np.array(hf))
            x_new = q - a1 / (2 * a2) * pk
        f_new, g = sys_.energy_grad(x_new)
        g_new = project_grad(g, C, coeff)
        q, fk = x_new, f_new
        if np.linalg.norm(g_new) / n < eps:
            conv = ii
            gk = g_new
            break
        beta = max((g_new - gk) @ g_new / (gk @ gk), 0.0)
        pk = -g_new + beta * pk
        gk = g_new
    return q, conv


def solve_kkt(sys_: QEqSystem, C, b):
    """Dense KKT solve [[H, C^T], [C, 0]] -- qeq.py:1530-1617 (matinv_optimize)."""
    H = sys_.hessian()
    n = H.shape[0]
    _, g0 = sys_.energy_grad(np.zeros(n))     # = chi (plus constant terms)
    if C is None or C.shape[0] == 0:
        return np.linalg.solve(H, -g0)
    m = C.shape[0]
    A = np.block([[H, C.T], [C, np.zeros((m, m))]])
    rhs = np.concatenate([-g0, b])
    return np.linalg.solve(A, rhs)[:n]


def solve_linear_cg(sys_: QEqSystem, q0, C, b, tol=1e-6, max_iter=500):
    """Projected linear CG on the same objective (the matrix-free solver the
    CUDA path implements); stops on ||P grad||_2 / N < tol (qeq.py:1516)."""
    coeff = projection_coeff(C)
    q = vector_projection(q0, C, b)
    n = q.shape[0]
    _, g = sys_.energy_grad(q)
    r = -project_grad(g, C, coeff)
    p = r.copy()
    rr = r @ r
    it = 0
    while np.sqrt(rr) / n >= tol and it < max_iter:
        Hp = project_grad(sys_.hvp(p), C, coeff)
        a = rr / (p @ Hp)
        q = q + a * p
        r = r - a * Hp
        rr_new = r @ r
        p = r + rr_new / rr * p
        rr = rr_new
        it += 1
    return q, it


# --------------------------------------------------------------------------
# electrode (constant potential)
# --------------------------------------------------------------------------
def setup_from_lammps(n_atoms, constraints, symm=False):
    """electrode.py:203-285.  ``constraints``: list of dicts with keys
    indices, mode ('conp'|'conq'), value, eta (LAMMPS 1/length), chi, hardness, ffield."""
    mask = np.zeros(n_atoms, dtype=bool)
    eta = np.zeros(n_atoms)
    chi = np.zeros(n_atoms)
    hard = np.zeros(n_atoms)
    C, b, ffm, ffp = [], [], [], []
    for c in constraints:
        idx = np.asarray(c["indices"], dtype=int)
        mask[idx] = True
        eta[idx] = 1 / c["eta"] * np.sqrt(2) / 2.0
        chi[idx] = c.get("chi", 0.0)
        hard[idx] = c.get("hardness", 0.0)
        if c["mode"] == "conq":
            row = np.zeros((1, n_atoms))
            row[0, idx] = 1.0
            C.append(row)
            b.append(c["value"])
        if c["mode"] == "conp":
            chi[idx] -= c["value"]
        if c.get("ffield", False):
            row = np.zeros((1, n_atoms))
            row[0, idx] = 1.0
            ffm.append(row)
            ffp.append(c["value"])
    if symm:
        C.append(np.ones((1, n_atoms)))
        b.append(0.0)
    if C:
        Cm = np.concatenate(C, 0)[:, mask]
        bv = np.array(b)
    else:
        Cm = np.zeros((0, int(mask.sum())))
        bv = np.zeros(0)
    ffm = np.concatenate(ffm, 0).astype(bool) if len(ffm) == 2 else None
    ffp = np.array(ffp) if ffm is not None else None
    return mask, eta, chi, hard, Cm, bv, ffm, ffp


def finite_field_add_chi(pos, box, ffm, ffp, axis=2):
    """electrode.py:288-336."""
    drop = ffp[0] - ffp[1]
    mx0 = pos[ffm[0], axis].max()
    mx1 = pos[ffm[1], axis].max()
    lz = box[axis][axis]
    z = pos[:, axis] / lz
    if mx0 > mx1:
        off, ef = z, -drop / lz
    else:
        off, ef = -z, drop / lz
    pot = drop * off
    return pot[ffm[0] | ffm[1]], ef


def electrode_infer(pos, box, charges, pairs, ds, bs, mask, eta, chi, hardness, C, b, ffm, ffp,
                    rcut, ethresh=1e-5, kappa=None, kmesh=None, slab_corr_flag=False, slab_axis=2,
                    solver="kkt", tol=1e-8):
    """Constant-potential electrode solve + final energy and forces -- electrode.py:339-560."""
    kw = dict(rcut=rcut, ethresh=ethresh, kappa=kappa, kmesh=kmesh, slab_corr_flag=slab_corr_flag,
              slab_axis=slab_axis)
    efield = None
    q_full = charges.copy()
    if mask.sum() > 0:
        # chi_elec = dE/dq with electrode charges zeroed (electrode.py:49-84, 490-500)
        qm = np.where(mask, 0.0, charges)
        s = QEqSystem(pos, box, np.zeros_like(eta), np.zeros_like(eta), eta, pairs, ds, bs, **kw)
        _, phi = s.energy_grad(qm)
        chi_e = (chi + phi)[mask]
        if ffm is not None:
            add, ef = finite_field_add_chi(pos, box, ffm, ffp, slab_axis)
            chi_e = chi_e + add
            efield = np.zeros(3)
            efield[slab_axis] = ef
        pm = mask[pairs[:, 0]] & mask[pairs[:, 1]]
        mapping = np.zeros(mask.size, dtype=np.int64)
        mapping[np.nonzero(mask)[0]] = np.arange(mask.sum())
        sub_pairs = np.stack([mapping[pairs[pm, 0]], mapping[pairs[pm, 1]]], 1)
        sub = QEqSystem(pos[mask], box, chi_e, hardness[mask], eta[mask], sub_pairs, ds[pm], bs[pm], **kw)
        if solver == "kkt":
            qe = solve_kkt(sub, C, b)
        else:
            Cc = C if C.shape[0] > 0 else np.zeros((0, int(mask.sum())))
            qe, _ = solve_linear_cg(sub, charges[mask], Cc, b, tol=tol)
        q_full[mask] = qe
    # final energy/forces with chi = hardness = 0 (electrode.py:87-133)
    o = coulomb_forces(pos, box, pairs, bs, q_full, **kw)
    E = o["E"]
    s = QEqSystem(pos, box, np.zeros_like(eta), np.zeros_like(eta), eta, pairs, ds, bs, **kw)
    Ed, dds_d, _, _ = damping(q_full, eta, pairs, ds, bs)
    dpd, _ = ds_backward(pos, box, pairs, dds_d)
    E += Ed
    F = o["forces"] - dpd
    if efield is not None:
        F = F + q_full[:, None] * efield[None, :]
        E += float((efield[None, :] * q_full[:, None] * pos).sum())
    return E, F, q_full
