"""Seeded synthetic workloads for the benchmark and the parity tests.

Every generator returns a plain dict of numpy arrays (host memory) with the
keys ``positions`` (n, 3) float64, ``cell`` (3, 3) float64 (rows are lattice
vectors), ``pbc`` (3,) bool, ``cutoff`` (float, per-atom radii or a per-type
matrix), optionally ``numbers`` (n,) int32, and ``quantities``.  There is no
public dataset behind any of them: the shapes, sizes and value distributions
are the ones the benchmark configurations name, drawn from
``numpy.random.default_rng(seed)``.
"""

import math

import numpy as np


def plain_small(seed=0, n=1000, box=10.0, cutoff=2.5):
    """1,000 atoms uniform in a 10 A cube, periodic, scalar cutoff 2.5 A."""
    rng = np.random.default_rng(seed)
    pos = rng.uniform(0.0, box, size=(n, 3))
    return dict(positions=pos, cell=np.diag([box, box, box]).astype(float),
                pbc=np.array([True, True, True]), cutoff=float(cutoff),
                quantities="ijdDS")


def fcc_bulk(seed=0, reps=64, a=3.6, sigma=0.1, cutoff=5.0, shear=(0.2, 0.1)):
    """FCC lattice of reps^3 unit cells (4 sites each) in a sheared periodic
    cell rows [[L,0,0],[xy*L,L,0],[xz*L,0,L]], Gaussian jitter sigma."""
    rng = np.random.default_rng(seed)
    L = reps * a
    cell = np.array([[L, 0.0, 0.0], [shear[0] * L, L, 0.0], [shear[1] * L, 0.0, L]])
    basis = np.array([[0.0, 0.0, 0.0], [0.5, 0.5, 0.0], [0.5, 0.0, 0.5],
                      [0.0, 0.5, 0.5]])
    g = np.stack(np.meshgrid(np.arange(reps), np.arange(reps), np.arange(reps),
                             indexing="ij"), axis=-1).reshape(-1, 3).astype(float)
    frac = ((g[:, None, :] + basis[None, :, :]) / reps).reshape(-1, 3)
    pos = frac @ cell + rng.normal(0.0, sigma, size=frac.shape)
    return dict(positions=np.ascontiguousarray(pos), cell=cell,
                pbc=np.array([True, True, True]), cutoff=float(cutoff),
                quantities="ijdDS")


def sparse_slab(seed=0, n=200_000, box=400.0, z0=180.0, z1=220.0,
                cutoffs=((2.0, 3.0), (3.0, 4.0))):
    """A 40 A slab of n atoms in a 400 A box, pbc (T,T,F), two types 50/50
    with a per-type cutoff matrix."""
    rng = np.random.default_rng(seed)
    xy = rng.uniform(0.0, box, size=(n, 2))
    z = rng.uniform(z0, z1, size=(n, 1))
    pos = np.ascontiguousarray(np.hstack([xy, z]))
    types = rng.integers(0, 2, size=n).astype(np.int32)
    return dict(positions=pos, cell=np.diag([box, box, box]).astype(float),
                pbc=np.array([True, True, False]),
                cutoff=np.array(cutoffs, dtype=float), numbers=types,
                quantities="ijdD")


def dilute_gas(seed=0, n=200_000, per_cell=0.5, cutoff=3.0):
    """n atoms uniform in a periodic cube sized so that the cutoff-sized cell
    grid holds `per_cell` atoms per cell on average (0.5: about 1.3 atoms
    per occupied cell), scalar cutoff, ijdDS."""
    rng = np.random.default_rng(seed)
    box = (n / per_cell) ** (1.0 / 3.0) * cutoff
    pos = rng.uniform(0.0, box, size=(n, 3))
    return dict(positions=pos, cell=np.diag([box, box, box]).astype(float),
                pbc=np.array([True, True, True]), cutoff=float(cutoff),
                quantities="ijdDS")


def _triclinic_cell(rng, edges, angles_deg):
    a, b, c = edges
    al, be, ga = np.radians(angles_deg)
    va = np.array([a, 0.0, 0.0])
    vb = np.array([b * math.cos(ga), b * math.sin(ga), 0.0])
    cx = c * math.cos(be)
    cy = c * (math.cos(al) - math.cos(be) * math.cos(ga)) / math.sin(ga)
    cz2 = c * c - cx * cx - cy * cy
    if cz2 <= (0.05 * c) ** 2:
        return None
    return np.array([va, vb, [cx, cy, math.sqrt(cz2)]])


def batched_systems(seed=1, nsys=4096, nmin=8, nmax=512, density=0.08,
                    radii=(3.0, 6.0), edge_range=(8.0, 25.0),
                    angle_range=(70.0, 110.0), min_edge=8.0):
    """Independent small systems: sizes log-uniform in [nmin, nmax], each with
    its own random triclinic cell (edges and angles drawn from the ranges,
    then scaled isotropically to the target density with every edge kept at
    least `min_edge`), random pbc flags, uniform fractional positions and
    per-atom radii (pair cutoff = r_i + r_j)."""
    rng = np.random.default_rng(seed)
    systems = []
    for _ in range(nsys):
        n = int(math.floor(math.exp(rng.uniform(math.log(nmin), math.log(nmax)))))
        n = max(nmin, min(nmax, n))
        while True:
            edges = rng.uniform(*edge_range, size=3)
            angles = rng.uniform(*angle_range, size=3)
            cell = _triclinic_cell(rng, edges, angles)
            if cell is not None:
                break
        vol = abs(np.linalg.det(cell))
        scale = (n / density / vol) ** (1.0 / 3.0)
        cell = cell * scale
        emin = np.linalg.norm(cell, axis=1).min()
        if emin < min_edge:
            cell = cell * (min_edge / emin)
        pbc = rng.integers(0, 2, size=3).astype(bool)
        frac = rng.uniform(0.0, 1.0, size=(n, 3))
        pos = np.ascontiguousarray(frac @ cell)
        r = rng.uniform(*radii, size=n)
        systems.append(dict(positions=pos, cell=cell, pbc=pbc, cutoff=r,
                            quantities="ijdDS"))
    return systems


def diff_lattice(seed=0, shape=(64, 64, 32), spacing=2.8, sigma=0.15,
                 cutoff=6.0):
    """Jittered simple-cubic lattice in a triclinic periodic cell."""
    rng = np.random.default_rng(seed)
    nx, ny, nz = shape
    s = spacing
    cell = np.array([[nx * s, 0.0, 0.0], [0.1 * nx * s, ny * s, 0.0],
                     [0.05 * nx * s, 0.05 * nx * s, nz * s]])
    g = np.stack(np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz),
                             indexing="ij"), axis=-1).reshape(-1, 3).astype(float)
    frac = g / np.array([nx, ny, nz], dtype=float)
    pos = frac @ cell + rng.normal(0.0, sigma, size=frac.shape)
    return dict(positions=np.ascontiguousarray(pos), cell=cell,
                pbc=np.array([True, True, True]), cutoff=float(cutoff),
                quantities="ijdDS")


def lj_droplet(n=1_000_000, lattice=1.6, cutoff=2.5, margin=3.0):
    """The LJ droplet of the reference's molecular-dynamics benchmark (reduced
    units): the n FCC sites (lattice constant `lattice`) closest to the
    centroid of an FCC block, centred at the origin, in an open (non-periodic)
    cubic box that encloses them with `margin` to spare; scalar cutoff."""
    nc = int(np.ceil(np.cbrt(3.0 * n / (16.0 * np.pi)))) + 2
    r = np.arange(-nc, nc + 1, dtype=float)
    g = np.stack(np.meshgrid(r, r, r, indexing="ij"), axis=-1).reshape(-1, 3)
    basis = np.array([[0.0, 0.0, 0.0], [0.5, 0.5, 0.0], [0.5, 0.0, 0.5], [0.0, 0.5, 0.5]])
    sites = ((g[:, None, :] + basis[None, :, :]) * lattice).reshape(-1, 3)
    sites -= sites.mean(axis=0)
    r2 = np.einsum("ij,ij->i", sites, sites)
    keep = np.argsort(r2, kind="stable")[:n]
    pos = np.ascontiguousarray(sites[keep])
    lo = pos.min(axis=0) - margin
    hi = pos.max(axis=0) + margin
    side = float((hi - lo).max())
    return dict(positions=pos - lo, cell=np.diag([side, side, side]),
                pbc=np.array([False, False, False]), cutoff=float(cutoff), quantities="ij")
