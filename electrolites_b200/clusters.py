"""Seeded water clusters and the densities the J/K workloads are built on.

Geometry: rigid waters (O-H 0.9572 A, H-O-H 104.52 deg) with uniformly random
orientations, oxygen positions uniform in a cube, rejected when closer than
2.7 A to an oxygen already placed.

Densities: the workloads ask for PySCF's "minao" initial guess, a
superposition of atomic densities projected into the AO basis, which is
block-diagonal by atom.  Without PySCF's atomic data, `atomic_density`
builds a density with the same structure: per atom, a seeded positive
semi-definite block D_A = sum_i n_i c_i c_i^T over S_A-orthonormal vectors,
scaled so that tr(D_A S_A) equals the atom's electron count; zero between
atoms.
"""
from __future__ import annotations

import math

import numpy as np

from .gto import Mole

R_OH = 0.9572
THETA_HOH = math.radians(104.52)


def _random_rotation(rng):
    q = rng.standard_normal(4)
    q /= np.linalg.norm(q)
    w, x, y, z = q
    return np.array([
        [1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
        [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
        [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def water_cluster(n: int, edge: float, seed: int, min_oo: float = 2.7,
                  max_tries: int = 200000):
    """[(symbol, (x, y, z)), ...] in Angstrom for n waters in a cube."""
    rng = np.random.default_rng(seed)
    local = np.array([[0.0, 0.0, 0.0],
                      [R_OH * math.sin(THETA_HOH / 2), 0.0,
                       R_OH * math.cos(THETA_HOH / 2)],
                      [-R_OH * math.sin(THETA_HOH / 2), 0.0,
                       R_OH * math.cos(THETA_HOH / 2)]])
    oxygens = []
    atoms = []
    tries = 0
    while len(oxygens) < n:
        tries += 1
        if tries > max_tries:
            raise RuntimeError(f'cannot place {n} waters in a {edge} A cube')
        c = rng.uniform(0, edge, 3)
        if oxygens and np.min(np.linalg.norm(np.array(oxygens) - c, axis=1)) < min_oo:
            continue
        oxygens.append(c)
        xyz = local @ _random_rotation(rng).T + c
        atoms += [('O', tuple(xyz[0])), ('H', tuple(xyz[1])), ('H', tuple(xyz[2]))]
    return atoms


def water_mole(n: int, edge: float, seed: int, basis: str = '6-31g*',
               cart: bool = True) -> Mole:
    return Mole(water_cluster(n, edge, seed), basis=basis, cart=cart)


def atomic_density(mol: Mole, seed: int) -> np.ndarray:
    """Block-diagonal (by atom) symmetric density, Cartesian AO basis.

    Per atom a minimal set of occupied orbitals is taken from the atom's own
    shells -- the first s shell (core), the second s shell and the first p
    shell when present (valence) -- mixed with 5% of the atom's other
    functions by a seeded random combination and orthonormalised in the
    atom's overlap metric.  Occupations follow a spherical atom: 2 per s
    orbital, the rest of the electrons spread evenly over the p orbitals.
    """
    from .gto import overlap_cart
    rng = np.random.default_rng(seed)
    nao = mol.nao_cart
    loc = mol.ao_loc_nr(True)
    D = np.zeros((nao, nao))
    cache = {}
    for ia, (b0, b1, p0, p1) in enumerate(mol.aoslice_by_atom(cart=True)):
        nel = int(mol._atm[ia, 0])
        key = mol.elements[ia] if hasattr(mol, 'elements') else ia
        if key not in cache:
            cache[key] = overlap_cart(mol, list(range(b0, b1)))
        Sa = cache[key]
        na = p1 - p0
        s_shells = [s for s in range(b0, b1) if mol._bas[s, 1] == 0]
        p_shells = [s for s in range(b0, b1) if mol._bas[s, 1] == 1]
        cols, occ = [], []
        nel_left = nel
        for s in s_shells[:2]:
            if nel_left <= 0:
                break
            cols.append([loc[s] - p0])
            occ.append(min(2.0, nel_left))
            nel_left -= occ[-1]
        if nel_left > 0 and p_shells:
            s = p_shells[0]
            for c in range(3):
                cols.append([loc[s] - p0 + c])
                occ.append(nel_left / 3)
            nel_left = 0
        V = np.zeros((na, len(cols)))
        for k, c in enumerate(cols):
            V[c[0], k] = 1.0
        V += 0.05 * rng.standard_normal(V.shape) * (V == 0)
        w, u = np.linalg.eigh(V.T @ Sa @ V)
        C = V @ (u / np.sqrt(w)) @ u.T
        Da = (C * np.array(occ)) @ C.T
        Da *= nel / np.trace(Da @ Sa)
        D[p0:p1, p0:p1] = Da
    return D


def uhf_pair(D: np.ndarray, seed: int, sigma_rel: float = 1e-3):
    """(D_alpha, D_beta): D_alpha = D/2 and D_beta = D_alpha plus a seeded
    symmetric Gaussian perturbation of standard deviation
    sigma_rel * max|D_alpha|."""
    rng = np.random.default_rng(seed)
    da = 0.5 * D
    p = rng.standard_normal(D.shape) * (sigma_rel * np.abs(da).max())
    p = (p + p.T) / math.sqrt(2)
    return np.stack([da, da + p])


def density_stack(D: np.ndarray, n_dm: int, seed: int, sigma_rel: float = 1e-3):
    """n_dm densities made like the UHF pair: D/2, then D/2 plus independent
    seeded symmetric Gaussian perturbations (sigma_rel * max|D/2|)."""
    if n_dm == 1:
        return (0.5 * D)[None].copy()
    rng = np.random.default_rng(seed)
    da = 0.5 * D
    out = [da]
    for _ in range(n_dm - 1):
        p = rng.standard_normal(D.shape) * (sigma_rel * np.abs(da).max())
        out.append(da + (p + p.T) / math.sqrt(2))
    return np.stack(out)


def uneven_batch(n_mol: int, seed: int, n_min: int = 1, n_max: int = 24,
                 bases=('6-31g*',), dm_min: int = 1, dm_max: int = 4):
    """Seeded batch of uneven water clusters: per molecule n ~ U{n_min..n_max}
    waters in a cube of edge 3.1 n^(1/3) A (2.7 A minimum O-O), a basis drawn
    uniformly from `bases`, and 1..4 densities (density_stack of its atomic
    density).  Returns [(mol, dms), ...]."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n_mol):
        n = int(rng.integers(n_min, n_max + 1))
        k = int(rng.integers(dm_min, dm_max + 1))
        basis = bases[int(rng.integers(0, len(bases)))]
        s = seed * 1000 + i
        mol = water_mole(n, 3.1 * n ** (1.0 / 3.0), s, basis=basis)
        out.append((mol, density_stack(atomic_density(mol, s), k, s + 1)))
    return out
