"""A minimal molecule/basis container in PySCF's array layout.

The J/K engine reads a molecule the way PySCF's integral library does: the
integer tables ``_atm`` (ATM_SLOTS = 6 per atom) and ``_bas`` (BAS_SLOTS = 8
per shell) and the float array ``_env``.  A real ``pyscf.gto.Mole`` has those
attributes and can be passed to everything in this package unchanged.  This
module builds the same arrays for the synthetic water clusters used by the
tests and the benchmark, without PySCF.

Coefficient convention (PySCF's ``make_bas_env``): the coefficient stored at
PTR_COEFF for primitive p of a shell of angular momentum l is
``d_p * N_l(a_p)`` with the radial normalisation
``N_l(a) = 1 / sqrt(Gamma(l + 3/2) / (2 (2a)^(l + 3/2)))``, rescaled so that
the contracted radial function has unit norm.  The angular factor libcint
applies to s and p shells is not stored; the engine applies it.

Cartesian components are ordered as PySCF orders them: for each lx from l
down to 0, ly from l - lx down to 0.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import basis_synth

ANGSTROM_TO_BOHR = 1.0 / 0.52917721092
ATM_SLOTS, BAS_SLOTS = 6, 8
CHARGE_OF, PTR_COORD = 0, 1
ATOM_OF, ANG_OF, NPRIM_OF, NCTR_OF, KAPPA_OF, PTR_EXP, PTR_COEFF = range(7)
PTR_ENV_START = 20

NUC_CHARGE = {'H': 1, 'He': 2, 'C': 6, 'N': 7, 'O': 8, 'F': 9}


def ncart(l: int) -> int:
    return (l + 1) * (l + 2) // 2


def nsph(l: int) -> int:
    return 2 * l + 1


def cart_comps(l: int):
    return [(lx, ly, l - lx - ly) for lx in range(l, -1, -1)
            for ly in range(l - lx, -1, -1)]


def gaussian_int(n: int, a: float) -> float:
    """int_0^inf r^n exp(-a r^2) dr."""
    return math.gamma((n + 1) / 2) / (2 * a ** ((n + 1) / 2))


def gto_norm(l: int, a: float) -> float:
    return 1.0 / math.sqrt(gaussian_int(2 * l + 2, 2 * a))


def normalize_shell(l: int, exps, coefs):
    exps = np.asarray(exps, dtype=np.float64)
    c = np.asarray(coefs, dtype=np.float64) * np.array(
        [gto_norm(l, a) for a in exps])
    ee = exps[:, None] + exps[None, :]
    s = np.einsum('p,q,pq->', c, c,
                  np.vectorize(lambda a: gaussian_int(2 * l + 2, a))(ee))
    return c / math.sqrt(s)


def _parse_atoms(atom):
    if isinstance(atom, str):
        out = []
        for item in atom.replace('\n', ';').split(';'):
            f = item.split()
            if len(f) == 4:
                out.append((f[0], tuple(float(v) for v in f[1:])))
        return out
    return [(s, tuple(float(v) for v in xyz)) for s, xyz in atom]


@dataclass
class Mole:
    """Molecule with a Gaussian basis, in PySCF's ``_atm/_bas/_env`` layout.

    atom:  "O 0 0 0; H 0 .76 .59" or [(symbol, (x, y, z)), ...], Angstrom.
    basis: a basis name known to ``basis_synth`` or a dict
           {symbol: [[l, (exp, coef), ...], ...]} (PySCF's internal format,
           one contraction per shell).
    """
    atom: object
    basis: object = '6-31g*'
    cart: bool = False
    _atm: np.ndarray = field(init=False, repr=False)
    _bas: np.ndarray = field(init=False, repr=False)
    _env: np.ndarray = field(init=False, repr=False)

    def __post_init__(self):
        self.build()

    def build(self):
        atoms = _parse_atoms(self.atom)
        if isinstance(self.basis, str):
            bdict = {s: basis_synth.shells(self.basis, s) for s, _ in atoms}
        else:
            bdict = self.basis
        env = [0.0] * PTR_ENV_START
        atm, bas = [], []
        self.elements = []
        for ia, (sym, xyz) in enumerate(atoms):
            self.elements.append(sym)
            ptr = len(env)
            env.extend(v * ANGSTROM_TO_BOHR for v in xyz)
            atm.append([NUC_CHARGE.get(sym, 0), ptr, 1, 0, 0, 0])
        for ia, (sym, _) in enumerate(atoms):
            for shell in bdict[sym]:
                l = int(shell[0])
                prims = np.asarray(shell[1:], dtype=np.float64)
                exps, coefs = prims[:, 0], prims[:, 1]
                c = normalize_shell(l, exps, coefs)
                pe = len(env)
                env.extend(exps.tolist())
                pc = len(env)
                env.extend(c.tolist())
                bas.append([ia, l, len(exps), 1, 0, pe, pc, 0])
        self._atm = np.asarray(atm, dtype=np.int32).reshape(-1, ATM_SLOTS)
        self._bas = np.asarray(bas, dtype=np.int32).reshape(-1, BAS_SLOTS)
        self._env = np.asarray(env, dtype=np.float64)
        return self

    # ------------------------------------------------------------------
    @property
    def natm(self) -> int:
        return len(self._atm)

    @property
    def nbas(self) -> int:
        return len(self._bas)

    def atom_coords(self) -> np.ndarray:
        """Bohr."""
        return np.array([self._env[p:p + 3] for p in self._atm[:, PTR_COORD]])

    @property
    def nelectron(self) -> int:
        return int(self._atm[:, CHARGE_OF].sum())

    def ao_loc_nr(self, cart=None) -> np.ndarray:
        cart = self.cart if cart is None else cart
        dims = [ncart(l) if cart else nsph(l) for l in self._bas[:, ANG_OF]]
        return np.concatenate([[0], np.cumsum(dims)]).astype(np.int32)

    @property
    def nao(self) -> int:
        return int(self.ao_loc_nr()[-1])

    @property
    def nao_cart(self) -> int:
        return int(self.ao_loc_nr(cart=True)[-1])

    def aoslice_by_atom(self, cart=None):
        loc = self.ao_loc_nr(cart)
        out = []
        for ia in range(self.natm):
            idx = np.nonzero(self._bas[:, ATOM_OF] == ia)[0]
            out.append((idx[0], idx[-1] + 1, loc[idx[0]], loc[idx[-1] + 1]))
        return np.array(out)

    def cart2sph_coeff(self) -> np.ndarray:
        """(nao_cart, nao_sph) matrix C with AO_sph = AO_cart @ C."""
        loc_c = self.ao_loc_nr(True)
        loc_s = self.ao_loc_nr(False)
        c = np.zeros((loc_c[-1], loc_s[-1]))
        for ish, l in enumerate(self._bas[:, ANG_OF]):
            c[loc_c[ish]:loc_c[ish + 1], loc_s[ish]:loc_s[ish + 1]] = \
                cart2sph_block(int(l))
        return c

    def intor_ovlp_cart(self) -> np.ndarray:
        """Cartesian overlap matrix (numpy, Obara-Saika), for building
        densities of a given electron count."""
        return overlap_cart(self)


# ----------------------------------------------------------------------
# Cartesian -> real spherical transformation
# ----------------------------------------------------------------------
def _real_ylm_times_rl(l, m, xyz):
    """r^l * real spherical harmonic Y_lm (orthonormal on the sphere) at
    points xyz (n, 3), from scipy's complex harmonics."""
    from scipy.special import sph_harm_y
    x, y, z = xyz.T
    r = np.sqrt(x * x + y * y + z * z)
    theta = np.arccos(np.clip(z / r, -1, 1))
    phi = np.arctan2(y, x)
    if m == 0:
        val = sph_harm_y(l, 0, theta, phi).real
    elif m > 0:
        val = math.sqrt(2) * (-1) ** m * sph_harm_y(l, m, theta, phi).real
    else:
        val = math.sqrt(2) * (-1) ** m * sph_harm_y(l, -m, theta, phi).imag
    return r ** l * val


_C2S_CACHE = {}


def cart2sph_block(l: int) -> np.ndarray:
    """(ncart(l), 2l+1) coefficients expressing r^l Y_lm through the
    Cartesian functions x^a y^b z^c as the engine normalises them
    (libcint's angular factor included for l < 2).  Spherical order is
    m = -l..l, except p, which PySCF keeps as x, y, z."""
    if l in _C2S_CACHE:
        return _C2S_CACHE[l]
    if l == 0:
        blk = np.ones((1, 1))
    elif l == 1:
        blk = np.eye(3)
    else:
        rng = np.random.default_rng(l)
        pts = rng.standard_normal((64, 3))
        mono = np.stack([pts[:, 0] ** a * pts[:, 1] ** b * pts[:, 2] ** c
                         for a, b, c in cart_comps(l)], axis=1)
        blk = np.zeros((ncart(l), 2 * l + 1))
        for k, m in enumerate(range(-l, l + 1)):
            target = _real_ylm_times_rl(l, m, pts)
            coef, *_ = np.linalg.lstsq(mono, target, rcond=None)
            coef[np.abs(coef) < 1e-13] = 0
            blk[:, k] = coef
    _C2S_CACHE[l] = blk
    return blk


# ----------------------------------------------------------------------
# Overlap integrals (only to normalise synthetic densities)
# ----------------------------------------------------------------------
def _overlap_1d(la, lb, a, b, Ax, Bx):
    p = a + b
    Px = (a * Ax + b * Bx) / p
    s = np.zeros((la + 2, lb + 2))
    s[0, 0] = math.sqrt(math.pi / p) * math.exp(-a * b / p * (Ax - Bx) ** 2)
    for i in range(la + 1):
        for j in range(lb + 1):
            if i == 0 and j == 0:
                continue
            if i > 0:
                v = (Px - Ax) * s[i - 1, j]
                if i > 1:
                    v += (i - 1) / (2 * p) * s[i - 2, j]
                if j > 0:
                    v += j / (2 * p) * s[i - 1, j - 1]
            else:
                v = (Px - Bx) * s[i, j - 1]
                if j > 1:
                    v += (j - 1) / (2 * p) * s[i, j - 2]
            s[i, j] = v
    return s


def common_fac(l: int) -> float:
    return {0: 0.282094791773878143, 1: 0.488602511902919921}.get(l, 1.0)


def overlap_cart(mol, shells=None) -> np.ndarray:
    """Cartesian overlap; with ``shells`` (a list of shell indices) only the
    block of those shells, in their AO order."""
    loc = mol.ao_loc_nr(True)
    coords = mol.atom_coords()
    bas, env = mol._bas, mol._env
    if shells is not None:
        dims = loc[1:] - loc[:-1]
        keep = np.zeros(mol.nbas, dtype=bool)
        keep[list(shells)] = True
        off = np.concatenate([[0], np.cumsum(np.where(keep, dims, 0))])
        S = np.zeros((off[-1], off[-1]))
        idx = sorted(shells)
    else:
        S = np.zeros((loc[-1], loc[-1]))
        off = loc
        idx = range(mol.nbas)
    for i in idx:
        li, npi = bas[i, ANG_OF], bas[i, NPRIM_OF]
        ei = env[bas[i, PTR_EXP]:bas[i, PTR_EXP] + npi]
        ci = env[bas[i, PTR_COEFF]:bas[i, PTR_COEFF] + npi] * common_fac(li)
        A = coords[bas[i, ATOM_OF]]
        for j in idx:
            lj, npj = bas[j, ANG_OF], bas[j, NPRIM_OF]
            ej = env[bas[j, PTR_EXP]:bas[j, PTR_EXP] + npj]
            cj = env[bas[j, PTR_COEFF]:bas[j, PTR_COEFF] + npj] * common_fac(lj)
            B = coords[bas[j, ATOM_OF]]
            blk = np.zeros((ncart(li), ncart(lj)))
            for a, ca in zip(ei, ci):
                for b, cb in zip(ej, cj):
                    sx = _overlap_1d(li, lj, a, b, A[0], B[0])
                    sy = _overlap_1d(li, lj, a, b, A[1], B[1])
                    sz = _overlap_1d(li, lj, a, b, A[2], B[2])
                    for u, (ax, ay, az) in enumerate(cart_comps(li)):
                        for v, (bx, by, bz) in enumerate(cart_comps(lj)):
                            blk[u, v] += ca * cb * sx[ax, bx] * sy[ay, by] * sz[az, bz]
            S[off[i]:off[i] + ncart(li), off[j]:off[j] + ncart(lj)] = blk
    return S
