"""B200-native direct-SCF Coulomb/exchange (J/K) engine.

Public API:
  * ``jk.VHFOpt`` -- a plan per molecule (device-resident pair and screening
    tables), with ``get_jk`` / ``get_k`` / ``get_j``;
  * ``jk.get_jk(mol, dm, ...)``, ``jk.get_j``, ``jk.get_k`` -- GPU4PySCF's
    module-level signatures;
  * ``jk.jk_energy_per_atom`` / ``VHFOpt.jk_energy_per_atom`` -- the nuclear
    gradient of the two-electron energy (GPU4PySCF's
    ``grad.rhf._jk_energy_per_atom``);
  * ``patch(*names)`` / ``patch_all()`` -- install the engine in place of
    GPU4PySCF's ``_VHFOpt.get_jk`` / ``get_k``, ``j_engine._VHFOpt.get_j``
    and ``grad.rhf._jk_energy_per_atom``, the targets the reference patches
    (electrolites/__init__.py:59-61, 73, 107, 329-350).  ``check_targets()``
    reports which targets exist.
"""
from __future__ import annotations

import importlib

from . import jk  # noqa: F401

__all__ = ['jk', 'patch', 'patch_all', 'patched', 'check_targets', 'MODULES']

# name -> (module path, class name, method name)
_TARGETS = {
    'fastjk': ('gpu4pyscf.scf.jk', '_VHFOpt', 'get_jk'),
    'fastk': ('gpu4pyscf.scf.jk', '_VHFOpt', 'get_k'),
    'fastj': ('gpu4pyscf.scf.j_engine', '_VHFOpt', 'get_j'),
    'fastejk': ('gpu4pyscf.grad.rhf', None, '_jk_energy_per_atom'),   # a module function
}
MODULES = tuple(_TARGETS)
_PATCHED = {}


def check_targets():
    """{name: None if the target exists, else the reason it does not}."""
    out = {}
    for name, (mod, cls, meth) in _TARGETS.items():
        try:
            m = importlib.import_module(mod)
            c = m if cls is None else getattr(m, cls)
            getattr(c, meth)
            out[name] = None
        except Exception as err:   # noqa: BLE001
            out[name] = f'{type(err).__name__}: {err}'
    return out


def _plan_for(opt):
    """The engine plan attached to a GPU4PySCF option object, built from its
    sorted Cartesian molecule on first use."""
    plan = getattr(opt, '_jk_b200', None)
    if plan is None:
        mol = getattr(opt, 'sorted_mol', None) or opt.mol
        tol = getattr(opt, 'direct_scf_tol', jk.DEFAULT_TOL)
        plan = jk.VHFOpt(_CartView(mol), tol).build()
        opt._jk_b200 = plan
    return plan


class _CartView:
    """A molecule seen through its Cartesian AO layout (GPU4PySCF's option
    objects work in the sorted Cartesian basis)."""

    def __init__(self, mol):
        self._m = mol
        self._atm, self._bas, self._env = mol._atm, mol._bas, mol._env

    def ao_loc_nr(self, cart=True):
        return self._m.ao_loc_nr(cart=True)


def _out(x, like):
    if hasattr(like, '__cuda_array_interface__') and not hasattr(like, 'data_ptr'):
        import cupy
        return cupy.asarray(x)
    return x


def _resolve_omega(opt, omega):
    """The operator's omega: the caller's, else the one riding on the option
    object's molecule, as the reference resolves it (resolve_rsh,
    electrolites/compat.py:178-187, called at electrolites/fastjk.py:287 and
    electrolites/fastk.py:661): GPU4PySCF sets the range of a
    range-separated functional on that mol.  None when neither names one."""
    if omega is not None:
        return omega
    for name in ('mol', 'sorted_mol'):
        m = getattr(opt, name, None)
        w = getattr(m, 'omega', None) if m is not None else None
        if w:
            return float(w)
    return None


def _get_jk(self, dms, hermi, verbose=None):
    if callable(dms):
        dms = dms()
    vj, vk = _plan_for(self).get_jk(dms, hermi, verbose, omega=_resolve_omega(self, None))
    return _out(vj, dms), _out(vk, dms)


def _get_k(self, dms, hermi, verbose=None, omega=None, lr_factor=None, sr_factor=None):
    if callable(dms):
        dms = dms()
    return _out(_plan_for(self).get_k(dms, hermi, verbose, _resolve_omega(self, omega),
                                      lr_factor, sr_factor), dms)


def _get_j(self, dms, verbose=None):
    if callable(dms):
        dms = dms()
    return _out(_plan_for(self).get_j(dms, verbose), dms)


def _jk_energy_per_atom(vhfopt, dm, j_factor=1., k_factor=1., verbose=None):
    """grad.rhf._jk_energy_per_atom: dm in the option's molecule basis,
    brought to its sorted Cartesian basis by the option object itself (as
    electrolites/fastejk.py:273-276 does); the operator's omega from the
    option's molecule.  Returns a numpy (natm, 3) array."""
    nao = vhfopt.mol.nao
    dm = dm.reshape(-1, nao, nao) if hasattr(dm, 'reshape') else dm
    dms = vhfopt.apply_coeff_C_mat_CT(dm)
    omega = _resolve_omega(vhfopt, None) or 0.0
    g = _plan_for(vhfopt).jk_energy_per_atom(dms, j_factor, k_factor, omega)
    return g.cpu().numpy()


_IMPL = {'fastjk': _get_jk, 'fastk': _get_k, 'fastj': _get_j,
         'fastejk': _jk_energy_per_atom}


def patch(*names):
    """Install the engine for the named targets ('fastjk', 'fastk',
    'fastj', 'fastejk').  Raises if a target does not exist (no silent partial
    patching)."""
    status = check_targets()
    for name in names:
        if name not in _TARGETS:
            raise KeyError(f'unknown target {name!r}; known: {MODULES}')
        if status[name] is not None:
            raise ImportError(f'cannot patch {name}: {status[name]}')
    for name in names:
        if name in _PATCHED:
            continue
        mod, cls, meth = _TARGETS[name]
        m = importlib.import_module(mod)
        c = m if cls is None else getattr(m, cls)
        _PATCHED[name] = getattr(c, meth)
        setattr(c, meth, _IMPL[name])
    return list(_PATCHED)


def patch_all():
    return patch(*MODULES)


def patched():
    return sorted(_PATCHED)
