"""Write oracle J/K fixtures for the water cluster of the CPU-runnable
workload: (H2O)_8, rigid waters in a 7 A cube (seed 20261203), 6-31G* shell
structure, one atom-block density, direct_scf_tol 1e-13.

The fixture holds the geometry seed, the density and the oracle's vj, vk, so
the GPU parity test can compare against it without running the oracle.

    python tests/golden/make_oracle_fixtures.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from electrolites_b200 import clusters  # noqa: E402
from oracle import oracle as O  # noqa: E402

SEED = 20261203


def main():
    mol = clusters.water_mole(8, 7.0, SEED, basis='6-31g*', cart=True)
    D = clusters.atomic_density(mol, SEED)
    vj, vk, nq = O.jk(mol, D, tol=1e-13)
    np.savez_compressed(os.path.join(HERE, 'h2o8_631gs_oracle.npz'), seed=SEED,
                        dm=D, vj=vj, vk=vk, nquartets=nq, tol=1e-13)
    print('quartets', nq)


if __name__ == '__main__':
    main()
