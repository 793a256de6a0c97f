"""The continuous-batching server on the GPU: every request's J/K per cycle
is the same served alone and in the mix (1e-10 absolute, the plain form's
parity bar), requests overlap on the device, admission keeps to the memory
budget, and the mixed form's energies stay within 1e-7 Eh of the plain
form's."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ATOL = 1e-10


@pytest.fixture(scope='module')
def torch():
    import torch
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    return torch


def test_results_same_alone_and_in_the_mix(torch):
    from electrolites_b200.serve import JKServer, latency_stats, poisson_requests, serve_alone
    reqs = poisson_requests(6, rate=5000.0, seed=3, n_min=2, n_max=8, cycles=3, keep=True)
    srv = JKServer()
    srv.run(reqs)
    assert max(srv.batch_sizes) > 1, 'requests should share batched builds'
    assert all(r.done_cycles == 3 and r.finished is not None for r in reqs)
    for r in reqs:
        alone = serve_alone(r)
        assert len(alone) == len(r.results) == 3
        for (mj, mk), (aj, ak) in zip(r.results, alone):
            assert np.abs(mj - aj).max() <= ATOL
            assert np.abs(mk - ak).max() <= ATOL
    st = latency_stats(reqs)
    assert 0 < st['p50_ms'] <= st['p99_ms'] and st['mols_per_s'] > 0
    assert srv.used == 0


def test_admission_keeps_to_the_memory_budget(torch):
    """A budget that holds one request at a time serialises them; every
    request still completes."""
    from electrolites_b200.serve import JKServer, matrix_bytes, poisson_requests, table_bound
    reqs = poisson_requests(4, rate=5000.0, seed=4, n_min=3, n_max=5, cycles=2)
    need = [matrix_bytes(r.dms.shape[-1], r.mol.nbas, r.dms.shape[0]) + table_bound(r.mol.nbas)
            for r in reqs]
    srv = JKServer(hbm_budget=float(min(need)) + 2.0)
    srv.run(reqs)
    assert max(srv.batch_sizes) == 1
    assert all(r.done_cycles == 2 for r in reqs)
    srv2 = JKServer(hbm_budget=float(sum(need)) + 2.0)
    srv2.run(poisson_requests(4, rate=5000.0, seed=4, n_min=3, n_max=5, cycles=2))
    assert max(srv2.batch_sizes) > 1


def test_mixed_serving_energies(torch):
    from electrolites_b200.serve import JKServer, poisson_requests
    plain = poisson_requests(4, rate=5000.0, seed=5, n_min=3, n_max=10, cycles=2)
    mixed = poisson_requests(4, rate=5000.0, seed=5, n_min=3, n_max=10, cycles=2)
    JKServer().run(plain)
    JKServer(mixed_threshold=1e-6).run(mixed)
    for p, m in zip(plain, mixed):
        for (pj, pk), (mj, mk) in zip(p.energies, m.energies):
            assert abs(pj - mj) <= 1e-7 and abs(pk - mk) <= 1e-7


def test_incremental_serving(torch):
    """Incremental mode: cycles between full rebuilds build J/K of the
    density change and add them.  Every cycle's J/K is the same alone and
    in the mix (1e-10), and within 1e-9 of a full build of that cycle's
    density (the terms the screening of the change drops are each below
    direct_scf_tol)."""
    from electrolites_b200.serve import JKServer, poisson_requests, serve_alone
    reqs = poisson_requests(4, rate=5000.0, seed=7, n_min=2, n_max=6, cycles=4, keep=True)
    srv = JKServer(incremental=True, rebuild_every=3)
    srv.run(reqs)
    assert max(srv.batch_sizes) > 1
    for r in reqs:
        inc_alone = serve_alone(r, incremental=True, rebuild_every=3)
        full = serve_alone(r)
        for c, ((mj, mk), (aj, ak), (fj, fk)) in enumerate(zip(r.results, inc_alone, full)):
            assert np.abs(mj - aj).max() <= ATOL
            assert np.abs(mk - ak).max() <= ATOL
            assert np.abs(mj - fj).max() <= 1e-9 and np.abs(mk - fk).max() <= 1e-9
