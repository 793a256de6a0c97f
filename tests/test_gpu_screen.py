"""Per-build screening thresholds and the loose-then-tight schedule on the
GPU.  A plan made at 1e-13 that builds at 1e-10 gives the J/K of a plan
made at 1e-10 (1e-12) and the oracle's J-only and K-only builds at 1e-10
(1e-10; the engine screens J and K by separate tests); the schedule's
final J/K, after the tight rebuild and tight increments, is within 1e-9 of
a full tight build of the final density (the incremental form's bar), and a
request's J/K per cycle is the same served alone and in the mix (1e-10)."""
import numpy as np
import pytest

from electrolites_b200 import clusters

pytestmark = pytest.mark.gpu


@pytest.fixture(scope='module')
def torch():
    import torch
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    return torch


def test_build_threshold(torch, oracle):
    from electrolites_b200._lib import JKError
    from electrolites_b200.jk import VHFOpt
    mol = clusters.water_mole(4, 5.5, 2, basis='6-31g*')
    D = clusters.density_stack(clusters.atomic_density(mol, 2), 2, 3)
    d = torch.as_tensor(D, device='cuda')
    tight = VHFOpt(mol, 1e-13).build()
    tj, tk = tight.get_jk(d, 1)
    nq_tight = sum(v[0] for v in tight.class_counts().values())
    tight.direct_scf_tol = 1e-10
    lj, lk = tight.get_jk(d, 1)
    nq_loose = sum(v[0] for v in tight.class_counts().values())
    assert nq_loose < nq_tight
    ref = VHFOpt(mol, 1e-10).build()
    rj, rk = ref.get_jk(d, 1)
    assert float((lj - rj).abs().max()) <= 1e-12 and float((lk - rk).abs().max()) <= 1e-12
    # the engine screens J and K by their own tests: the oracle's J-only and
    # K-only builds apply the same ones
    oj, _, _ = oracle.jk(mol, D, tol=1e-10, with_k=False)
    _, ok, _ = oracle.jk(mol, D, tol=1e-10, with_j=False)
    assert np.abs(lj.cpu().numpy() - oj).max() <= 1e-10
    assert np.abs(lk.cpu().numpy() - ok).max() <= 1e-10
    tight.direct_scf_tol = 1e-13
    bj, bk = tight.get_jk(d, 1)
    assert float((bj - tj).abs().max()) <= 1e-12 and float((bk - tk).abs().max()) <= 1e-12
    assert sum(v[0] for v in tight.class_counts().values()) == nq_tight
    ref.direct_scf_tol = 1e-12
    with pytest.raises(JKError, match='below the plan'):
        ref.get_jk(d, 1)


def test_loose_then_tight_trajectory(torch):
    from electrolites_b200 import screen
    from electrolites_b200.jk import VHFOpt
    from electrolites_b200.serve import advance_density
    mol = clusters.water_mole(6, 6.5, 5, basis='6-31g*')
    d = torch.as_tensor(clusters.density_stack(clusters.atomic_density(mol, 5), 2, 6),
                        device='cuda')
    S = torch.as_tensor(mol.intor_ovlp_cart(), device='cuda')
    opt = VHFOpt(mol, 1e-13).build()
    lt = screen.LooseTightJK(opt, S)
    gen = torch.Generator(device='cuda')
    gen.manual_seed(7)
    for c in range(12):
        vj, vk = lt.jk(d)
        advance_density(d, 3e-2 * 0.5 ** c, gen)
    vj, vk = lt.jk(d)
    assert lt.decisions[0] == screen.FULL
    assert screen.LOOSE_INC in lt.decisions and screen.REBUILD in lt.decisions
    r = lt.decisions.index(screen.REBUILD)
    assert all(x == screen.LOOSE_INC for x in lt.decisions[1:r])
    assert all(x == screen.TIGHT_INC for x in lt.decisions[r + 1:]) and len(lt.decisions) > r + 1
    assert opt.direct_scf_tol == 1e-13
    fj, fk = opt.get_jk(d, 1)
    assert float((vj - fj).abs().max()) <= 1e-9 and float((vk - fk).abs().max()) <= 1e-9


def test_loose_then_tight_serving(torch):
    from electrolites_b200 import screen
    from electrolites_b200.serve import JKServer, poisson_requests, serve_alone
    reqs = poisson_requests(4, rate=5000.0, seed=9, n_min=2, n_max=6, cycles=8, keep=True,
                            sigma=3e-2, sigma_decay=0.5)
    srv = JKServer(incremental=True, loose_tight=True)
    srv.run(reqs)
    assert max(srv.batch_sizes) > 1
    for r in reqs:
        alone = serve_alone(r, incremental=True, loose_tight=True)
        for (mj, mk), (aj, ak) in zip(r.results, alone):
            assert np.abs(mj - aj).max() <= 1e-10
            assert np.abs(mk - ak).max() <= 1e-10
    st = srv.screen_stats
    assert st['loose_builds'] > 0 and st['tight_builds'] >= len(reqs)
    assert screen.ScreenPhase().loose == screen.LOOSE
