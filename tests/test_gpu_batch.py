"""Batched builds, CUDA-graph replay, sharded builds and the mixed-precision
form on the GPU, checked against single-molecule builds and the oracle.

Tolerances: 1e-10 absolute on every J/K element (the plain form's parity
bar) between a batched and a single build, and against the oracle; the
mixed form's J/K energies within 1e-7 Eh of the plain form's."""
import numpy as np
import pytest

from electrolites_b200 import clusters
from electrolites_b200.gto import Mole

pytestmark = pytest.mark.gpu

ATOL = 1e-10
ETOL_MIXED = 1e-7


@pytest.fixture(scope='module')
def torch():
    import torch
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    return torch


def spdf_mol():
    b = {
        'H': [[0, (1.3, 0.6), (0.3, 0.5)], [1, (0.9, 1.0)], [2, (0.7, 1.0)], [3, (0.6, 1.0)]],
        'C': [[0, (2.1, 1.0)], [1, (0.5, 1.0)], [2, (0.9, 0.5), (0.35, 0.6)], [3, (1.2, 1.0)]],
    }
    return Mole([('H', (0.0, 0.0, 0.0)), ('C', (-0.5, 1.1, 0.6))], basis=b, cart=True)


def batch_mols():
    """Uneven molecules: 1-5 waters in two bases, and an s/p/d/f pair."""
    mols = [clusters.water_mole(n, 3.1 * n ** (1 / 3), 100 + n, basis=b)
            for n, b in [(1, '6-31g*'), (3, 'def2-svp'), (2, '6-31g*'), (5, '6-31g*'),
                         (1, 'def2-svp'), (4, 'def2-svp')]]
    return mols + [spdf_mol()]


def dens_stack(mol, n_dm, hermi, seed):
    rng = np.random.default_rng(seed)
    D = clusters.atomic_density(mol, seed)
    out = np.stack([D + 1e-3 * np.abs(D).max() * rng.standard_normal(D.shape)
                    for _ in range(n_dm)])
    if hermi == 1:
        out = 0.5 * (out + out.transpose(0, 2, 1))
    elif hermi == 2:
        out = out - out.transpose(0, 2, 1)
    return out


@pytest.fixture(scope='module')
def opts(torch):
    from electrolites_b200.jk import VHFOpt
    mols = batch_mols()
    return mols, [VHFOpt(m, 1e-13).build() for m in mols]


def _single(torch, opts, dms, hermi, with_j=True, with_k=True, thr=0.0):
    out = []
    for o, d in zip(opts, dms):
        vj, vk = o.get_jk(d, hermi, with_j=with_j, with_k=with_k, mixed_threshold=thr)
        out.append((vj, vk))
    return out


def _maxdiff(a, b):
    return float((a - b).abs().max())


@pytest.mark.parametrize('hermi', [1, 0, 2])
def test_batch_matches_single_builds(torch, oracle, opts, hermi):
    from electrolites_b200.batch import JKBatch
    mols, plans = opts
    dms = [torch.as_tensor(dens_stack(m, 1 + i % 4, hermi, 7 + i), device='cuda')
           for i, m in enumerate(mols)]
    batch = JKBatch()
    vj, vk = batch.build(plans, dms, hermi)
    ref = _single(torch, plans, dms, hermi)
    for i in range(len(mols)):
        assert _maxdiff(vj[i], ref[i][0]) <= ATOL
        assert _maxdiff(vk[i], ref[i][1]) <= ATOL
    # two members against the oracle directly
    for i in (0, len(mols) - 1):
        rj, rk, _ = oracle.jk(mols[i], dms[i].cpu().numpy(), tol=1e-13)
        if hermi == 2:
            rj = np.zeros_like(rj)
        assert np.abs(vj[i].cpu().numpy() - rj).max() <= ATOL
        assert np.abs(vk[i].cpu().numpy() - rk).max() <= ATOL
    counts = batch.class_counts()
    assert sum(q for q, _ in counts.values()) > 0


def test_batch_j_only_and_k_only(torch, opts):
    from electrolites_b200.batch import JKBatch
    mols, plans = opts
    dms = [torch.as_tensor(dens_stack(m, 2, 1, 3 + i), device='cuda') for i, m in enumerate(mols)]
    batch = JKBatch()
    ref = _single(torch, plans, dms, 1)
    vj, vk = batch.build(plans, dms, 1, with_j=True, with_k=False)
    assert vk is None
    for i in range(len(mols)):
        assert _maxdiff(vj[i], ref[i][0]) <= ATOL
    vj, vk = batch.build(plans, dms, 1, with_j=False, with_k=True)
    assert vj is None
    for i in range(len(mols)):
        assert _maxdiff(vk[i], ref[i][1]) <= ATOL


def test_graph_capture_and_replay_with_new_densities(torch, opts):
    """The first use_graph call runs directly, the second captures, later
    calls replay; densities rewritten in place between calls give the
    results of single builds on the new values."""
    from electrolites_b200.batch import JKBatch
    mols, plans = opts
    dms = [torch.as_tensor(dens_stack(m, 1 + i % 3, 1, 20 + i), device='cuda')
           for i, m in enumerate(mols)]
    vj = [torch.empty_like(d) for d in dms]
    vk = [torch.empty_like(d) for d in dms]
    batch = JKBatch()
    seen = []
    for cycle in range(4):
        for i, m in enumerate(mols):
            dms[i].copy_(torch.as_tensor(dens_stack(m, dms[i].shape[0], 1, 40 + 7 * cycle + i)))
        batch.build(plans, dms, 1, vj=vj, vk=vk, use_graph=True)
        st = batch.stats()
        seen.append((st['graph_captured'], st['graph_replayed']))
        ref = _single(torch, plans, dms, 1)
        for i in range(len(mols)):
            assert _maxdiff(vj[i], ref[i][0]) <= ATOL
            assert _maxdiff(vk[i], ref[i][1]) <= ATOL
    assert seen == [(False, False), (True, False), (False, True), (False, True)]
    # a different parameter set recaptures
    batch.build(plans, dms, 1, vj=vj, vk=vk, use_graph=True, mixed_threshold=1e-9)
    assert batch.stats()['graph_captured']


def test_batch_range_error_names_the_molecule(torch):
    """A plan keeps the shell pairs that can pass the screening for |D| up
    to 1e6; a density far beyond that is reported with the molecule's index
    instead of silently losing quartets.  direct_scf_tol = 1 makes the plans
    drop pairs at these small sizes."""
    from electrolites_b200._lib import JKError
    from electrolites_b200.batch import JKBatch
    from electrolites_b200.jk import VHFOpt
    mols = [clusters.water_mole(1, 3.0, 1, basis='6-31g*'),
            clusters.water_mole(6, 9.0, 2, basis='6-31g*')]
    plans = [VHFOpt(m, 1.0).build() for m in mols]
    dms = [torch.as_tensor(dens_stack(m, 1, 1, 5), device='cuda') for m in mols]
    batch = JKBatch()
    batch.build(plans, dms, 1)
    dms[1] = dms[1] * 1e9
    with pytest.raises(JKError, match='item 1'):
        batch.build(plans, dms, 1)
    # the flag is cleared: the next build works
    dms[1] = dms[1] * 1e-9
    batch.build(plans, dms, 1)


@pytest.mark.parametrize('size', [2, 3])
def test_shards_sum_to_the_full_build(torch, opts, size):
    """Tasks t = rank + size * n per rank: the sum over ranks is the whole
    build (each rank's build runs alone here; no kernel waits on another)."""
    mols, plans = opts
    o = plans[3]
    d = torch.as_tensor(dens_stack(mols[3], 2, 0, 9), device='cuda')
    fj, fk = o.get_jk(d, 0)
    sj, sk = torch.zeros_like(fj), torch.zeros_like(fk)
    parts = []
    for r in range(size):
        o.set_shard(r, size)
        vj, vk = o.get_jk(d, 0)
        sj += vj
        sk += vk
        parts.append(float(vk.abs().max()))
    o.set_shard(0, 1)
    assert all(p > 0 for p in parts)
    assert _maxdiff(sj, fj) <= ATOL and _maxdiff(sk, fk) <= ATOL


def test_mixed_precision_error_and_batch(torch):
    """(H2O)_8 in 6-31G*: the mixed form's J/K energies stay within 1e-7 Eh
    of the plain form's at thresholds 1e-6..1e-10, FP32 quartets are used,
    and a batched mixed build equals the single mixed builds."""
    from electrolites_b200.batch import JKBatch
    from electrolites_b200.jk import VHFOpt
    mol = clusters.water_mole(8, 7.0, 0, basis='6-31g*')
    o = VHFOpt(mol, 1e-13).build()
    D = torch.as_tensor(dens_stack(mol, 2, 1, 1), device='cuda')
    pj, pk = o.get_jk(D, 1)
    ej = 0.5 * float((D * pj).sum())
    ek = -0.25 * float((D * pk).sum())
    n32 = []
    for thr in (1e-6, 1e-8, 1e-10):
        mj, mk = o.get_jk(D, 1, mixed_threshold=thr)
        n32.append(sum(c[2] for c in o.class_counts(with_f32=True).values()))
        assert abs(0.5 * float((D * mj).sum()) - ej) <= ETOL_MIXED
        assert abs(-0.25 * float((D * mk).sum()) - ek) <= ETOL_MIXED
    assert n32[0] >= n32[1] >= n32[2] and n32[0] > 0
    mj, mk = o.get_jk(D, 1, mixed_threshold=1e-6)
    bj, bk = JKBatch().build([o, o], [D, D.clone()], 1, mixed_threshold=1e-6)
    for v in (bj[0], bj[1]):
        assert _maxdiff(v, mj) <= ATOL
    for v in (bk[0], bk[1]):
        assert _maxdiff(v, mk) <= ATOL


def test_split_screening_matches_separate_j_and_k_builds(torch, opts):
    """J and K terms of a quartet are screened by their own tests, so a J+K
    build gives the J of a J-only build and the K of a K-only build."""
    mols, plans = opts
    o = plans[3]
    d = torch.as_tensor(dens_stack(mols[3], 2, 1, 13), device='cuda')
    vj, vk = o.get_jk(d, 1)
    j_only, _ = o.get_jk(d, 1, with_j=True, with_k=False)
    _, k_only = o.get_jk(d, 1, with_j=False, with_k=True)
    assert _maxdiff(vj, j_only) <= 1e-12
    assert _maxdiff(vk, k_only) <= 1e-12


def test_one_or_two_class_streams_agree(torch, opts):
    """Per-class timing runs every class kernel on one stream; the default
    spreads them over two.  Both give the same J/K."""
    mols, plans = opts
    o = plans[5]
    d = torch.as_tensor(dens_stack(mols[5], 3, 0, 17), device='cuda')
    a = o.get_jk(d, 0)
    o.set_timing(True)
    b = o.get_jk(d, 0)
    ms, launches = o.last_class_ms()
    o.set_timing(False)
    assert ms and launches > 0
    assert _maxdiff(a[0], b[0]) <= 1e-12 and _maxdiff(a[1], b[1]) <= 1e-12


def test_grouped_tasks_split_and_single_view_launch(torch):
    """Batched register-form tasks cover a bra pair's candidates over all its
    ket sub-lists.  A (H2O)_12 member with the smallest task size splits
    those ranges over several tasks; 193 molecules put 193 views in every
    class, so each class's second launch holds one view and still runs the
    batched (grouped) kernel.  Both equal one build per molecule (1e-10)."""
    from electrolites_b200.batch import JKBatch
    from electrolites_b200.jk import VHFOpt, class_keys
    mols = [clusters.water_mole(12, 8.0, 31, basis='6-31g*'),
            clusters.water_mole(1, 3.0, 32, basis='6-31g*'),
            clusters.water_mole(3, 4.5, 33, basis='def2-svp')]
    plans = [VHFOpt(m, 1e-13).build() for m in mols]
    dms = [torch.as_tensor(dens_stack(m, 2, 1, 40 + i), device='cuda') for i, m in enumerate(mols)]
    batch = JKBatch()
    for c in range(len(class_keys())):
        batch.set_tuning(c, 4096)          # many tasks: the smallest task size
    vj, vk = batch.build(plans, dms, 1)
    ref = _single(torch, plans, dms, 1)
    for i in range(len(mols)):
        assert _maxdiff(vj[i], ref[i][0]) <= ATOL
        assert _maxdiff(vk[i], ref[i][1]) <= ATOL
    mols = [clusters.water_mole(1, 3.0, 100 + i, basis='6-31g*') for i in range(193)]
    plans = [VHFOpt(m, 1e-13).build() for m in mols]
    dms = [torch.as_tensor(dens_stack(m, 1, 1, i), device='cuda') for i, m in enumerate(mols)]
    vj, vk = JKBatch().build(plans, dms, 1)
    for i in (0, 100, 191, 192):
        rj, rk = plans[i].get_jk(dms[i], 1)
        assert _maxdiff(vj[i], rj) <= ATOL and _maxdiff(vk[i], rk) <= ATOL
