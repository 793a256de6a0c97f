"""The sharded (multi-GPU) build's host side on CPU ranks: world size 2 and
3 over gloo, each rank's engine replaced by the oracle restricted to the
rank's share of the bra shell pairs.  The all-reduced vj / vk equal the
unsharded oracle build on every rank; a rank that dies before the exchange
makes the others fail with an error instead of waiting forever (host-side
fault injection)."""
import datetime
import os
import socket

import numpy as np
import pytest

TIMEOUT_S = 20


def _free_port():
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        return s.getsockname()[1]


def _inputs():
    from electrolites_b200 import clusters
    mol = clusters.water_mole(2, 4.0, 3, basis='6-31g*')
    dms = clusters.density_stack(clusters.atomic_density(mol, 4), 2, 5)
    return mol, dms


class OracleShard:
    """Stands in for a VHFOpt on a CPU rank: a 'build' is the oracle J/K over
    the bra shell pairs p with p % size == rank."""

    def __init__(self, mol):
        self.mol = mol
        self.rank, self.size = 0, 1

    def set_shard(self, rank, size):
        self.rank, self.size = rank, size

    def build_jk_async(self, dms, hermi, with_j, with_k, vj, vk, mixed_threshold=0.0,
                       stream=None):
        import torch

        from oracle import oracle as O
        nb = self.mol.nbas
        pairs = np.arange(self.rank, nb * (nb + 1) // 2, self.size)
        rj, rk, _ = O.jk_sample(self.mol, dms.numpy(), pairs, tol=1e-13)
        if with_j:
            vj.copy_(torch.as_tensor(rj))
        if with_k:
            vk.copy_(torch.as_tensor(rk))

    def sync(self, stream=None):
        pass


def _worker(rank, size, port, queue, die_rank):
    import torch
    import torch.distributed as dist

    from electrolites_b200.shard import ShardedJK
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    dist.init_process_group('gloo', rank=rank, world_size=size,
                            timeout=datetime.timedelta(seconds=TIMEOUT_S))
    try:
        mol, dms = _inputs()
        sj = ShardedJK(OracleShard(mol))
        if rank == die_rank:
            os._exit(3)                       # the injected failure: gone before the exchange
        vj, vk = sj.get_jk(torch.as_tensor(dms), 1)
        queue.put((rank, 'ok', vj.numpy(), vk.numpy()))
    except Exception as e:                    # noqa: BLE001 - reported to the test
        queue.put((rank, 'error', repr(e), None))
    finally:
        try:
            dist.destroy_process_group()
        except Exception:
            pass


def _run(size, die_rank=-1):
    import multiprocessing as mp
    ctx = mp.get_context('spawn')
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, size, port, q, die_rank)) for r in range(size)]
    for p in procs:
        p.start()
    out = {}
    expect = size - (1 if die_rank >= 0 else 0)
    for _ in range(expect):
        r, status, a, b = q.get(timeout=3 * TIMEOUT_S + 60)
        out[r] = (status, a, b)
    for p in procs:
        p.join(TIMEOUT_S + 30)
        if p.is_alive():
            p.kill()
    return out


@pytest.mark.parametrize('size', [2, 3])
def test_sharded_build_sums_to_full(oracle, size):
    mol, dms = _inputs()
    rj, rk, _ = oracle.jk(mol, dms, tol=1e-13)
    out = _run(size)
    assert sorted(out) == list(range(size))
    for r, (status, vj, vk) in out.items():
        assert status == 'ok', vj
        assert np.abs(vj - rj).max() <= 1e-12
        assert np.abs(vk - rk).max() <= 1e-12


def test_dead_rank_fails_the_exchange(oracle):
    out = _run(2, die_rank=1)
    assert list(out) == [0]
    status, msg, _ = out[0]
    assert status == 'error', 'the surviving rank must not return a partial result'
