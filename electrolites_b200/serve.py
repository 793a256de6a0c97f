"""Serving J/K builds with continuous batching.

A request is one molecule with 1-4 densities that needs J/K for a number of
SCF-like cycles (each cycle: a J/K build of the current densities, then the
densities move on).  The server keeps, per admitted request, its plan (pair
and screening tables) and its density / J / K buffers resident on the
device across all of its cycles, and runs every admitted request's next
cycle together in one batched build (electrolites_b200.batch.JKBatch):

  * admission: a request that has arrived waits until its device memory
    (estimated from its size before its plan exists, exact afterwards) fits
    the HBM budget next to the requests already admitted, and a slot is
    free;
  * each iteration launches one batched build over all admitted requests
    (asynchronously), admits new arrivals -- building their plans on the
    host and on a private stream -- while the device works, then waits,
    hands each request its J/K, advances its densities and retires the
    requests that finished their cycles, freeing their memory;
  * requests that arrive while others are on the device join at the next
    iteration (continuous batching), so their work shares the device with
    the requests already in flight;
  * incremental mode (optional): J and K are linear in the density, so a
    cycle after the first builds J/K of the change Delta D = D - D_prev and
    adds them to the previous J/K; the change is small (1e-4 of D per cycle
    here), so the density-weighted screening drops most quartets.  Every
    `rebuild_every`-th cycle is a full build, which bounds the drift from
    terms the screening dropped;
  * loose-then-tight screening (optional, with incremental mode): each
    request follows the schedule of electrolites_b200.screen.ScreenPhase
    (the reference's electrolites/fastscfscreen.py) in place of the
    periodic rebuilds: incremental builds at a loose threshold while its
    density step is large, one tight rebuild at the switch, tight increments
    after it.  Requests in different phases share one batched build (each
    plan screens at its own threshold).

Latency of a request = completion of its last cycle - its arrival.  The
reference has no serving layer; this sits on top of the same J/K call the
reference patches (electrolites/fastjk.py:276).
"""
from __future__ import annotations

import collections
import dataclasses
import time

import numpy as np

from . import screen
from .batch import JKBatch
from .jk import VHFOpt


def _torch():
    import torch
    return torch


@dataclasses.dataclass
class Request:
    rid: int
    mol: object                    # electrolites_b200.gto.Mole (or PySCF Mole)
    dms: np.ndarray                # (n_dm, nao, nao) Cartesian, first cycle
    cycles: int = 10
    sigma: float = 1e-4            # per-cycle symmetric perturbation, relative to max|D|
    sigma_decay: float = 1.0       # the perturbation of cycle c is sigma * sigma_decay**c
    arrival: float = 0.0           # seconds after the start of the run
    seed: int = 0
    keep: bool = False             # keep every cycle's (vj, vk) on the host
    # filled by the server
    admitted: float = None
    finished: float = None
    done_cycles: int = 0
    energies: list = dataclasses.field(default_factory=list)
    results: list = dataclasses.field(default_factory=list)


def matrix_bytes(nao: int, nbas: int, n_dm: int, incremental: bool = False) -> int:
    """Device bytes of a request's matrices: densities, J, K, and its share
    of the build workspace (half-J/K accumulators, symmetrised densities,
    the pair-interleaved copy of the K densities, screening table) for
    hermi = 1; incremental mode keeps four more (the previous density, the
    density change, accumulated J and K)."""
    return 8 * nao * nao * n_dm * (3 + 4 + (4 if incremental else 0)) + 4 * nbas * nbas


def table_bound(nbas: int) -> int:
    """Upper estimate of a plan's pair tables before it exists: nbas^2/2
    pairs of 40-byte records with 9 primitive pairs of 80 bytes each."""
    return nbas * nbas // 2 * (40 + 9 * 80)


def advance_density(d, sigma, gen):
    """D <- D + symmetric Gaussian noise of std sigma * max|D|, on the
    device and without a host synchronisation."""
    torch = _torch()
    noise = torch.randn(d.shape, generator=gen, dtype=d.dtype, device=d.device)
    noise = (noise + noise.transpose(-1, -2)) * (d.abs().amax() * (sigma / 2 ** 0.5))
    d.add_(noise)


class _Active:
    __slots__ = ('req', 'opt', 'dms', 'vj', 'vk', 'gen', 'bytes', 'prev', 'delta', 'jacc', 'kacc',
                 'inc', 'screen')

    def j(self):
        return self.jacc if self.jacc is not None else self.vj

    def k(self):
        return self.kacc if self.kacc is not None else self.vk


class JKServer:
    """Continuous-batching J/K server on one device."""

    def __init__(self, device: int | None = None, hbm_budget: float = 0.5,
                 max_active: int = 512, mixed_threshold: float = 0.0, tol: float = 1e-13,
                 use_graph: bool = False, incremental: bool = False, rebuild_every: int = 5,
                 loose_tight: bool = False, loose: float = screen.LOOSE,
                 switch: float = screen.SWITCH, max_loose: int = screen.MAX_LOOSE):
        torch = _torch()
        self.device = torch.cuda.current_device() if device is None else int(device)
        self.dev = torch.device('cuda', self.device)
        free, total = torch.cuda.mem_get_info(self.dev)
        # budget: a fraction of the device's memory (<= 1) or bytes (> 1)
        self.budget = int(hbm_budget * total) if hbm_budget <= 1 else int(hbm_budget)
        self.max_active = max_active
        self.mixed_threshold = mixed_threshold
        self.tol = tol
        self.use_graph = use_graph
        self.incremental = incremental
        self.rebuild_every = max(1, int(rebuild_every))
        if loose_tight and not incremental:
            raise ValueError('loose-then-tight screening needs incremental mode')
        self.loose_tight = loose_tight
        self.screen_args = (loose, switch, max_loose)
        self.batch = JKBatch(self.device)
        self.stream = torch.cuda.Stream(self.dev)         # batched builds, density updates
        self.admit_stream = torch.cuda.Stream(self.dev)   # uploads of admitted requests
        self.queue = collections.deque()
        self.active = []
        self.used = 0
        self.iterations = 0
        self.batch_sizes = []
        self.screen_stats = {'loose_builds': 0, 'rebuilds': 0, 'tight_builds': 0, 'capped': 0}

    # ------------------------------------------------------------------
    def _admit(self, now):
        """Admit arrived requests in arrival order while memory and slots allow."""
        torch = _torch()
        while self.queue and len(self.active) < self.max_active:
            req = self.queue[0]
            if req.arrival > now:
                break
            n_dm, nao = req.dms.shape[0], req.dms.shape[-1]
            mats = matrix_bytes(nao, req.mol.nbas, n_dm, self.incremental)
            need = mats + table_bound(req.mol.nbas)
            if self.active and self.used + need > self.budget:
                break                                   # wait for memory to free up
            self.queue.popleft()
            a = _Active()
            a.req = req
            # the upload runs on its own stream: a pageable copy waits for
            # its stream's earlier work, which must not be the running build
            a.opt = VHFOpt(req.mol, self.tol, device=self.device).build()
            with torch.cuda.stream(self.admit_stream):
                a.dms = torch.as_tensor(req.dms, device=self.dev).contiguous()
                a.vj = torch.empty_like(a.dms)
                a.vk = torch.empty_like(a.dms)
                a.prev = a.delta = a.jacc = a.kacc = None
                if self.incremental:
                    a.prev = torch.empty_like(a.dms)
                    a.delta = torch.empty_like(a.dms)
                    a.jacc = torch.empty_like(a.dms)
                    a.kacc = torch.empty_like(a.dms)
            a.inc = False
            a.screen = screen.ScreenPhase(*self.screen_args) if self.loose_tight else None
            a.gen = torch.Generator(device=self.dev)
            a.gen.manual_seed(req.seed)
            tables, _ = a.opt.memory()
            a.bytes = mats + tables
            self.used += a.bytes
            req.admitted = now
            self.active.append(a)

    def _inputs(self):
        """This cycle's build input per active request: its density, or in
        incremental mode the change since its previous cycle."""
        torch = _torch()
        out = []
        with torch.cuda.stream(self.stream):
            for a in self.active:
                if a.screen is not None:
                    d = a.screen.decide(a.req.done_cycles > 0,
                                        lambda: screen.density_step(a.dms, a.prev))
                    a.inc = d in (screen.LOOSE_INC, screen.TIGHT_INC)
                    a.opt.direct_scf_tol = a.screen.tol(d, self.tol)
                else:
                    a.inc = self.incremental and a.req.done_cycles % self.rebuild_every != 0
                if a.inc:
                    torch.sub(a.dms, a.prev, out=a.delta)
                    out.append(a.delta)
                else:
                    out.append(a.dms)
        return out

    def _finish_cycle(self, now):
        torch = _torch()
        still = []
        with torch.cuda.stream(self.stream):
            for a in self.active:
                if self.incremental:
                    if a.inc:
                        a.jacc.add_(a.vj)
                        a.kacc.add_(a.vk)
                    else:
                        a.jacc.copy_(a.vj)
                        a.kacc.copy_(a.vk)
                    a.prev.copy_(a.dms)
            e = torch.stack([torch.stack([0.5 * (a.dms * a.j()).sum(), -0.25 * (a.dms * a.k()).sum()])
                             for a in self.active]).cpu().numpy()
        for i, a in enumerate(self.active):
            req = a.req
            req.energies.append((float(e[i, 0]), float(e[i, 1])))
            if req.keep:
                req.results.append((a.j().cpu().numpy(), a.k().cpu().numpy()))
            req.done_cycles += 1
            if req.done_cycles >= req.cycles:
                req.finished = now
                self.used -= a.bytes
                if a.screen is not None:
                    for key, v in a.screen.stats.items():
                        self.screen_stats[key] += v
                continue
            with torch.cuda.stream(self.stream):
                advance_density(a.dms, req.sigma * req.sigma_decay ** (req.done_cycles - 1), a.gen)
            still.append(a)
        self.active = still

    def run(self, requests, clock=None):
        """Serve `requests` (arrival times in seconds from now); returns them
        with latencies filled in.  clock: a function returning seconds
        (time.perf_counter by default)."""
        torch = _torch()
        clock = clock or time.perf_counter
        self.queue = collections.deque(sorted(requests, key=lambda r: r.arrival))
        t0 = clock()
        with torch.cuda.device(self.dev):
            while self.queue or self.active:
                now = clock() - t0
                if not self.active:
                    self._admit(now)
                    if not self.active:
                        wait = self.queue[0].arrival - now
                        if wait > 0:
                            time.sleep(min(wait, 0.05))
                        continue
                opts = [a.opt for a in self.active]
                self.stream.wait_stream(self.admit_stream)
                self.batch.build_async(opts, self._inputs(), 1, True, True,
                                       [a.vj for a in self.active], [a.vk for a in self.active],
                                       self.mixed_threshold, self.use_graph, self.stream)
                self.batch_sizes.append(len(opts))
                self.iterations += 1
                n_before = len(self.active)
                self._admit(clock() - t0)          # overlaps with the device work
                newly = self.active[n_before:]
                self.active = self.active[:n_before]
                self.batch.sync(self.stream)
                self._finish_cycle(clock() - t0)
                self.active += newly
        return requests


def latency_stats(requests):
    """{'p50_ms', 'p99_ms', 'mean_ms', 'mols_per_s'} of served requests."""
    lat = np.array([r.finished - r.arrival for r in requests])
    span = max(r.finished for r in requests) - min(r.arrival for r in requests)
    return {'p50_ms': float(np.percentile(lat, 50) * 1e3),
            'p99_ms': float(np.percentile(lat, 99) * 1e3),
            'mean_ms': float(lat.mean() * 1e3),
            'mols_per_s': len(requests) / span if span > 0 else float('inf')}


def poisson_requests(n: int, rate: float, seed: int, n_min: int = 3, n_max: int = 60,
                     bases=('6-31g*', 'def2-svp'), cycles: int = 10, sigma: float = 1e-4,
                     keep: bool = False, sigma_decay: float = 1.0):
    """n requests with exponential inter-arrival times (rate per second):
    water clusters of n_min..n_max waters (cube edge 3.1 n^(1/3) A), a basis
    drawn from `bases`, 1-4 densities."""
    from . import clusters
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(n):
        t += rng.exponential(1.0 / rate)
        nw = int(rng.integers(n_min, n_max + 1))
        k = int(rng.integers(1, 5))
        basis = bases[int(rng.integers(0, len(bases)))]
        s = seed * 10000 + i
        mol = clusters.water_mole(nw, 3.1 * nw ** (1.0 / 3.0), s, basis=basis)
        dms = clusters.density_stack(clusters.atomic_density(mol, s), k, s + 1)
        out.append(Request(rid=i, mol=mol, dms=dms, cycles=cycles, sigma=sigma, arrival=t,
                           seed=s, keep=keep, sigma_decay=sigma_decay))
    return out


def serve_alone(req: Request, device: int | None = None, mixed_threshold: float = 0.0,
                tol: float = 1e-13, incremental: bool = False, rebuild_every: int = 5,
                loose_tight: bool = False, loose: float = screen.LOOSE,
                switch: float = screen.SWITCH, max_loose: int = screen.MAX_LOOSE):
    """The same request served by itself: one build per cycle on its own
    plan, the same density updates (and the same incremental or
    loose-then-tight schedule).  Returns [(vj, vk), ...] per cycle."""
    torch = _torch()
    dev = torch.device('cuda', torch.cuda.current_device() if device is None else device)
    opt = VHFOpt(req.mol, tol, device=dev.index).build()
    d = torch.as_tensor(req.dms, device=dev).contiguous()
    gen = torch.Generator(device=dev)
    gen.manual_seed(req.seed)
    lt = (screen.LooseTightJK(opt, None, loose, switch, max_loose, mixed_threshold)
          if loose_tight else None)
    out = []
    prev = jacc = kacc = None
    for c in range(req.cycles):
        if lt is not None:
            jacc, kacc = lt.jk(d)
        elif incremental and c % max(1, int(rebuild_every)) != 0:
            vj, vk = opt.get_jk(d - prev, 1, mixed_threshold=mixed_threshold)
            jacc, kacc = jacc + vj, kacc + vk
        else:
            jacc, kacc = opt.get_jk(d, 1, mixed_threshold=mixed_threshold)
        prev = d.clone()
        out.append((jacc.cpu().numpy(), kacc.cpu().numpy()))
        if c + 1 < req.cycles:
            advance_density(d, req.sigma * req.sigma_decay ** c, gen)
    return out
