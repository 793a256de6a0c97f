#!/usr/bin/env python
"""Benchmark of the direct-SCF J/K build on B200.

Workload (default): (H2O)_96, rigid waters in a 15 A cube (seed 20261204),
6-31G* shell structure (synthetic exponents, see
electrolites_b200/basis_synth.py), Cartesian AOs, UHF density pair
D_alpha = D_atom/2, D_beta = D_alpha + symmetric Gaussian noise
(sigma = 1e-3 max|D_alpha|), hermi = 1, J and K, direct_scf_tol 1e-13,
plain all-FP64 form.  One step = one J/K build of both densities.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload NAME] [--mixed THRESHOLD]

Prints one JSON line (rank 0).  value = J/K builds per second of the whole
job (device-timed with CUDA events, densities resident in HBM); e2e = the
same through jk_build_host from pinned host buffers, copies included.  With
N > 1 ranks (torchrun, one GPU each) the build is sharded: every rank
evaluates the tasks rank, rank + N, ... of each class launch and one NCCL
all-reduce of the (vj, vk) buffer completes the build on every rank (strong
scaling: one build per step for the whole job); timing is the max over
ranks.  The default run also reports the plain-vs-mixed threshold sweep
(1e-10..1e-6) on this workload and on (H2O)_64 def2-TZVP, the uneven
512-molecule batch (one build per molecule vs batched FP64 vs batched
mixed) and a serving run.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    # name: (waters, cube edge A, basis, UHF pair, seed)
    'h2o96_631gs_uhf': (96, 15.0, '6-31g*', True, 20261204),
    'h2o8_631gs': (8, 7.0, '6-31g*', False, 20261203),
    'h2o32_631gs_uhf': (32, 10.4, '6-31g*', True, 20261204),
    'h2o64_tzvp': (64, 12.5, 'def2-tzvp', False, 20261205),
    'h2o16_tzvp': (16, 7.8, 'def2-tzvp', False, 20261205),
}
DEFAULT = 'h2o96_631gs_uhf'
TOL = 1e-13
L2_FLUSH_BYTES = 256 << 20      # > 126 MB L2


def make_inputs(name):
    import numpy as np
    from electrolites_b200 import clusters
    n, edge, basis, uhf, seed = WORKLOADS[name]
    mol = clusters.water_mole(n, edge, seed, basis=basis, cart=True)
    D = clusters.atomic_density(mol, seed)
    dms = clusters.uhf_pair(D, seed + 1) if uhf else D[None]
    return mol, np.ascontiguousarray(dms)


class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""
    FIELDS = ('index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,'
              'clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,'
              'clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap')

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix='.csv')
            os.close(fd)
            self.f = open(self.path, 'w')
            self.proc = subprocess.Popen(
                ['nvidia-smi', f'--query-gpu={self.FIELDS}', '--format=csv,noheader,nounits',
                 '-lms', '200', '-i', str(self.device)], stdout=self.f,
                stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(5)
        except Exception:
            self.proc.kill()
        self.f.close()
        rows = [r.split(',') for r in open(self.path).read().strip().splitlines() if r]
        os.unlink(self.path)
        sm, smax, reasons = [], 0.0, set()
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap']
        for r in rows:
            try:
                sm.append(float(r[1]))
                smax = max(smax, float(r[2]))
                for nm, v in zip(names, r[5:9]):
                    if 'Active' in v and 'Not' not in v:
                        reasons.add(nm)
            except (ValueError, IndexError):
                continue
        if not sm:
            return None
        return {'sm_mhz': statistics.median(sm), 'sm_max_mhz': smax,
                'reasons': sorted(reasons), 'samples': len(sm)}


def cpu_sample(mol, dms, budget_s=15.0, nthreads=0, seed=1):
    """Oracle J/K on a random sample of bra shell pairs, scaled to a full
    build: returns (builds/s, threads, description)."""
    import numpy as np
    from oracle import oracle as O
    nthreads = nthreads or os.cpu_count() or 1
    npair = mol.nbas * (mol.nbas + 1) // 2
    rng = np.random.default_rng(seed)
    n, spent, nq_tot, used = 8, 0.0, 0, 0
    while spent < budget_s and used < npair:
        take = rng.choice(npair, size=min(n, npair - used), replace=False)
        t0 = time.perf_counter()
        _, _, nq = O.jk_sample(mol, dms, take, tol=TOL, nthreads=nthreads)
        spent += time.perf_counter() - t0
        used += len(take)
        nq_tot += nq
        n = max(8, int(n * min(4.0, max(1.5, budget_s / max(spent, 1e-3) / 2))))
    t_full = spent * npair / used
    desc = (f'{used} of {npair} bra shell pairs drawn uniformly (seed {seed}), all '
            f'their kets, {nq_tot} quartets in {spent:.1f} s; time scaled by '
            f'{npair / used:.1f} to a full build')
    return 1.0 / t_full, nthreads, desc


def run_reference(args, rank):
    if rank != 0:
        return
    mol, dms = make_inputs(args.workload)
    vals = []
    threads, desc = os.cpu_count(), ''
    for it in range(args.warmup + args.steps):
        v, threads, desc = cpu_sample(mol, dms, budget_s=min(20.0, 60.0 / max(1, args.steps)),
                                      seed=1 + it)
        if it >= args.warmup:
            vals.append(v)
    v = statistics.mean(vals)
    line = {'impl': 'reference', 'metric': 'jk_builds_per_s', 'value': v,
            'unit': 'builds/s', 'n_gpus': args.gpus, 'steps': args.steps,
            'warmup': args.warmup, 'ms_per_step': 1e3 / v, 'higher_is_better': True,
            'scaling': 'strong', 'vs_baseline': None, 'dtype': 'f64', 'data': 'synthetic',
            'config': {'workload': args.workload, 'hermi': 1, 'direct_scf_tol': TOL,
                       'form': 'plain'},
            'cpu_baseline': {'value': v, 'unit': 'builds/s', 'cores': threads,
                             'kind': 'port', 'sample': desc},
            'e2e': {'value': v, 'unit': 'builds/s', 'h2d_bytes_per_step': 0,
                    'd2h_bytes_per_step': 0}}
    print(json.dumps(line), flush=True)


BATCH_SEED = 20261206
BATCH_MOLS = 512
BATCH_MIXED = 1e-6


def _timed(fn, steps, warmup, stream, flush):
    """Device ms per call of fn(): CUDA events on `stream`, L2 flushed
    (untimed) before each timed call."""
    import torch
    for _ in range(max(3, warmup)):
        fn()
    torch.cuda.synchronize()
    total = 0.0
    for _ in range(steps):
        flush.zero_()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(stream)
        fn()
        e.record(stream)
        e.synchronize()
        total += s.elapsed_time(e)
    return total / steps


def run_batch(args, dev, stream, flush, peak_tflops):
    """Uneven batch: 512 water clusters (n ~ U{1..24}, cube 3.1 n^(1/3) A,
    6-31G*, 1-4 densities each, seed 20261206).  Times the plain FP64 form
    as one build per molecule, and the batched form (one launch stream for
    all molecules, replayed from a CUDA graph) in FP64 and mixed precision;
    reports molecule-builds per second and the mixed form's largest J/K
    energy error against the plain one."""
    import torch

    from electrolites_b200 import clusters, flop_model
    from electrolites_b200.batch import JKBatch
    from electrolites_b200.jk import VHFOpt
    t0 = time.perf_counter()
    items = clusters.uneven_batch(BATCH_MOLS, BATCH_SEED)
    opts = [VHFOpt(m, TOL, device=dev.index).build() for m, _ in items]
    dms = [torch.as_tensor(d, device=dev) for _, d in items]
    setup_s = time.perf_counter() - t0
    vj = [torch.empty_like(d) for d in dms]
    vk = [torch.empty_like(d) for d in dms]
    bj = [torch.empty_like(d) for d in dms]
    bk = [torch.empty_like(d) for d in dms]
    batch = JKBatch(dev.index)

    def seq():
        for o, d, j, k in zip(opts, dms, vj, vk):
            o.build_jk_async(d, 1, True, True, j, k, 0.0, stream)

    def bat(thr):
        return lambda: batch.build_async(opts, dms, 1, True, True, bj, bk, thr, True, stream)

    steps, warm = max(2, min(args.steps, 3)), args.warmup
    ms_plain = _timed(seq, steps, warm, stream, flush)
    for o in opts:
        o.sync(stream)
    ej = torch.stack([0.5 * (d * j).sum() for d, j in zip(dms, vj)])
    ek = torch.stack([-0.25 * (d * k).sum() for d, k in zip(dms, vk)])
    ms_b64 = _timed(bat(0.0), steps, warm, stream, flush)
    batch.sync(stream)
    counts = batch.class_counts()
    err64 = max(float((torch.stack([0.5 * (d * j).sum() for d, j in zip(dms, bj)]) - ej).abs().max()),
                float((torch.stack([-0.25 * (d * k).sum() for d, k in zip(dms, bk)]) - ek).abs().max()))
    ms_mix = _timed(bat(BATCH_MIXED), steps, warm, stream, flush)
    batch.sync(stream)
    st = batch.stats()
    c32 = batch.class_counts(with_f32=True)
    errj = float((torch.stack([0.5 * (d * j).sum() for d, j in zip(dms, bj)]) - ej).abs().max())
    errk = float((torch.stack([-0.25 * (d * k).sum() for d, k in zip(dms, bk)]) - ek).abs().max())
    _, launches = batch.last_class_ms()
    # algorithmic flops of the batch: the model per molecule needs per-molecule
    # counts, so the class totals are used with the mean density count
    n_dm = sum(d.shape[0] for d in dms)
    flops = flop_model.build_flops(counts, n_dm / len(dms), n_dm / len(dms))
    nq = sum(v[0] for v in counts.values())
    nq32 = sum(v[2] for v in c32.values())
    return {
        'workload': f'batch{BATCH_MOLS}_631gs', 'molecules': BATCH_MOLS, 'densities': n_dm,
        'nao_cart_mean': sum(o.nao for o in opts) / len(opts),
        'nao_cart_max': max(o.nao for o in opts), 'setup_s': round(setup_s, 1),
        'steps': steps, 'quartets': nq,
        'plain_ms': ms_plain, 'plain_mol_builds_per_s': BATCH_MOLS * 1e3 / ms_plain,
        'batched_fp64_ms': ms_b64, 'batched_fp64_mol_builds_per_s': BATCH_MOLS * 1e3 / ms_b64,
        'batched_fp64_energy_err': err64,
        'batched_mixed_ms': ms_mix, 'batched_mixed_mol_builds_per_s': BATCH_MOLS * 1e3 / ms_mix,
        'mixed_threshold': BATCH_MIXED, 'mixed_fp32_quartet_frac': nq32 / max(1, nq),
        'mixed_energy_err_j': errj, 'mixed_energy_err_k': errk,
        'speedup_batched_fp64_vs_plain': ms_plain / ms_b64,
        'speedup_batched_mixed_vs_plain': ms_plain / ms_mix,
        'batched_fp64_tflops_model': flops / (ms_b64 * 1e-3) / 1e12,
        'batched_fp64_peak_frac': flops / (ms_b64 * 1e-3) / 1e12 / peak_tflops,
        'graph_replayed': st['graph_replayed'], 'launches_per_build': launches,
    }


SERVE_SEED = 20261207
MIXED_SWEEP = (1e-10, 1e-8, 1e-7, 1e-6)
MIXED_WORKLOADS = ('h2o96_631gs_uhf', 'h2o64_tzvp')


def run_mixed(args, dev, stream, flush):
    """Plain FP64 against the mixed form at each threshold of the sweep, on
    the (H2O)_96 6-31G* UHF pair and (H2O)_64 def2-TZVP: device ms per build,
    the fraction of quartets run in FP32, and the J/K energy and largest
    element errors against the plain build (E_J = 1/2 tr(D J),
    E_K = -1/4 tr(D K) summed over the densities)."""
    import torch

    from electrolites_b200.jk import VHFOpt
    out = {}
    for w in MIXED_WORKLOADS:
        mol, dms_h = make_inputs(w)
        opt = VHFOpt(mol, TOL, device=dev.index).build()
        dms = torch.as_tensor(dms_h, device=dev)
        res = {}
        for thr in (0.0,) + MIXED_SWEEP:
            vj = torch.empty_like(dms)
            vk = torch.empty_like(dms)
            ms = _timed(lambda: opt.build_jk_async(dms, 1, True, True, vj, vk, thr, stream),
                        2, 1, stream, flush)
            opt.sync(stream)
            c = opt.class_counts(with_f32=True)
            nq = sum(v[0] for v in c.values())
            n32 = sum(v[2] for v in c.values())
            ej = float(0.5 * (dms * vj).sum())
            ek = float(-0.25 * (dms * vk).sum())
            res[thr] = (ms, n32 / max(1, nq), ej, ek, vj, vk)
        p = res[0.0]
        row = {'nao_cart': mol.nao_cart, 'n_dm': int(dms.shape[0]), 'plain_ms': round(p[0], 2),
               'thresholds': {}}
        for thr in MIXED_SWEEP:
            m = res[thr]
            row['thresholds'][f'{thr:g}'] = {
                'ms': round(m[0], 2), 'speedup': round(p[0] / m[0], 3),
                'fp32_quartet_frac': round(m[1], 3),
                'dE_J': m[2] - p[2], 'dE_K': m[3] - p[3],
                'max_dJ': float((m[4] - p[4]).abs().max()),
                'max_dK': float((m[5] - p[5]).abs().max())}
        out[w] = row
    return out


RSH_OMEGA, RSH_LR, RSH_SR = 0.3, 1.0, 0.157706   # an omega-B97X-type exchange mixture


def run_rsh(args, dev, stream, flush, opt, dms):
    """Range-separated exchange lr K_erf(w) + sr K_erfc(w) on the main
    workload (K only, the reference's get_k_rsh): one fused build of
    sr K_full + (lr - sr) K_lr against the two one-term builds it replaces;
    device ms per K and the largest element difference."""
    import torch
    terms = [(RSH_SR, 0.0), (RSH_LR - RSH_SR, RSH_OMEGA)]
    vk = torch.empty_like(dms)
    fused = _timed(lambda: opt.build_jk_async(dms, 1, False, True, None, vk, 0.0, stream,
                                              terms=terms), 2, 1, stream, flush)
    opt.sync(stream)
    ka = torch.empty_like(dms)
    kb = torch.empty_like(dms)

    def two():
        opt.build_jk_async(dms, 1, False, True, None, ka, 0.0, stream, terms=terms[:1])
        opt.build_jk_async(dms, 1, False, True, None, kb, 0.0, stream, terms=terms[1:])

    sep = _timed(two, 2, 1, stream, flush)
    opt.sync(stream)
    return {'omega': RSH_OMEGA, 'lr_factor': RSH_LR, 'sr_factor': RSH_SR,
            'fused_ms': round(fused, 2), 'two_builds_ms': round(sep, 2),
            'speedup': round(sep / fused, 3),
            'max_dK': float((vk - ka - kb).abs().max())}


SCF_CYCLES, SCF_SIGMA0, SCF_DECAY, SCF_SEED = 14, 3e-2, 0.5, 20261207


def run_scf_screen(args, dev, stream, opt, dms_h):
    """Loose-then-tight screening (the reference's fastscfscreen) on a
    synthetic SCF-like trajectory of the main workload: cycle c moves the
    densities by symmetric noise of SCF_SIGMA0 * SCF_DECAY**c * max|D|.
    Tight incremental builds (J/K of D - D_last at direct_scf_tol from the
    second cycle on) against the loose-then-tight schedule (step: the AO
    density change); device ms summed over the cycles, the schedule's
    decisions, and each final J/K against a full tight build of the final
    density."""
    import torch

    from electrolites_b200 import screen
    from electrolites_b200.serve import advance_density

    def trajectory(loose_tight):
        d = torch.as_tensor(dms_h, device=dev).contiguous()
        gen = torch.Generator(device=dev)
        gen.manual_seed(SCF_SEED)
        lt = screen.LooseTightJK(opt) if loose_tight else None
        vj = vk = last = None
        total = 0.0
        with torch.cuda.stream(stream):
            for c in range(SCF_CYCLES):
                s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                s.record(stream)
                if lt is not None:
                    vj, vk = lt.jk(d)
                elif last is None:
                    vj, vk = opt.get_jk(d, 1)
                else:
                    dj, dk = opt.get_jk(d - last, 1)
                    vj, vk = vj + dj, vk + dk
                e.record(stream)
                e.synchronize()
                total += s.elapsed_time(e)
                last = d.clone()
                if c + 1 < SCF_CYCLES:
                    advance_density(d, SCF_SIGMA0 * SCF_DECAY ** c, gen)
            fj, fk = opt.get_jk(d, 1)
        out = {'ms': round(total, 2), 'final_max_dJ': float((vj - fj).abs().max()),
               'final_max_dK': float((vk - fk).abs().max())}
        if lt is not None:
            out['decisions'] = {k: lt.decisions.count(k) for k in
                                (screen.FULL, screen.LOOSE_INC, screen.REBUILD, screen.TIGHT_INC)}
        return out

    tight = trajectory(False)
    lt = trajectory(True)
    return {'cycles': SCF_CYCLES, 'sigma0': SCF_SIGMA0, 'decay': SCF_DECAY,
            'loose': screen.LOOSE, 'switch': screen.SWITCH, 'step': 'AO density change',
            'tight_incremental': tight, 'loose_then_tight': lt,
            'speedup': round(tight['ms'] / lt['ms'], 3)}


def run_serve(args, dev):
    """Serving: Poisson arrivals of water-cluster requests (3-60 waters,
    6-31G* or def2-SVP, 1-4 densities, 10 SCF-like cycles with a 1e-4
    relative density perturbation per cycle), continuous batching over
    resident plans with admission by an HBM budget (half the device).
    Plain and mixed forms at each rate, and the mixed form with incremental
    builds (cycles between full rebuilds every 5th build J/K of the density
    change); mols/s and latency percentiles."""
    from electrolites_b200.serve import JKServer, latency_stats, poisson_requests
    out = {'workload': 'serve_h2o3-60_631gs_svp', 'requests': args.serve_requests,
           'cycles': 10, 'hbm_budget': 'half of device memory', 'rates': []}
    for rate in args.serve_rates:
        row = {'rate_req_per_s': rate}
        for form, thr, inc in (('plain', 0.0, False), ('mixed', BATCH_MIXED, False),
                               ('mixed_incremental', BATCH_MIXED, True)):
            reqs = poisson_requests(args.serve_requests, rate, SERVE_SEED)
            srv = JKServer(dev.index, hbm_budget=0.5, mixed_threshold=thr, incremental=inc,
                           rebuild_every=5)
            srv.run(reqs)
            st = latency_stats(reqs)
            row[form] = {k: round(v, 3) for k, v in st.items()}
            row[form]['mean_batch'] = round(sum(srv.batch_sizes) / len(srv.batch_sizes), 2)
            row[form]['iterations'] = srv.iterations
        out['rates'].append(row)
    return out


def run_ours(args, rank, world):
    import ctypes

    import numpy as np
    import torch
    import torch.distributed as dist

    from electrolites_b200 import _lib, flop_model
    from electrolites_b200.jk import VHFOpt

    local = int(os.environ.get('LOCAL_RANK', 0))
    torch.cuda.set_device(local)
    dev = torch.device('cuda', local)
    mol, dms_h = make_inputs(args.workload)
    n_dm = dms_h.shape[0]
    opt = VHFOpt(mol, TOL, device=local).build()
    opt.set_timing(True)
    dms = torch.as_tensor(dms_h, device=dev)
    # vj and vk in one buffer: with N > 1 ranks each rank builds its share of
    # every class's tasks and one all-reduce of the buffer completes J and K
    buf = torch.empty((2,) + tuple(dms.shape), dtype=torch.float64, device=dev)
    vj, vk = buf[0], buf[1]
    if world > 1:
        opt.set_shard(rank, world)
    flush = torch.empty(L2_FLUSH_BYTES // 8, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    thr = float(args.mixed)

    def one():
        opt.build_jk_async(dms, 1, True, True, vj, vk, thr, stream)
        if world > 1:
            dist.all_reduce(buf)

    for _ in range(max(3, args.warmup)):
        one()
    opt.sync(stream)

    peak = ctypes.c_double()
    _lib.check(_lib.lib().jk_fp64_peak(local, ctypes.byref(peak)), 'jk_fp64_peak')
    peak_tflops = peak.value

    clocks = ClockSampler(local)
    clocks.start()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    evs = []
    class_ms = {}
    launches = 0
    for _ in range(args.steps):
        flush.zero_()                                   # L2 flush, outside the timing
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(stream)
        one()
        e.record(stream)
        evs.append((s, e))
        cm, launches = opt.last_class_ms()             # syncs; between steps
        for k, v in cm.items():
            class_ms[k] = class_ms.get(k, 0.0) + v
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clk = clocks.stop()
    opt.sync(stream)
    step_ms = [s.elapsed_time(e) for s, e in evs]
    total_ms = sum(step_ms)
    if world > 1:
        t = torch.tensor([total_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    ms_per_step = total_ms / args.steps

    # algorithmic flops of one build
    stats = opt.class_counts()         # this rank's share when sharded
    n_k, n_j = n_dm, n_dm
    flops = flop_model.build_flops(stats, n_j, n_k)
    nq = sum(v[0] for v in stats.values())
    if world > 1:
        t = torch.tensor([float(flops), float(nq)], dtype=torch.float64, device=dev)
        dist.all_reduce(t)
        flops, nq = float(t[0]), int(t[1])
    for k in class_ms:
        class_ms[k] /= args.steps
    dom = max(class_ms, key=class_ms.get) if class_ms else None
    dom_flops = flop_model.build_flops({dom: stats[dom]}, n_j, n_k) if dom else 0
    achieved = dom_flops / (class_ms[dom] * 1e-3) / 1e12 if dom else 0.0

    # e2e through the host-buffer entry point, pinned buffers
    dm_pin = torch.as_tensor(dms_h).pin_memory()
    vj_pin = torch.empty_like(dm_pin).pin_memory()
    vk_pin = torch.empty_like(dm_pin).pin_memory()
    L = _lib.lib()

    def one_host():
        if world == 1:        # the C ABI's host-buffer entry point
            _lib.check(L.jk_build_host(opt.plan, ctypes.c_void_p(dm_pin.data_ptr()), n_dm, 1, 1,
                                       1, ctypes.c_void_p(vj_pin.data_ptr()),
                                       ctypes.c_void_p(vk_pin.data_ptr()), thr,
                                       ctypes.c_void_p(stream.cuda_stream)), 'jk_build_host')
            return
        dms.copy_(dm_pin, non_blocking=True)
        one()
        vj_pin.copy_(vj, non_blocking=True)
        vk_pin.copy_(vk, non_blocking=True)
        stream.synchronize()
    one_host()
    e2e_steps = max(1, min(args.steps, 3))
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        flush.zero_()
        torch.cuda.synchronize()
        one_host()
    e2e_s = (time.perf_counter() - t0) / e2e_steps
    if world > 1:
        t = torch.tensor([e2e_s], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    bytes_in = dm_pin.numel() * 8
    bytes_out = 2 * dm_pin.numel() * 8

    # correctness guard on the timed output: symmetric, finite
    assert torch.isfinite(vj).all() and torch.isfinite(vk).all()

    rsh = None
    if rank == 0 and world == 1 and not args.no_rsh:
        rsh = run_rsh(args, dev, stream, flush, opt, dms)

    scf_screen = None
    if rank == 0 and world == 1 and not args.no_scf_screen:
        scf_screen = run_scf_screen(args, dev, stream, opt, dms_h)

    mixed = None
    if rank == 0 and world == 1 and not args.no_mixed:
        mixed = run_mixed(args, dev, stream, flush)

    batched = None
    if rank == 0 and world == 1 and not args.no_batch:
        batched = run_batch(args, dev, stream, flush, peak_tflops)

    serving = None
    if rank == 0 and world == 1 and args.serve_requests > 0:
        serving = run_serve(args, dev)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        v, thr_used, desc = cpu_sample(mol, dms_h, budget_s=args.cpu_budget)
        cpu = {'value': v, 'unit': 'builds/s', 'cores': thr_used, 'kind': 'port',
               'sample': desc}

    if rank == 0:
        line = {
            'metric': 'jk_builds_per_s', 'value': 1e3 / ms_per_step, 'unit': 'builds/s',
            'n_gpus': world, 'steps': args.steps, 'warmup': max(3, args.warmup),
            'ms_per_step': ms_per_step, 'higher_is_better': True, 'scaling': 'strong',
            'vs_baseline': None, 'dtype': 'f64' if thr <= 0 else 'f64+f32',
            'data': 'synthetic',
            'config': {'workload': args.workload, 'nao_cart': mol.nao_cart, 'nbas': mol.nbas,
                       'n_dm': n_dm, 'hermi': 1, 'direct_scf_tol': TOL,
                       'form': 'plain' if thr <= 0 else f'mixed {thr:g}',
                       'parallelism': 'one GPU' if world == 1 else
                       f'{world} ranks, tasks interleaved, one NCCL all-reduce of vj/vk',
                       'l2': 'flushed between steps (256 MB write, untimed)',
                       'quartets': nq, 'build_tflops': flops / (ms_per_step * 1e-3) / 1e12,
                       'fp64_peak_tflops': peak_tflops,
                       'fp64_peak_frac': flops / (ms_per_step * 1e-3) / 1e12 / peak_tflops,
                       'class_ms': {''.join(map(str, k)): round(v, 3) for k, v in
                                    sorted(class_ms.items(), key=lambda kv: -kv[1])[:12]}},
            'roofline': {'bound': 'fp64', 'kernel': 'jk_class_kernel ' + ''.join(map(str, dom)) if dom else None,
                         'achieved': achieved, 'peak': peak_tflops, 'unit': 'TFLOP/s',
                         'frac': achieved / peak_tflops if peak_tflops else None,
                         'peak_source': 'in-run FP64 FMA probe (jk_fp64_peak)',
                         'traffic': None},
            'e2e': {'value': 1.0 / e2e_s, 'unit': 'builds/s', 'h2d_bytes_per_step': bytes_in,
                    'd2h_bytes_per_step': bytes_out},
            'gpu_launches': launches * args.steps,
            'clocks': clk,
            'cpu_baseline': cpu,
            'mixed': mixed,
            'range_separated': rsh,
            'loose_then_tight': scf_screen,
            'batched': batched,
            'serving': serving,
        }
        print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=5)
    ap.add_argument('--warmup', type=int, default=3)
    ap.add_argument('--impl', default='ours', choices=['ours', 'reference'])
    ap.add_argument('--workload', default=DEFAULT, choices=sorted(WORKLOADS))
    ap.add_argument('--mixed', type=float, default=0.0)
    ap.add_argument('--cpu-budget', type=float, default=15.0)
    ap.add_argument('--no-cpu-baseline', action='store_true')
    ap.add_argument('--serve-requests', type=int, default=32,
                    help='requests per serving run (0: skip serving)')
    ap.add_argument('--serve-rates', type=float, nargs='+', default=[50.0],
                    help='Poisson arrival rates (requests/s) of the serving runs')
    ap.add_argument('--no-mixed', action='store_true',
                    help='skip the plain-vs-mixed threshold sweep')
    ap.add_argument('--no-scf-screen', action='store_true',
                    help='skip the loose-then-tight screening trajectory')
    ap.add_argument('--no-rsh', action='store_true',
                    help='skip the fused range-separated exchange comparison')
    ap.add_argument('--no-batch', action='store_true',
                    help='skip the uneven-batch comparison (plain vs batched vs mixed)')
    args = ap.parse_args()
    world = int(os.environ.get('WORLD_SIZE', 1))
    rank = int(os.environ.get('RANK', 0))
    if args.impl == 'reference':
        run_reference(args, rank)
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(int(os.environ.get('LOCAL_RANK', 0)))
        dist.init_process_group('nccl', timeout=datetime.timedelta(seconds=600))
    try:
        run_ours(args, rank, world)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == '__main__':
    main()
