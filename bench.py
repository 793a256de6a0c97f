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
job (device-timed with CUDA events, densities resident in HBM, the default
launch path: no per-class events); e2e = the same through jk_build_host from
pinned host buffers, copies included.  A second, separately timed pass with
per-class events on the class streams (the same launch order) gives the
dominant class kernel's in-situ time for the roofline.  With N > 1 ranks
(one GPU each; `--gpus N` starts them itself through torch.distributed.run
when WORLD_SIZE is unset) the build is sharded: every rank evaluates the
tasks rank, rank + N, ... of each class launch and one NCCL all-reduce of
the (vj, vk) buffer completes the build on every rank (strong scaling: one
build per step for the whole job); timing is the max over ranks.

The default run also reports: the timed build's errors against the fast
FP64 CPU checker (oracle/jk_check.c), whose full, unsampled build of the
same workload on all host cores is the CPU baseline; the plain-vs-mixed
threshold sweep (1e-10..1e-6) on this workload and on (H2O)_64 def2-TZVP,
each with its errors against the checker; the uneven 512-molecule batch;
a serving sweep over request rates.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
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


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def checker_build(mol, dms, nthreads=0, shard=0, nshard=1):
    """The fast FP64 CPU checker (oracle/jk_check.c) on `nthreads` host
    threads: (vj, vk, quartets, seconds) of bra-pair shard `shard` of
    `nshard` (0 of 1: the whole build)."""
    from oracle import oracle as O
    t0 = time.perf_counter()
    vj, vk, nq = O.jk_fast(mol, dms, tol=TOL, nthreads=nthreads or host_cores(),
                           shard=shard, nshard=nshard)
    return vj, vk, nq, time.perf_counter() - t0


class BackgroundCheck(threading.Thread):
    """A checker build on a worker thread (ctypes releases the GIL), so that
    the host cores work while the GPU runs other measurements."""

    def __init__(self, mol, dms, nthreads):
        super().__init__(daemon=True)
        self.args = (mol, dms, nthreads)
        self.result = None
        self.error = None

    def run(self):
        try:
            self.result = checker_build(*self.args)
        except Exception as err:   # noqa: BLE001
            self.error = err


def errors_vs(dms, vj, vk, rj, rk):
    """Largest element errors and energy errors (E_J = 1/2 tr(D J),
    E_K = -1/4 tr(D K), summed over the densities) of (vj, vk) against the
    checker's (rj, rk)."""
    import numpy as np
    ej = 0.5 * np.einsum('nij,nji->', dms, vj) - 0.5 * np.einsum('nij,nji->', dms, rj)
    ek = -0.25 * np.einsum('nij,nji->', dms, vk) + 0.25 * np.einsum('nij,nji->', dms, rk)
    return {'max_dJ': float(np.abs(vj - rj).max()), 'max_dK': float(np.abs(vk - rk).max()),
            'dE_J': float(ej), 'dE_K': float(ek)}


REF_SHARDS = 8


def run_reference(args, rank):
    """The CPU arm: the fast FP64 checker (the restated reference algorithm,
    oracle/jk_check.c) on all host cores.  Step s builds bra-pair shard
    s mod 8 of 8 of the workload (interleaved bra pairs, so every shard has
    the same mix), so 8 consecutive steps are one full, unsampled build and
    the timed region covers whole builds; value = builds per second."""
    if rank != 0:
        return
    mol, dms = make_inputs(args.workload)
    cores = host_cores()
    times = []
    for it in range(args.warmup + args.steps):
        _, _, _, dt = checker_build(mol, dms, cores, it % REF_SHARDS, REF_SHARDS)
        if it >= args.warmup:
            times.append(dt)
    step_s = sum(times) / len(times)
    v = (1.0 / REF_SHARDS) / step_s
    desc = (f'fast FP64 checker (oracle/jk_check.c), {cores} threads; step = bra-pair shard '
            f'(s mod {REF_SHARDS}) of {REF_SHARDS} of the full build, so {REF_SHARDS} steps '
            f'are one unsampled build')
    line = {'impl': 'reference', 'metric': 'jk_builds_per_s', 'value': v,
            'unit': 'builds/s', 'n_gpus': args.gpus, 'steps': args.steps,
            'warmup': args.warmup, 'ms_per_step': step_s * 1e3, 'higher_is_better': True,
            'scaling': 'strong', 'vs_baseline': None, 'dtype': 'f64', 'data': 'synthetic',
            'config': {'workload': args.workload, 'nao_cart': mol.nao_cart, 'n_dm': int(dms.shape[0]),
                       'hermi': 1, 'direct_scf_tol': TOL, 'form': 'plain',
                       'builds_per_step': 1.0 / REF_SHARDS},
            'cpu_baseline': {'value': v, 'unit': 'builds/s', 'cores': cores,
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


def run_mixed(args, dev, stream, flush, workloads=MIXED_WORKLOADS):
    """Plain FP64 against the mixed form at each threshold of the sweep, on
    the (H2O)_96 6-31G* UHF pair and (H2O)_64 def2-TZVP: device ms per build,
    the fraction of quartets run in FP32, and the J/K energy and largest
    element errors against the plain build (E_J = 1/2 tr(D J),
    E_K = -1/4 tr(D K) summed over the densities).  Returns the table and
    each form's (vj, vk) on the host, for the errors against the checker."""
    import torch

    from electrolites_b200.jk import VHFOpt
    out, host = {}, {}
    for w in workloads:
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
        host[w] = (mol, dms_h, {thr: (r[4].cpu().numpy(), r[5].cpu().numpy())
                                for thr, r in res.items()})
        del opt, res
    return out, host


def mixed_vs_checker(table, host, checks):
    """Adds each form's errors against the checker: 'vs_checker' per row
    (plain) and per threshold."""
    for w, (mol, dms_h, arrs) in host.items():
        if w not in checks:
            continue
        rj, rk = checks[w]
        table[w]['plain_vs_checker'] = errors_vs(dms_h, *arrs[0.0], rj, rk)
        for thr in MIXED_SWEEP:
            table[w]['thresholds'][f'{thr:g}']['vs_checker'] = errors_vs(dms_h, *arrs[thr], rj, rk)


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


def run_jonly(args, dev, stream, flush, opt, dms):
    """J-only builds of the main workload (the reference's get_j): the
    default per-class choice (the Rys J engine where it measured faster)
    against the McMurchie-Davidson kernel in every class that has one;
    device ms per build and the largest element difference."""
    import torch
    vj = torch.empty_like(dms)
    opt.set_jmd(-1)
    dflt = _timed(lambda: opt.build_jk_async(dms, 1, True, False, vj, None, 0.0, stream),
                  2, 1, stream, flush)
    opt.sync(stream)
    ref = vj.clone()
    opt.set_jmd(1)
    md = _timed(lambda: opt.build_jk_async(dms, 1, True, False, vj, None, 0.0, stream),
                2, 1, stream, flush)
    opt.sync(stream)
    opt.set_jmd(-1)
    return {'default_ms': round(dflt, 2), 'md_every_class_ms': round(md, 2),
            'max_dJ': float((vj - ref).abs().max())}


GRAD_WORKLOAD, GRAD_CHECK = 'h2o32_631gs_uhf', 'h2o8_631gs'
GRAD_J, GRAD_K = 1.0, 0.2


def run_grad(args, dev, stream, flush, check):
    """Nuclear gradient of the two-electron energy (the reference's
    fastejk, jk_grad): device ms per gradient on (H2O)_32 6-31G* UHF against
    one J/K build of the same densities, and (check) the gradient of the
    (H2O)_8 UHF pair against the checker's analytic gradient."""
    import numpy as np
    import torch

    from electrolites_b200 import clusters
    from electrolites_b200.jk import VHFOpt
    mol, dms_h = make_inputs(GRAD_WORKLOAD)
    opt = VHFOpt(mol, TOL).build()
    dms = torch.as_tensor(dms_h, device=dev)
    g_ms = _timed(lambda: opt.jk_energy_per_atom(dms, GRAD_J, GRAD_K, stream=stream), 2, 1,
                  stream, flush)
    jk_ms = _timed(lambda: opt.build_jk_async(dms, 1, stream=stream), 2, 1, stream, flush)
    opt.sync(stream)
    out = {'workload': GRAD_WORKLOAD, 'j_factor': GRAD_J, 'k_factor': GRAD_K,
           'natm': int(mol.natm), 'grad_ms': round(g_ms, 2), 'jk_build_ms': round(jk_ms, 2),
           'ratio': round(g_ms / jk_ms, 2)}
    if check:
        from oracle import oracle as O
        mc, dc = make_inputs(GRAD_CHECK)
        dc = clusters.uhf_pair(dc[0], 20261208)
        oc = VHFOpt(mc, TOL).build()
        g = oc.jk_energy_per_atom(torch.as_tensor(dc, device=dev), GRAD_J, GRAD_K).cpu().numpy()
        rg, _ = O.grad_jk_fast(mc, dc, GRAD_J, GRAD_K, tol=TOL, nthreads=host_cores())
        err = float(np.abs(g - rg).max() / np.abs(rg).max())
        out['check'] = {'workload': GRAD_CHECK + ' UHF pair', 'max_rel_err': err,
                        'force_sum': float(np.abs(g.sum(axis=0)).max()),
                        'checker': 'oracle/jk_check.c', 'pass': err <= 1e-9}
    return out


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


SERVE_FORMS = {'plain': (0.0, False), 'mixed': (BATCH_MIXED, False),
               'mixed_incremental': (BATCH_MIXED, True)}


def run_serve(args, dev):
    """Serving: Poisson arrivals of water-cluster requests (3-60 waters,
    6-31G* or def2-SVP, 1-4 densities, 10 SCF-like cycles with a 1e-4
    relative density perturbation per cycle), continuous batching over
    resident plans with admission by an HBM budget (half the device).  For
    each rate and form: mols/s, latency percentiles, the run's length and
    whether p99 stayed bounded (below half the run length: requests did not
    pile up); the highest bounded rate per form.  Rates below the server's
    capacity (about 1.5 requests/s of this workload on one GPU) take
    --serve-low-requests requests, the others --serve-requests."""
    from electrolites_b200.serve import JKServer, latency_stats, poisson_requests
    out = {'workload': 'serve_h2o3-60_631gs_svp', 'cycles': 10,
           'hbm_budget': 'half of device memory', 'forms': list(args.serve_forms), 'rates': []}
    best = {f: None for f in args.serve_forms}
    for rate in args.serve_rates:
        n_req = args.serve_low_requests if rate <= 2.0 else args.serve_requests
        row = {'rate_req_per_s': rate, 'requests': n_req}
        for form in args.serve_forms:
            thr, inc = SERVE_FORMS[form]
            reqs = poisson_requests(n_req, rate, SERVE_SEED)
            srv = JKServer(dev.index, hbm_budget=0.5, mixed_threshold=thr, incremental=inc,
                           rebuild_every=5)
            srv.run(reqs)
            st = latency_stats(reqs)
            span = max(r.finished for r in reqs) - min(r.arrival for r in reqs)
            r = {k: round(v, 3) for k, v in st.items()}
            r['run_s'] = round(span, 2)
            r['p99_bounded'] = bool(st['p99_ms'] * 1e-3 < 0.5 * span)
            r['mean_batch'] = round(sum(srv.batch_sizes) / len(srv.batch_sizes), 2)
            r['iterations'] = srv.iterations
            row[form] = r
            if r['p99_bounded'] and (best[form] is None or rate > best[form]):
                best[form] = rate
        out['rates'].append(row)
    out['highest_bounded_rate'] = best
    return out


# DRAM traffic of a class kernel's launch (dram__bytes_read.sum +
# dram__bytes_write.sum, one ncu capture) on the (H2O)_32 6-31G* UHF case
# (608 Cartesian AOs), and the AO count it was taken at.  The kernels read
# their inputs -- densities, pair and primitive tables -- about once from
# DRAM (the rest hits L2), so the traffic follows the data's size, nao^2, and
# not the quartet count; the bench scales it by (nao / 608)^2.  Source:
# profiles/jk_class_kernels_h2o32_631gs_uhf.md.
TRAFFIC_SMALL = {(1, 0, 0, 0): 13473280, (0, 0, 0, 0): 12206080, (1, 0, 1, 0): 13282560,
                 (2, 0, 0, 0): 11496448, (2, 0, 1, 0): 12419584}
TRAFFIC_NAO = 608


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

    def timed_steps(per_class):
        """K device-timed builds (L2 flushed, untimed, before each); with
        per_class, also the class kernels' in-situ times summed."""
        evs, class_ms = [], {}
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        for _ in range(args.steps):
            flush.zero_()                               # L2 flush, outside the timing
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record(stream)
            one()
            e.record(stream)
            evs.append((s, e))
            if per_class:
                cm, _ = opt.last_class_ms()              # syncs; between steps
                for k, v in cm.items():
                    class_ms[k] = class_ms.get(k, 0.0) + v
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        total = sum(s.elapsed_time(e) for s, e in evs)
        if world > 1:
            t = torch.tensor([total], device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            total = float(t.item())
        return total / args.steps, {k: v / args.steps for k, v in class_ms.items()}

    # the headline: the default launch path, no per-class events
    clocks = ClockSampler(local)
    clocks.start()
    ms_per_step, _ = timed_steps(False)
    clk = clocks.stop()
    opt.sync(stream)
    _, launches = opt.last_class_ms()
    vj_timed, vk_timed = vj.cpu().numpy(), vk.cpu().numpy()

    # the class kernels' in-situ times: the same launch order (two class
    # streams) with each class's events on its own stream, timed separately;
    # then each class kernel timed alone (class kernels serialised), the
    # duration the roofline of the dominant kernel is taken from
    opt.set_timing(2)
    ms_instrumented, class_ms_situ = timed_steps(True)
    opt.set_timing(1)
    ms_serial, class_ms = timed_steps(True)
    opt.set_timing(False)

    # algorithmic flops of one build
    stats = opt.class_counts()         # this rank's share when sharded
    n_k, n_j = n_dm, n_dm
    flops = flop_model.build_flops(stats, n_j, n_k)
    nq = sum(v[0] for v in stats.values())
    if world > 1:
        t = torch.tensor([float(flops), float(nq)], dtype=torch.float64, device=dev)
        dist.all_reduce(t)
        flops, nq = float(t[0]), int(t[1])
    dom = max(class_ms, key=class_ms.get) if class_ms else None
    dom_flops = flop_model.build_flops({dom: stats[dom]}, n_j, n_k) if dom else 0
    achieved = dom_flops / (class_ms[dom] * 1e-3) / 1e12 if dom else 0.0
    t_small = TRAFFIC_SMALL.get(dom)
    traffic = t_small * (mol.nao_cart / TRAFFIC_NAO) ** 2 if t_small else None

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
    assert np.isfinite(vj_timed).all() and np.isfinite(vk_timed).all()

    solo = rank == 0 and world == 1
    check = solo and not args.no_check
    # the def2-TZVP checker build runs on the host cores while the GPU
    # measures the other forms (it is not a timed CPU number)
    bg = None
    if check and not args.no_mixed and 'h2o64_tzvp' in MIXED_WORKLOADS:
        mol2, dms2 = make_inputs('h2o64_tzvp')
        bg = BackgroundCheck(mol2, dms2, max(1, host_cores() - 2))
        bg.start()

    rsh = run_rsh(args, dev, stream, flush, opt, dms) if solo and not args.no_rsh else None
    jonly = run_jonly(args, dev, stream, flush, opt, dms) if solo and not args.no_jonly else None
    grad = run_grad(args, dev, stream, flush, check) if solo and not args.no_grad else None
    scf_screen = (run_scf_screen(args, dev, stream, opt, dms_h)
                  if solo and not args.no_scf_screen else None)
    mixed = mixed_host = None
    if solo and not args.no_mixed:
        mixed, mixed_host = run_mixed(args, dev, stream, flush)
    batched = None
    if solo and not args.no_batch:
        batched = run_batch(args, dev, stream, flush, peak_tflops)
    serving = None
    if solo and args.serve_forms and args.serve_rates:
        serving = run_serve(args, dev)

    # CPU baseline: one full, unsampled checker build of the workload on all
    # host cores (nothing else running), which is also the parity reference
    # of the timed GPU build
    cpu = parity = None
    if bg is not None:
        bg.join()
    if check:
        cores = host_cores()
        rj, rk, cnq, cs = checker_build(mol, dms_h, cores)
        cpu = {'value': 1.0 / cs, 'unit': 'builds/s', 'cores': cores, 'kind': 'port',
               'sample': f'one full, unsampled build of {args.workload} ({cnq} quartets) by the '
                         f'fast FP64 checker oracle/jk_check.c in {cs:.1f} s'}
        parity = errors_vs(dms_h, vj_timed, vk_timed, rj, rk)
        parity.update({'checker': 'oracle/jk_check.c', 'element_tol': 1e-10,
                       'energy_tol_eh': 1e-9,
                       'pass': parity['max_dJ'] <= 1e-10 and parity['max_dK'] <= 1e-10 and
                       abs(parity['dE_J']) <= 1e-9 and abs(parity['dE_K']) <= 1e-9})
        checks = {args.workload: (rj, rk)}
        if bg is not None and bg.result is not None:
            checks['h2o64_tzvp'] = bg.result[:2]
        if mixed is not None:
            mixed_vs_checker(mixed, mixed_host, checks)
        if bg is not None and bg.error is not None:
            parity['tzvp_check_error'] = str(bg.error)

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
                       'timed_path': 'default launch order (two class streams, no per-class events)',
                       'quartets': nq, 'build_tflops': flops / (ms_per_step * 1e-3) / 1e12,
                       'fp64_peak_tflops': peak_tflops,
                       'fp64_peak_frac': flops / (ms_per_step * 1e-3) / 1e12 / peak_tflops,
                       'instrumented_ms_per_step': ms_instrumented,
                       'serialised_ms_per_step': ms_serial,
                       'class_ms': {''.join(map(str, k)): round(v, 3) for k, v in
                                    sorted(class_ms.items(), key=lambda kv: -kv[1])[:12]},
                       'class_ms_in_situ': {''.join(map(str, k)): round(v, 3) for k, v in
                                            sorted(class_ms_situ.items(),
                                                   key=lambda kv: -kv[1])[:12]}},
            'roofline': {'bound': 'fp64', 'kernel': 'jk_class_kernel ' + ''.join(map(str, dom)) if dom else None,
                         'achieved': achieved, 'peak': peak_tflops, 'unit': 'TFLOP/s',
                         'frac': achieved / peak_tflops if peak_tflops else None,
                         'peak_source': 'in-run FP64 FMA probe (jk_fp64_peak)',
                         'duration_source': 'the kernel timed alone (class kernels serialised, '
                                            'CUDA events), separate timed pass',
                         'traffic': traffic,
                         'traffic_unit': 'bytes per launch',
                         'traffic_source': 'ncu dram bytes of this kernel on (H2O)_32 (608 AOs), '
                                           'scaled by (nao/608)^2' if traffic else None},
            'e2e': {'value': 1.0 / e2e_s, 'unit': 'builds/s', 'h2d_bytes_per_step': bytes_in,
                    'd2h_bytes_per_step': bytes_out},
            'gpu_launches': launches * args.steps,
            'clocks': clk,
            'parity': parity,
            'cpu_baseline': cpu,
            'mixed': mixed,
            'range_separated': rsh,
            'j_only': jonly,
            'gradient': grad,
            'loose_then_tight': scf_screen,
            'batched': batched,
            'serving': serving,
        }
        print(json.dumps(line), flush=True)


def run_dry(args, rank, world):
    """The multi-rank launcher and exchange without a GPU (gloo): each rank
    adds a rank-dependent share of a fixed matrix, one all-reduce sums the
    shares, rank 0 checks the sum and prints the JSON line shape.  It times
    nothing and claims no throughput."""
    import numpy as np
    import torch
    import torch.distributed as dist
    full = np.arange(64, dtype=np.float64).reshape(8, 8)
    share = np.where(np.arange(64).reshape(8, 8) % world == rank, full, 0.0)
    buf = torch.as_tensor(share)
    if world > 1:
        dist.all_reduce(buf)
    ok = bool(np.array_equal(buf.numpy(), full))
    if rank == 0:
        print(json.dumps({'metric': 'jk_builds_per_s', 'value': None, 'unit': 'builds/s',
                          'n_gpus': world, 'steps': args.steps, 'warmup': args.warmup,
                          'dry_run': True, 'exchange_ok': ok,
                          'config': {'workload': args.workload, 'parallelism':
                                     f'{world} ranks (gloo, no GPU)'}}), flush=True)
    if not ok:
        raise SystemExit('dry run: the all-reduced shares do not sum to the matrix')


def launch_ranks(args):
    """`--gpus N` without a launcher: start N ranks through
    torch.distributed.run on this node (127.0.0.1) and return their exit
    code.  Fails when fewer than N CUDA devices are visible."""
    import socket
    if not args.dry_run:
        import torch
        n = torch.cuda.device_count()
        if n < args.gpus:
            raise SystemExit(f'bench.py: --gpus {args.gpus} but {n} CUDA device(s) visible')
    with socket.socket() as sk:
        sk.bind(('127.0.0.1', 0))
        port = sk.getsockname()[1]
    env = dict(os.environ)
    if not args.dry_run:
        # NCCL's communicator set-up lines name the rank count
        env.setdefault('NCCL_DEBUG', 'INFO')
        env.setdefault('NCCL_DEBUG_SUBSYS', 'INIT')
    cmd = [sys.executable, '-m', 'torch.distributed.run', '--nnodes=1',
           f'--nproc-per-node={args.gpus}', '--master-addr=127.0.0.1',
           f'--master-port={port}', os.path.abspath(__file__)] + sys.argv[1:]
    return subprocess.call(cmd, env=env)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=5)
    ap.add_argument('--warmup', type=int, default=3)
    ap.add_argument('--impl', default='ours', choices=['ours', 'reference'])
    ap.add_argument('--workload', default=DEFAULT, choices=sorted(WORKLOADS))
    ap.add_argument('--mixed', type=float, default=0.0)
    ap.add_argument('--no-check', action='store_true',
                    help='skip the checker builds (parity, CPU baseline, mixed errors)')
    ap.add_argument('--serve-rates', type=float, nargs='*', default=[0.5, 1.0, 2.0, 50.0, 2000.0],
                    help='Poisson arrival rates (requests/s) of the serving runs')
    ap.add_argument('--serve-requests', type=int, default=24,
                    help='requests per serving run above 2 requests/s')
    ap.add_argument('--serve-low-requests', type=int, default=12,
                    help='requests per serving run at 2 requests/s or less')
    ap.add_argument('--serve-forms', nargs='*', default=['plain', 'mixed_incremental'],
                    choices=sorted(SERVE_FORMS), help='server forms to run (none: skip serving)')
    ap.add_argument('--no-mixed', action='store_true',
                    help='skip the plain-vs-mixed threshold sweep')
    ap.add_argument('--no-scf-screen', action='store_true',
                    help='skip the loose-then-tight screening trajectory')
    ap.add_argument('--no-rsh', action='store_true',
                    help='skip the fused range-separated exchange comparison')
    ap.add_argument('--no-jonly', action='store_true',
                    help='skip the J-only builds (Rys J engine against McMurchie-Davidson)')
    ap.add_argument('--no-grad', action='store_true',
                    help='skip the nuclear-gradient measurement')
    ap.add_argument('--no-batch', action='store_true',
                    help='skip the uneven-batch comparison (plain vs batched vs mixed)')
    ap.add_argument('--dry-run', action='store_true',
                    help='launcher and exchange only, on CPU ranks (gloo); no GPU, no timing')
    args = ap.parse_args()
    if args.gpus > 1 and 'WORLD_SIZE' not in os.environ and args.impl == 'ours':
        sys.exit(launch_ranks(args))
    world = int(os.environ.get('WORLD_SIZE', 1))
    rank = int(os.environ.get('RANK', 0))
    if args.impl == 'reference':
        run_reference(args, rank)
        return
    if 'WORLD_SIZE' in os.environ and world != args.gpus:
        raise SystemExit(f'bench.py: --gpus {args.gpus} but WORLD_SIZE={world}')
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        if not args.dry_run:
            torch.cuda.set_device(int(os.environ.get('LOCAL_RANK', 0)))
        dist.init_process_group('gloo' if args.dry_run else 'nccl',
                                timeout=datetime.timedelta(seconds=600))
    try:
        if args.dry_run:
            run_dry(args, rank, world)
        else:
            run_ours(args, rank, world)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == '__main__':
    main()
