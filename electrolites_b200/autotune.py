"""Per-class launch tuning of the J/K engine, picked by measurement.

Every class kernel has three runtime knobs (jk_plan_set_tuning /
jk_batch_set_tuning): the number of tasks per SM its task size aims at --
more, smaller tasks balance the persistent grid better, fewer, larger ones
stage fewer bra pairs and claim fewer tasks -- a cap on resident blocks per
SM, and whether mixed-precision builds run the class's low-bound quartets
in FP32 (the per-class tuned threshold of the mixed form: a class where FP32
measures slower keeps FP64).  The tuner times every candidate setting on a
workload, all classes at once with per-class CUDA-event times, keeps the
fastest setting of each class, and stores the table as JSON keyed by device
name and form
('single' for one-molecule builds, 'batch' for batched builds).  Plans and
batches created later on a device with a stored table start from it.

    python -m electrolites_b200.autotune [--out electrolites_b200/tuning.json]

The reference picks its launch shapes in its code generator
(electrolites/codegen/gen_khigh.py); here they are measured on the device.
"""
from __future__ import annotations

import argparse
import json
import os

from .jk import class_keys

HERE = os.path.dirname(os.path.abspath(__file__))
TABLE_PATH = os.path.join(HERE, 'tuning.json')

# (tasks per SM, blocks-per-SM cap; 0 = occupancy limit)
CANDIDATES = [(16, 0), (32, 0), (64, 0), (128, 0), (256, 0), (64, 1)]
# threshold of the mixed builds the FP32 choice is measured on
MIXED_THRESHOLD = 1e-6


def _key(k):
    return ''.join(map(str, k))


def _class_ms(target, run, reps):
    run()
    tot = {}
    for _ in range(reps):
        run()
        ms, _ = target.last_class_ms()
        for k, v in ms.items():
            tot[k] = tot.get(k, 0.0) + v / reps
    return tot


def tune(target, run, run_mixed=None, reps: int = 2, candidates=CANDIDATES) -> dict:
    """target: a VHFOpt or JKBatch; run(): one synchronised plain build on it
    and run_mixed(): one mixed build, both without graph replay (per-class
    times come from its events).  Returns {class key: [tasks_per_sm,
    blocks_per_sm, fp32]} and applies it."""
    keys = class_keys()
    target.set_timing(True)
    best = {}
    for cand in candidates:
        for i in range(len(keys)):
            target.set_tuning(i, *cand)
        for k, v in _class_ms(target, run, reps).items():
            if k not in best or v < best[k][0]:
                best[k] = (v, cand)
    target.set_tuning(-1, 0, 0, -1)
    table = {_key(k): list(c) + [-1] for k, (_, c) in best.items()}
    if run_mixed is not None:
        timed = {}
        for fp32 in (1, 0):
            apply(target, {k: v[:2] + [fp32] for k, v in table.items()})
            timed[fp32] = _class_ms(target, run_mixed, reps)
        for k in timed[1]:
            on, off = timed[1][k], timed[0].get(k, timed[1][k])
            if _key(k) in table:
                table[_key(k)][2] = 1 if on < 0.99 * off else 0
    apply(target, table)
    return table


def tune_jmd(opt, run_j, reps: int = 2) -> dict:
    """J-only builds: per class, the Rys J engine against the
    McMurchie-Davidson J kernel (the reference's J engine,
    electrolites/fastj.py:540-569, picked there per class), timed with
    per-class CUDA events on run_j() (one synchronised J-only build on
    opt).  Returns {class key: [rys ms, md ms, 1 if MD is kept]} for the
    classes that have an MD kernel, and applies the choice (MD kept where it
    is at least 3% faster)."""
    keys = class_keys()
    opt.set_timing(True)
    timed = {}
    for mode in (0, 1):
        opt.set_jmd(mode)
        timed[mode] = _class_ms(opt, run_j, reps)
    opt.set_jmd(0)
    out = {}
    for i, k in enumerate(keys):
        if k not in timed[1] or k not in timed[0]:
            continue
        try:
            opt.set_jmd(1, i)
        except Exception:   # noqa: BLE001 -- no MD kernel for this class
            continue
        rys, md = timed[0][k], timed[1][k]
        keep = md < 0.97 * rys
        opt.set_jmd(1 if keep else 0, i)
        out[_key(k)] = [round(rys, 4), round(md, 4), int(keep)]
    opt.set_timing(False)
    return out


def apply(target, table: dict):
    """Set a stored table on a VHFOpt or JKBatch (classes absent from the
    table keep their defaults)."""
    for i, k in enumerate(class_keys()):
        c = table.get(_key(k))
        if c is not None:
            target.set_tuning(i, int(c[0]), int(c[1]), int(c[2]) if len(c) > 2 else -1)


def device_name(device: int) -> str:
    import torch
    return torch.cuda.get_device_name(device)


def load(device: int, form: str, path: str = TABLE_PATH):
    """The stored table of this device and form, or None."""
    try:
        with open(path) as f:
            data = json.load(f)
    except (OSError, ValueError):
        return None
    return data.get(device_name(device), {}).get(form)


def save(device: int, form: str, table: dict, workload: str, path: str = TABLE_PATH):
    data = {}
    if os.path.exists(path):
        with open(path) as f:
            data = json.load(f)
    entry = data.setdefault(device_name(device), {})
    entry[form] = table
    entry.setdefault('workloads', {})[form] = workload
    with open(path, 'w') as f:
        json.dump(data, f, indent=1, sort_keys=True)


def main():
    import torch

    from . import clusters
    from .batch import JKBatch
    from .jk import VHFOpt
    ap = argparse.ArgumentParser()
    ap.add_argument('--out', default=TABLE_PATH)
    ap.add_argument('--reps', type=int, default=2)
    ap.add_argument('--batch-mols', type=int, default=512)
    ap.add_argument('--jmd-only', action='store_true',
                    help='only compare the McMurchie-Davidson J kernel with the Rys J '
                         'engine per class (J-only builds) and print the table')
    args = ap.parse_args()
    dev = torch.device('cuda', torch.cuda.current_device())
    # single: (H2O)_96, 6-31G*, UHF pair
    mol = clusters.water_mole(96, 15.0, 20261204)
    dms = torch.as_tensor(clusters.uhf_pair(clusters.atomic_density(mol, 20261204), 20261205),
                          device=dev)
    opt = VHFOpt(mol, 1e-13).build()
    if args.jmd_only:
        for name, (m, d) in {'(H2O)96 6-31G* UHF pair': (mol, dms),
                             '(H2O)16 def2-TZVP': (lambda m2: (m2, torch.as_tensor(
                                 clusters.atomic_density(m2, 20261205)[None], device=dev)))(
                                 clusters.water_mole(16, 7.8, 20261205, basis='def2-tzvp'))}.items():
            o = opt if m is mol else VHFOpt(m, 1e-13).build()
            t = tune_jmd(o, lambda: o.get_j(d), args.reps)
            print(name, 'J-only, ms per class: [Rys J engine, McMurchie-Davidson, MD kept]')
            for k, v in sorted(t.items(), key=lambda kv: -kv[1][0]):
                print(f'  {k}  {v[0]:9.3f}  {v[1]:9.3f}  {v[2]}')
        return
    table = tune(opt, lambda: opt.get_jk(dms, 1),
                 lambda: opt.get_jk(dms, 1, mixed_threshold=MIXED_THRESHOLD), args.reps)
    save(dev.index, 'single', table, '(H2O)96 6-31G* UHF pair', args.out)
    print('single', json.dumps(table))
    # batch: uneven 1-24 water clusters, 6-31G*, 1-4 densities
    items = clusters.uneven_batch(args.batch_mols, 20261206)
    opts = [VHFOpt(m, 1e-13).build() for m, _ in items]
    bd = [torch.as_tensor(d, device=dev) for _, d in items]
    batch = JKBatch(dev.index)
    table = tune(batch, lambda: batch.build(opts, bd, 1),
                 lambda: batch.build(opts, bd, 1, mixed_threshold=MIXED_THRESHOLD), args.reps)
    save(dev.index, 'batch', table, f'{args.batch_mols} water clusters 1-24, 6-31G*', args.out)
    print('batch', json.dumps(table))


if __name__ == '__main__':
    main()
