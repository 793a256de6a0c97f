"""bench.py's launcher paths on CPU: `--gpus 2` starts two ranks itself
(torch.distributed.run on 127.0.0.1, gloo in the dry run) and prints one JSON
line with n_gpus = 2 after an all-reduce of the ranks' shares; the reference
arm times the fast CPU checker in shards whose sum is a full build."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _last_json(out):
    lines = [ln for ln in out.splitlines() if ln.startswith('{')]
    assert lines, out[-2000:]
    return json.loads(lines[-1])


def test_bench_starts_its_own_ranks():
    r = subprocess.run([sys.executable, os.path.join(ROOT, 'bench.py'), '--gpus', '2',
                        '--dry-run', '--steps', '1', '--warmup', '0'],
                       capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    line = _last_json(r.stdout)
    assert line['n_gpus'] == 2 and line['exchange_ok'] and line['dry_run']
    assert sum(1 for ln in r.stdout.splitlines() if ln.startswith('{')) == 1


def test_reference_arm_on_the_cpu_workload():
    r = subprocess.run([sys.executable, os.path.join(ROOT, 'bench.py'), '--impl', 'reference',
                        '--workload', 'h2o8_631gs', '--steps', '2', '--warmup', '1'],
                       capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    line = _last_json(r.stdout)
    assert line['impl'] == 'reference' and line['value'] > 0
    assert line['config']['builds_per_step'] == 1 / 8
    assert line['cpu_baseline']['cores'] >= 1
    assert line['e2e']['h2d_bytes_per_step'] == 0
