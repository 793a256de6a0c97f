"""The autotuner's selection logic on CPU, with a stand-in engine whose
per-class kernel times depend on the settings in a known way."""
import json

import pytest


class FakeTarget:
    """Per-class times: class k is fastest at tasks_per_sm = 32 * 2^k with
    no blocks cap; FP32 makes even classes faster and odd classes slower in
    mixed builds."""

    def __init__(self, keys):
        self.keys = keys
        self.tune = {i: (64, 0, -1) for i in range(len(keys))}
        self.mixed = False
        self.timing = False

    def set_timing(self, on=True):
        self.timing = on

    def set_tuning(self, cls, tasks, bps, fp32=-1):
        if cls == -1:
            self.tune = {i: (64, 0, -1) for i in range(len(self.keys))}
        else:
            self.tune[cls] = (tasks, bps, fp32)

    def last_class_ms(self):
        out = {}
        for i, k in enumerate(self.keys):
            t, b, f = self.tune[i]
            best = 32 << i
            ms = 10.0 + abs(t - best) / 16.0 + (2.0 if b else 0.0)
            if self.mixed and f == 1:
                ms *= 0.9 if i % 2 == 0 else 1.2
            out[k] = ms
        return out, 1


def test_tune_picks_fastest_settings_and_fp32(monkeypatch):
    from electrolites_b200 import autotune
    keys = [(0, 0, 0, 0), (1, 0, 0, 0), (1, 0, 1, 0), (1, 1, 0, 0)]
    monkeypatch.setattr(autotune, 'class_keys', lambda: keys)
    t = FakeTarget(keys)

    def run():
        t.mixed = False

    def run_mixed():
        t.mixed = True

    table = autotune.tune(t, run, run_mixed, reps=1)
    assert table['0000'] == [32, 0, 1]
    assert table['1000'] == [64, 0, 0]
    assert table['1010'] == [128, 0, 1]
    assert table['1100'] == [256, 0, 0]
    # the table is applied to the target
    assert t.tune[0] == (32, 0, 1) and t.tune[3] == (256, 0, 0)


def test_table_round_trip(tmp_path, monkeypatch):
    from electrolites_b200 import autotune
    monkeypatch.setattr(autotune, 'device_name', lambda d: 'Test GPU')
    path = str(tmp_path / 'tuning.json')
    autotune.save(0, 'single', {'0000': [32, 0, 1]}, 'w1', path)
    autotune.save(0, 'batch', {'1000': [64, 1, 0]}, 'w2', path)
    assert autotune.load(0, 'single', path) == {'0000': [32, 0, 1]}
    assert autotune.load(0, 'batch', path) == {'1000': [64, 1, 0]}
    data = json.load(open(path))
    assert data['Test GPU']['workloads'] == {'single': 'w1', 'batch': 'w2'}
    monkeypatch.setattr(autotune, 'device_name', lambda d: 'Other GPU')
    assert autotune.load(0, 'single', path) is None


def test_committed_table_is_well_formed():
    from electrolites_b200 import autotune
    try:
        data = json.load(open(autotune.TABLE_PATH))
    except FileNotFoundError:
        pytest.skip('no measured table')
    for dev, entry in data.items():
        for form in ('single', 'batch'):
            for key, v in entry.get(form, {}).items():
                assert len(key) == 4 and key.isdigit()
                assert v[0] > 0 and v[1] >= 0 and (len(v) < 3 or v[2] in (-1, 0, 1))


class FakeJmd:
    """J-only per-class times: class 0 is faster with the MD kernel, class 1
    slower, class 2 has no MD kernel (set_jmd on it raises)."""

    def __init__(self, keys):
        self.keys = keys
        self.mode = {i: 0 for i in range(len(keys))}

    def set_timing(self, on=True):
        pass

    def set_jmd(self, mode=1, cls=-1):
        if cls == 2 and mode == 1:
            raise RuntimeError('no MD kernel')
        for i in (range(len(self.keys)) if cls < 0 else [cls]):
            if i != 2:
                self.mode[i] = mode

    def last_class_ms(self):
        base = {0: 10.0, 1: 10.0, 2: 5.0}
        md = {0: 8.0, 1: 14.0, 2: 5.0}
        return {k: (md[i] if self.mode[i] else base[i]) for i, k in enumerate(self.keys)}, 1


def test_tune_jmd_keeps_md_where_faster(monkeypatch):
    from electrolites_b200 import autotune
    keys = [(1, 0, 0, 0), (2, 0, 0, 0), (3, 3, 3, 3)]
    monkeypatch.setattr(autotune, 'class_keys', lambda: keys)
    t = FakeJmd(keys)
    out = autotune.tune_jmd(t, lambda: None, reps=1)
    assert out == {'1000': [10.0, 8.0, 1], '2000': [10.0, 14.0, 0]}
    assert t.mode == {0: 1, 1: 0, 2: 0}
