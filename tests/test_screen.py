"""Host logic of the loose-then-tight schedule (electrolites_b200.screen),
checked against the reference's phase rules (electrolites/fastscfscreen.py:
97-127): a full build starts the loose phase, loose increments run while
the step is at least the switch and fewer than max_loose have run, the
first step below the switch (or the cap) is a tight rebuild, and the cycles
after it are tight increments whose step is never evaluated."""
import numpy as np
import pytest

from electrolites_b200 import screen
from electrolites_b200.screen import FULL, LOOSE_INC, REBUILD, TIGHT_INC, ScreenPhase


def _never():
    raise AssertionError('the step is evaluated only in the loose phase')


def test_phase_sequence():
    s = ScreenPhase(loose=1e-10, switch=1e-3, max_loose=30)
    seq = [s.decide(False, _never)]
    seq += [s.decide(True, st) for st in (5e-2, 1e-2, 2e-3, 9e-4)]
    seq += [s.decide(True, _never) for _ in range(3)]
    assert seq == [FULL, LOOSE_INC, LOOSE_INC, LOOSE_INC, REBUILD, TIGHT_INC, TIGHT_INC, TIGHT_INC]
    assert s.stats == {'loose_builds': 3, 'rebuilds': 1, 'tight_builds': 4, 'capped': 0}


def test_cap_ends_the_loose_phase():
    s = ScreenPhase(max_loose=2)
    seq = [s.decide(False, _never)] + [s.decide(True, 1.0) for _ in range(4)]
    assert seq == [FULL, LOOSE_INC, LOOSE_INC, REBUILD, TIGHT_INC]
    assert s.stats['capped'] == 1


def test_full_build_restarts_the_schedule():
    s = ScreenPhase()
    assert [s.decide(False, _never), s.decide(True, 1e-4), s.decide(True, _never)] == \
        [FULL, REBUILD, TIGHT_INC]
    assert s.decide(False, _never) == FULL
    assert s.decide(True, lambda: 1.0) == LOOSE_INC
    assert s.nloose == 1


def test_thresholds():
    s = ScreenPhase(loose=1e-10)
    assert s.tol(LOOSE_INC, 1e-13) == 1e-10
    assert s.tol(TIGHT_INC, 1e-13) == 1e-13
    assert s.tol(REBUILD, 1e-13) == 1e-13
    assert s.tol(FULL, 1e-13) == 1e-13
    # a tight threshold above the loose one is never lowered
    assert s.tol(LOOSE_INC, 1e-8) == 1e-8


def test_density_step_lowdin_and_ao():
    torch = pytest.importorskip('torch')
    rng = np.random.default_rng(3)
    a = rng.standard_normal((6, 6))
    S = a @ a.T + 6 * np.eye(6)
    w, u = np.linalg.eigh(S)
    x = (u * np.sqrt(w)) @ u.T
    d1 = rng.standard_normal((2, 6, 6))
    d0 = rng.standard_normal((2, 6, 6))
    xt = screen.ovlp_sqrt(torch.as_tensor(S))
    assert np.abs(xt.numpy() - x).max() < 1e-12
    ref = np.abs(x @ (d1 - d0) @ x).max()
    got = screen.density_step(torch.as_tensor(d1), torch.as_tensor(d0), xt)
    assert abs(got - ref) < 1e-12
    assert screen.density_step(torch.as_tensor(d1), torch.as_tensor(d0)) == np.abs(d1 - d0).max()
