"""Loose-then-tight screening of incremental J/K builds.

The schedule of the reference's direct-SCF wrapper
(electrolites/fastscfscreen.py:97-127): while the density still moves by
more than ``switch`` per cycle, the incremental builds (J/K of
Delta D = D - D_last, added to the previous J/K) screen at the looser
``loose`` threshold; at the first cycle whose step is below ``switch`` -- or
after ``max_loose`` loose builds, whatever the step -- J/K are rebuilt from
scratch at the tight threshold, and the cycles after that are incremental
and tight.  Everything the converged answer is made of (the last full build
and every increment after it) is therefore at the tight threshold; the loose
cycles only shape the path there.

The step is the largest element of S^1/2 (D - D_last) S^1/2 (the density
change in the Loewdin basis) when the overlap S is given, else of
D - D_last itself (fastscfscreen.py:80-94).  The loose threshold reaches the
builds through the option object's ``direct_scf_tol``, which builds read at
call time (``VHFOpt.apply_tol`` / ``jk_plan_set_tol``), as the reference
raises ``_VHFOpt.direct_scf_tol`` for the duration of a loose build
(fastscfscreen.py:112-123).
"""
from __future__ import annotations

LOOSE = 1e-10
SWITCH = 1e-3
MAX_LOOSE = 30

# decisions of ScreenPhase.decide
FULL, REBUILD, LOOSE_INC, TIGHT_INC = 'full', 'rebuild', 'loose', 'tight'


class ScreenPhase:
    """Per-molecule state of the schedule (fastscfscreen.py:97-127).

    ``decide(incremental, step)`` returns what this cycle's build is:
    FULL (the first build of a run, or a caller's own full build: tight,
    from scratch; it starts the loose phase), REBUILD (the switch: tight,
    from scratch), LOOSE_INC (incremental at the loose threshold) or
    TIGHT_INC (incremental at the tight one).  ``step`` is a number or a
    function returning one; it is evaluated only in the loose phase."""

    def __init__(self, loose=LOOSE, switch=SWITCH, max_loose=MAX_LOOSE):
        self.loose = float(loose)
        self.switch = float(switch)
        self.max_loose = int(max_loose)
        self.phase = TIGHT_INC
        self.nloose = 0
        self.stats = {'loose_builds': 0, 'rebuilds': 0, 'tight_builds': 0, 'capped': 0}

    def decide(self, incremental, step):
        if not incremental:
            self.phase = LOOSE_INC
            self.nloose = 0
            self.stats['tight_builds'] += 1
            return FULL
        if self.phase == LOOSE_INC:
            capped = self.nloose >= self.max_loose
            if capped or (step() if callable(step) else step) < self.switch:
                self.phase = TIGHT_INC
                self.stats['rebuilds'] += 1
                self.stats['capped'] += int(capped)
                return REBUILD
            self.nloose += 1
            self.stats['loose_builds'] += 1
            return LOOSE_INC
        self.stats['tight_builds'] += 1
        return TIGHT_INC

    def tol(self, decision, tight):
        """The screening threshold of a build of this decision."""
        return max(float(tight), self.loose) if decision == LOOSE_INC else float(tight)


def ovlp_sqrt(S):
    """S^1/2 of a symmetric positive (semi)definite overlap (torch tensor)."""
    import torch
    w, u = torch.linalg.eigh(S)
    return (u * torch.sqrt(torch.clamp(w, min=0.0))) @ u.transpose(-1, -2)


def density_step(dm, dm_last, x=None):
    """max |x (dm - dm_last) x| with x = S^1/2, or max |dm - dm_last|."""
    d = dm - dm_last
    if x is not None and x.shape[-1] == d.shape[-1]:
        d = x @ d @ x
    return float(d.abs().max())


class LooseTightJK:
    """Incremental J/K of one molecule under the loose-then-tight schedule.

    ``jk(dm)`` is called once per cycle with the cycle's densities (n_dm,
    nao, nao), hermi = 1; the first call (or any call after ``reset()``) is
    a full build.  Returns (vj, vk) of dm; ``decisions`` records each
    cycle's build."""

    def __init__(self, opt, ovlp=None, loose=LOOSE, switch=SWITCH, max_loose=MAX_LOOSE,
                 mixed_threshold=0.0):
        self.opt = opt
        self.tight = float(opt.direct_scf_tol)
        self.x = ovlp_sqrt(ovlp) if ovlp is not None else None
        self.state = ScreenPhase(loose, switch, max_loose)
        self.mixed_threshold = mixed_threshold
        self.decisions = []
        self.reset()

    def reset(self):
        self.dm_last = self.vj = self.vk = None

    def jk(self, dm):
        inc = self.dm_last is not None
        d = self.state.decide(inc, lambda: density_step(dm, self.dm_last, self.x))
        self.decisions.append(d)
        self.opt.direct_scf_tol = self.state.tol(d, self.tight)
        try:
            if d in (FULL, REBUILD):
                self.vj, self.vk = self.opt.get_jk(dm, 1, mixed_threshold=self.mixed_threshold)
            else:
                vj, vk = self.opt.get_jk(dm - self.dm_last, 1,
                                         mixed_threshold=self.mixed_threshold)
                self.vj = self.vj + vj
                self.vk = self.vk + vk
        finally:
            self.opt.direct_scf_tol = self.tight
        self.dm_last = dm.clone()
        return self.vj, self.vk
