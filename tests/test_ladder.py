"""The linear-solver ladder's switching rules (the reference's ``Auto``), with stand-in solvers
on the CPU: failures, near misses, non-finite answers, exceptions and the timed probe."""

import pytest
import torch

from zvcfd_b200.linear import Ladder, SolveInfo


class Clock:
    def __init__(self):
        self.t = 0.0

    def __call__(self):
        return self.t


class Fake:
    """A solver whose k-th solve returns ``script[k]``: ``(residual, converged, seconds)``, or
    ``"nan"`` / ``"raise"``; ``x`` is filled with the solver's tag."""

    made = []

    def __init__(self, tag, script, clock):
        self.tag, self.script, self.clock, self.calls, self.closed = tag, list(script), clock, 0, False
        Fake.made.append(self)

    def solve(self, A, b, x0=None, rtol=None):
        step = self.script[min(self.calls, len(self.script) - 1)]
        self.calls += 1
        if step == "raise":
            raise RuntimeError(f"{self.tag} set-up failed")
        x = torch.full((8,), float(self.tag[-1]), dtype=torch.float64)
        if step == "nan":
            x[3] = float("nan")
            return x, SolveInfo(200, float("nan"), 0.0)
        res, ok, sec = step
        self.clock.t += sec
        return x, SolveInfo(5, res, sec, 0.0, ok)

    def close(self):
        self.closed = True


def ladder(scripts, **kw):
    clock = Clock()
    Fake.made = []
    rungs = [(f"r{i}", (lambda i=i, s=s: Fake(f"r{i}", s, clock))) for i, s in enumerate(scripts)]
    return Ladder(rungs, rtol=0.1, clock=clock, **kw), clock


B = torch.zeros(8, dtype=torch.float64)


def test_a_failure_resolves_the_same_system_with_the_next_rung_and_keeps_it():
    lad, _ = ladder([[(5.0, False, 1.0)], [(0.05, True, 1.0)]], probe_at=None)
    x, info = lad.solve(None, B)
    assert info.converged and float(x[0]) == 1.0
    assert lad.active == "r1" and len(lad.switches) == 1
    assert lad.switches[0][:2] == ("r0", "r1") and "residual 5.0e+00" in lad.switches[0][2]
    assert Fake.made[0].closed
    lad.solve(None, B)
    assert lad.active == "r1" and Fake.made[1].calls == 2


def test_a_near_miss_is_accepted_unconverged():
    lad, _ = ladder([[(0.5, False, 1.0)], [(0.05, True, 1.0)]], probe_at=None)
    x, info = lad.solve(None, B)                # 0.5 <= fail_ratio (10) x rtol (0.1)
    assert not info.converged and lad.active == "r0" and not lad.switches


@pytest.mark.parametrize("bad", ["nan", "raise"])
def test_non_finite_answers_and_exceptions_are_failures(bad):
    lad, _ = ladder([[bad], [(0.05, True, 1.0)]], probe_at=None)
    x, info = lad.solve(None, B)
    assert info.converged and lad.active == "r1"
    why = lad.switches[0][2]
    assert ("non-finite" in why) if bad == "nan" else ("set-up failed" in why)


def test_when_every_rung_fails():
    lad, _ = ladder([["raise"], ["nan"]], probe_at=None)
    with pytest.raises(RuntimeError, match="every linear solver failed"):
        lad.solve(None, B)
    lad, _ = ladder([["raise"], [(5.0, False, 1.0)]], probe_at=None)
    x, info = lad.solve(None, B)                # finite: the last rung's answer is returned
    assert not info.converged and float(x[0]) == 1.0


def test_the_probe_keeps_a_faster_rung_and_returns_when_it_fails():
    lad, clock = ladder([[(0.05, True, 1.0)], [(0.05, True, 0.5), (5.0, False, 0.5)],
                         [(0.05, True, 9.0)]], probe="r1", probe_at=2, probe_margin=0.8)
    lad.solve(None, B)
    assert lad.active == "r0" and lad.probe is None
    x, info = lad.solve(None, B)                # the probe: 0.5 s against 1.0 s
    assert lad.active == "r1" and float(x[0]) == 1.0
    assert lad.probe == {"first_s": 1.0, "probe_s": 0.5, "probe_converged": True}
    assert lad.switches[-1][2].startswith("probe:")
    x, info = lad.solve(None, B)                # the probed rung fails: back to r0, not r2
    assert lad.active == "r0" and float(x[0]) == 0.0 and info.converged
    assert lad.switches[-1][:2] == ("r1", "r0")
    assert lad.switches[-1][2].startswith("probed solver failed")


def test_a_slower_probe_is_dropped():
    lad, _ = ladder([[(0.05, True, 1.0)], [(0.05, True, 0.9)]], probe="r1", probe_at=1,
                    probe_margin=0.8)
    x, _ = lad.solve(None, B)
    assert lad.active == "r0" and float(x[0]) == 0.0 and not lad.switches
    assert lad.probe["probe_s"] == pytest.approx(0.9) and Fake.made[-1].closed


def test_the_device_ladder_is_named_like_the_reference():
    from zvcfd_b200 import linear

    with pytest.raises(ValueError, match="b200-auto"):
        linear.make("amgx")
    assert Ladder.name == "auto"


def test_presets_restate_the_reference_amgx_presets():
    """``B200AMG(preset=...)`` takes the reference's AmgX preset names and sets the smoother,
    sweeps and relaxation of each; explicit arguments win."""
    from zvcfd_b200.linear import PRESETS, B200AMG

    assert set(PRESETS) == {"gs", "robust", "dilu-p", "dilu"}
    want = {"gs": ("gs", 1, 2), "robust": ("ilu0", 1, 1), "dilu-p": ("dilu", 1, 2),
            "dilu": ("dilu", 1, 2)}
    for name, (smoother, pre, post) in want.items():
        a = B200AMG(preset=name)
        assert (a.smoother, a.presweeps, a.postsweeps) == (smoother, pre, post), name
        a.close()
    a = B200AMG(preset="robust", smoother="gs")
    assert a.smoother == "gs"
    a.close()
    try:
        B200AMG(preset="nope")
    except ValueError as e:
        assert "preset" in str(e)
    else:
        raise AssertionError("an unknown preset is accepted")
