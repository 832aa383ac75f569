"""The outer loop's control logic on the CPU, with a scripted iteration in place of the device
one: stopping rules, time-step schedules, the BDF levels each step sees, callbacks."""

from types import SimpleNamespace

import pytest
import torch

from zvcfd_b200.solver import B200Solver, time_steps


def _rec(du=1.0, dp=1.0, rms=1.0, lin=True):
    return {"du": du, "dp": dp, "rms_u": rms, "rms_v": rms, "rms_w": rms, "rms_p": rms,
            "linear_converged": lin, "linear_iterations": 3, "linear_residual": 0.05,
            "seconds": 0.0}


def _solver(script):
    """A ``B200Solver`` whose ``iterate`` replays ``script`` (a record, or a function of the
    solver returning one) and notes the time level it ran at."""
    s = object.__new__(B200Solver)
    s._lumped, s.t, s._time, s.iteration = {}, 0.0, None, 0
    s.U = torch.zeros((4, 3), dtype=torch.float64)
    s.mdot = {"tet": torch.zeros((2, 4), dtype=torch.float64)}
    s.seen, s.bc_times = [], []
    s.bc = SimpleNamespace(update=s.bc_times.append)
    s._refresh_boundary = s._apply_fixed = lambda: None
    s.patch_flows = dict
    it = iter(script)

    def iterate():
        r = next(it)
        r = dict(r(s) if callable(r) else r)
        s.iteration += 1
        r["iteration"] = s.iteration
        s.seen.append(None if s._time is None else (s.t, s._time[1], s._time[3]))
        return r

    s.iterate = iterate
    return s


def test_steady_convergence_needs_two_iterations_and_a_converged_linear_solve():
    s = _solver([_rec(1e-12, 1e-12), _rec(1e-12, 1e-12, lin=False), _rec(1e-12, 1e-12)])
    rep = s.solve(max_iterations=10, tol=1e-10)
    assert rep["converged"] and rep["iterations"] == 3
    s = _solver([_rec(1e-3, 1e-3)] * 4)
    rep = s.solve(max_iterations=4, tol=1e-10)
    assert not rep["converged"] and rep["iterations"] == 4


def test_residual_target_stops_the_iterations():
    s = _solver([_rec(rms=1e-3), _rec(rms=1e-3), _rec(rms=1e-7)])
    rep = s.solve(max_iterations=10, tol=1e-12, residual_target=1e-6)
    assert rep["converged"] and rep["iterations"] == 3


def test_variable_steps_reach_the_bdf_levels_and_the_boundary_at_each_time():
    s = _solver([_rec(1e-12, 1e-12)] * 12)
    got = []
    rep = s.solve_transient([0.1, 0.2, 0.05], scheme="bdf2", loops=4, tol=1e-10,
                            callback=lambda sv, dt: got.append((sv.t, dt)))
    assert rep["converged"] and rep["iterations"] == 6          # two loops per step
    assert s.bc_times == pytest.approx([0.1, 0.3, 0.35])
    assert [g[1] for g in got] == [0.1, 0.2, 0.05]
    # (time, this step, previous step) seen by each loop: the variable-step BDF2 inputs
    assert [t for t, _, _ in s.seen] == pytest.approx([0.1] * 2 + [0.3] * 2 + [0.35] * 2)
    assert [(h, prev) for _, h, prev in s.seen] == [(0.1, None)] * 2 + [(0.2, 0.1)] * 2 + \
        [(0.05, 0.2)] * 2
    assert all("t" in r for r in rep["history"]) and s._time is None


def test_a_step_whose_loops_run_out_is_reported():
    s = _solver([_rec(1e-12, 1e-12)] * 2 + [_rec(1e-3, 1e-3)] * 3)
    seen = []
    rep = s.solve_transient(0.5, 2, loops=3, tol=1e-10, callback=seen.append)
    assert not rep["converged"] and rep["iterations"] == 5 and len(seen) == 2


def test_time_step_schedules():
    assert list(time_steps(0.25, 3, 0.0)) == [0.25] * 3
    assert list(time_steps([0.1, 0.2, 0.3], None, 0.0)) == [0.1, 0.2, 0.3]
    assert list(time_steps([0.1, 0.2, 0.3], 2, 0.0)) == [0.1, 0.2]
    assert list(time_steps(lambda t: 0.1 if t < 0.25 else 0.2, 4, 0.0)) == \
        pytest.approx([0.1, 0.1, 0.1, 0.2])
    with pytest.raises(ValueError):
        list(time_steps(0.1, None, 0.0))
    with pytest.raises(ValueError):
        list(time_steps(lambda t: 0.1, None, 0.0))
