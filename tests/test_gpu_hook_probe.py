"""Hook invocation counts, as the reference's HookProbeMethod test
(test/test_capturing.jl:44-61): residual! runs preprocess_state! once, every
SSP-RK stage runs it once, and post_step! runs once per completed step.  The
counts are kept on the device (frg_solve_hook_calls), so steps replayed from
CUDA graphs and batched steps are counted as well.
"""
import pytest

import frforge_b200 as F
from frforge_b200.batch import Batch

from pairs import pair_1d, pair_2d, smooth_state_2d

pytestmark = pytest.mark.gpu

PRE = ("preprocess_state", "preprocess_positivity_zhang_shu", (1e-13, 1e-13))
POST = ("post_step", "positivity_zhang_shu", (1e-13, 1e-13))


def _probe(state, eq, method=None):
    s = F.GpuSolve(state, eq, method or F.PerssonAVMethod())
    s.set_hook(*PRE)
    s.set_hook(*POST)
    return s


def test_residual_and_sense_each_make_one_work_state():
    orc, state, _ = pair_2d(p=2, nx=8, ny=6, flux="hllc", method="persson")
    s = _probe(state, F.Euler2D(1.4))
    assert s.hook_calls() == {"post_step": 0, "numerical_flux_method": None, "extrapolate_interface": None, "preprocess_state": 0}
    s.upload(smooth_state_2d(orc), 0.0)
    s.residual()
    assert s.hook_calls()["preprocess_state"] == 1
    s.sense()
    assert s.hook_calls() == {"post_step": 0, "numerical_flux_method": None, "extrapolate_interface": None, "preprocess_state": 2}
    s.apply_post_step()
    assert s.hook_calls()["post_step"] == 1
    s.close()


@pytest.mark.parametrize("time,stages", [("ssp_rk3", 3), ("ssp_rk2", 2)])
def test_steps_count_one_work_state_per_stage_and_one_post_step_per_step(time, stages):
    orc, state, _ = pair_2d(p=3, nx=10, ny=8, flux="hllc", time=time, method="persson")
    s = _probe(state, F.Euler2D(1.4))
    s.upload(smooth_state_2d(orc), 0.0)
    r = s.advance(0.05, cfl=0.2)
    assert r["status"] == "ok" and r["n_steps"] > 3
    calls = s.hook_calls()
    assert calls["preprocess_state"] == stages * r["n_steps"]
    assert calls["post_step"] == r["n_steps"]
    assert s.info()["residual_evals"] == stages * r["n_steps"]
    # a fixed-dt run that stops on max_steps, then host-driven steps
    r2 = s.advance(1.0, dt=1e-4, max_steps=5)
    assert r2["n_steps"] == 5
    s.step(1e-4)
    n = r["n_steps"] + 6
    assert s.hook_calls() == {"post_step": n, "numerical_flux_method": None, "extrapolate_interface": None, "preprocess_state": stages * n}
    s.close()


def test_1d_counts_and_the_inline_flux_override():
    orc, state, _ = pair_1d(p=3, nel=32, flux="hllc", method="persson")
    orc.ic_sod()
    s = _probe(state, F.Euler1D(1.4), F.FluxOverridePersson(flux="rusanov", alpha=0.9))
    s.upload(orc.u.copy(), 0.0)
    r = s.advance(0.02, cfl=0.1)
    assert r["status"] == "ok"
    assert s.hook_calls() == {"post_step": r["n_steps"], "numerical_flux_method": None, "extrapolate_interface": None,
                              "preprocess_state": 3 * r["n_steps"]}
    assert s.info()["residual_evals"] == 3 * r["n_steps"]
    s.close()


def test_batched_post_step_counts_per_instance():
    b = Batch(capacity=2)
    slots, steps = [], []
    for nx, t_final in ((8, 0.02), (12, 0.04)):
        orc, state, _ = pair_2d(p=2, nx=nx, ny=nx, method="persson")
        i = b.add(state, F.Euler2D(1.4), F.PositivityPreservingPersson())
        b.upload(i, smooth_state_2d(orc), 0.0)
        b.start(i, t_final, cfl=0.2)
        slots.append(i)
    res = b.run()
    for i in slots:
        assert res[i]["status"] == "ok"
        assert b.hook_calls(i)["post_step"] == res[i]["n_steps"]
    b.close()
