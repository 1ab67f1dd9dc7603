"""Small 1D solves (at most 8 tiles of 64 elements) advance through
loop1d_kernel: one thread-block cluster runs K steps of the time loop per
launch.  Its steps agree with the per-stage launches (frg_time_stages runs
the same steps one kernel per stage) to rounding -- the compiler fuses a few
multiply-adds differently in the two kernels, so the bar is 1e-11 relative
L-infinity with identical step counts, times and status -- for every scheme,
method and size up to the cluster limit; a larger mesh keeps the step
graphs."""
import numpy as np
import pytest

import frforge_b200 as F

from pairs import pair_1d, rel_linf

pytestmark = pytest.mark.gpu

CASES = [
    # (builder kwargs, IC, steps, dt)
    (dict(p=3, nel=256, method="persson"), "sod", 150, None),                         # C1-like
    (dict(p=2, nel=100, flux="hllc", time="ssp_rk2", method="persson", left="periodic",
          right="periodic"), "wave", 90, None),
    (dict(p=5, nel=500, method="persson", av_form="element_local_DD"), "shu", 40, None),  # 8 tiles
    (dict(p=1, nel=30, method="null"), "sod", 70, 2e-3),                                # fixed dt
    (dict(p=4, nel=600, flux="hllc", method="persson"), "sod", 20, None),              # 10 tiles: graphs
]


def _ic(orc, name):
    if name == "sod":
        orc.ic_sod()
    elif name == "shu":
        orc.ic_shu_osher()
    else:
        orc.ic_density_wave()
    return orc.u.copy()


@pytest.mark.parametrize("k", range(len(CASES)))
def test_advance_equals_per_stage_launches(k):
    kw, ic, steps, dt = CASES[k]
    orc, state, solve = pair_1d(**kw)
    u0 = _ic(orc, ic)
    solve.upload(u0, 0.0)
    r_loop = solve.advance(1e9, cfl=0.15, dt=dt, max_steps=steps)
    u_loop, t_loop = solve.download()
    solve.upload(u0, 0.0)
    r_again = solve.advance(1e9, cfl=0.15, dt=dt, max_steps=steps)
    u_again, _ = solve.download()
    solve.upload(u0, 0.0)
    _, r_launch = solve.time_stages(steps, cfl=0.15, dt=dt)
    u_launch, t_launch = solve.download()
    assert r_loop["status"] == r_launch["status"] == "max_steps"
    assert r_loop["n_steps"] == r_launch["n_steps"] == steps
    # deterministic run to run
    assert r_again == r_loop and np.array_equal(u_again, u_loop)
    assert np.all(np.isfinite(u_loop))
    # the same steps as the launched kernels up to the compiler's choice of
    # fused multiply-adds in the two kernels
    dev = rel_linf(u_loop, u_launch)
    print(f"case {k}: t {t_loop!r} vs {t_launch!r}, rel Linf {dev:.3e}, "
          f"points differing {int(np.sum(u_loop != u_launch))} of {u_loop.size}")
    assert t_loop == pytest.approx(t_launch, rel=1e-13)
    assert dev <= 1e-11


def test_finished_run_and_restart():
    # a run that reaches t_final inside a launch stops there (the last step
    # clipped), and a second advance continues from the stored state
    orc, state, solve = pair_1d(p=3, nel=128, method="persson")
    solve.upload(_ic(orc, "sod"), 0.0)
    r = solve.advance(0.01, cfl=0.15)
    assert r["status"] == "ok" and r["t"] == pytest.approx(0.01, abs=1e-15) and r["n_steps"] > 1
    r2 = solve.advance(0.02, cfl=0.15)
    assert r2["status"] == "ok" and r2["t"] == pytest.approx(0.02, abs=1e-15) and r2["n_steps"] > 1
    u, t = solve.download()
    assert t == r2["t"] and np.all(np.isfinite(u))
