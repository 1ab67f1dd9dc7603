"""Batched execution (frg_batch_*).

* An instance's result does not depend on the rest of the batch: every
  instance of a mixed batch, including ones that join or leave between runs,
  ends bit-identical to the same instance run alone in a batch.
* The batched kernels agree with the single-solve path (frg_advance, itself
  checked against the oracle in test_gpu_parity.py) to 1e-10 relative L-inf
  with identical status and step count.  They are not bitwise equal to it:
  the two kernels read the mesh and stage descriptors from different memory
  (shared memory vs kernel parameters), so the compiler fuses a few
  multiply-adds differently.
* Instances large enough to fill the device alone (a full wave of batched
  tiles) run solo inside the batch, through the single-solve stage kernels:
  they end bit-identical to the single-solve path.
* One batched instance is checked against the oracle directly."""
import numpy as np
import pytest

import frforge_b200 as F
from frforge_b200 import _lib as L
from frforge_b200.batch import Batch, solve_bytes

from pairs import (four_quadrant_state, pair_1d, pair_2d, prim2cons1, rel_linf, smooth_state_2d)

pytestmark = pytest.mark.gpu


def _sod(orc):
    orc.ic_sod()
    return orc.u.copy()


# (builder kwargs, IC, run arguments)
MIX = [
    (dict(dim=2, p=1, nx=12, ny=12, flux="rusanov", method="persson"), "smooth",
     dict(t_final=1.0, cfl=0.1, max_steps=40)),
    (dict(dim=2, p=3, nx=20, ny=20, flux="hllc", method="persson", bcs=("transmissive",) * 4), "quad",
     dict(t_final=1.0, cfl=0.1, max_steps=35)),
    (dict(dim=2, p=3, nx=13, ny=9, flux="hllc", method="persson", bcs=("transmissive",) * 4), "quad",
     dict(t_final=0.02, cfl=0.1, max_steps=1000)),
    (dict(dim=2, p=4, nx=10, ny=14, flux="rusanov", time="ssp_rk2", method="persson",
          av_form="element_local_DD"), "smooth", dict(t_final=0.03, dt=1e-3, max_steps=1000)),
    (dict(dim=2, p=5, nx=8, ny=8, flux="rusanov", method="null"), "smooth",
     dict(t_final=1.0, cfl=0.1, max_steps=25)),
    (dict(dim=2, p=2, nx=12, ny=12, flux="rusanov", method="persson", wavy=1), "smooth",
     dict(t_final=1.0, cfl=0.1, max_steps=30)),
    (dict(dim=2, p=2, nx=16, ny=8, flux="hllc", method="persson",
          bcs=("reflecting", "transmissive", ("dirichlet", (1.0, 0.3, 0.0, 2.0)), "reflecting")), "quad",
     dict(t_final=1.0, cfl=0.1, max_steps=30)),
    (dict(dim=1, p=2, nel=64, method="persson"), "sod", dict(t_final=0.05, cfl=0.15, max_steps=10**6)),
    (dict(dim=1, p=3, nel=100, time="ssp_rk2", method="null", left="periodic", right="periodic"),
     "wave1d", dict(t_final=1.0, cfl=0.1, max_steps=45)),
]


def _build(kw):
    kw = dict(kw)
    dim = kw.pop("dim")
    return (pair_2d if dim == 2 else pair_1d)(**kw)


def _ic(orc, name, seed):
    if name == "smooth":
        return smooth_state_2d(orc, seed=seed)
    if name == "quad":
        return four_quadrant_state(orc, seed=seed, jump_scale=0.25)
    if name == "sod":
        return _sod(orc)
    x = orc.coords()
    return prim2cons1(1.0 + 0.2 * np.sin(2 * np.pi * x), 1.0 + 0 * x, 1.0 + 0 * x)


def _run_alone(solve, u0, run):
    solve.upload(u0, 0.0)
    r = solve.advance(run["t_final"], cfl=run.get("cfl", 0.2), dt=run.get("dt"), max_steps=run["max_steps"])
    u, t = solve.download()
    return r, u, t


def _close(u, u_ref, tol=1e-10):
    nan = np.isnan(u_ref)
    assert np.array_equal(np.isnan(u), nan)
    if nan.all():
        return
    assert rel_linf(np.where(nan, 0.0, u), np.where(nan, 0.0, u_ref)) <= tol


def _solo(state, kw, run):
    """The instance run alone in a batch: the bitwise reference of the mix."""
    b = Batch(capacity=1)
    i = b.add(state, _eq(kw), _method(kw))
    b.start(i, run["t_final"], cfl=run.get("cfl", 0.2), dt=run.get("dt"), max_steps=run["max_steps"])
    r = b.run()[i]
    u, t = b.download(i)
    b.close()
    return r, u, t


def _setup(cases, seed0=11):
    out = []
    for k, (kw, ic, run) in enumerate(cases):
        orc, state, solve = _build(kw)
        u0 = _ic(orc, ic, seed0 + k)
        state.u[...] = u0
        state.t = 0.0
        out.append((orc, state, solve, u0, run, kw))
    return out


def _method(kw):
    if kw.get("method", "null") == "null":
        return F.NullCapturing()
    return F.PerssonAVMethod(c_av=kw.get("c_av", 0.1), av_form=kw.get("av_form", "conservative_br0"))


def _eq(kw):
    return F.Euler2D(1.4) if kw["dim"] == 2 else F.Euler1D(1.4)


def test_batch_mix_matches_solo_bitwise_and_single_path():
    items = _setup(MIX)
    single = [_run_alone(solve, u0, run) for (_, _, solve, u0, run, _) in items]
    solo = [_solo(state, kw, run) for (_, state, _, _, run, kw) in items]
    b = Batch(capacity=len(items) + 3)
    slots = []
    for (orc, state, solve, u0, run, kw) in items:
        i = b.add(state, _eq(kw), _method(kw))
        b.start(i, run["t_final"], cfl=run.get("cfl", 0.2), dt=run.get("dt"), max_steps=run["max_steps"])
        slots.append(i)
    res = b.run()
    assert b.n_running == 0
    for k, i in enumerate(slots):
        r = res[i]
        u, t = b.download(i)
        # in the mix == alone in a batch, bit for bit
        r_solo, u_solo, t_solo = solo[k]
        assert r == r_solo, k
        assert t == t_solo and np.array_equal(u, u_solo), k
        # == the single-solve path to 1e-10
        r_one, u_one, t_one = single[k]
        assert r["status"] == r_one["status"] and r["n_steps"] == r_one["n_steps"], k
        assert t == pytest.approx(t_one, rel=1e-13, abs=1e-15), k
        _close(u, u_one)
    # empty slots report None
    assert all(res[k] is None for k in range(len(items), len(items) + 3))
    b.close()


def test_large_instances_run_solo_bitwise_equal_to_single_path():
    # 200^2 P=3 RK3 (1,250 batched 8x4 tiles) and 200^2 P=2 RK2 (625 8x8
    # tiles) fill a wave of 296 resident tiles and run solo; the 12^2
    # instance is batched beside them
    cases = [
        (dict(dim=2, p=3, nx=200, ny=200, flux="hllc", method="persson", bcs=("transmissive",) * 4), "quad",
         dict(t_final=1.0, cfl=0.1, max_steps=6)),
        (dict(dim=2, p=2, nx=200, ny=200, flux="rusanov", time="ssp_rk2", method="persson"), "smooth",
         dict(t_final=1.0, cfl=0.1, max_steps=5)),
        (dict(dim=2, p=3, nx=12, ny=12, flux="hllc", method="persson", bcs=("transmissive",) * 4), "quad",
         dict(t_final=1.0, cfl=0.1, max_steps=9)),
    ]
    items = _setup(cases, seed0=40)
    single = [_run_alone(solve, u0, run) for (_, _, solve, u0, run, _) in items]
    solo_small = _solo(items[2][1], items[2][5], items[2][4])
    b = Batch(capacity=3)
    slots = []
    for (orc, state, solve, u0, run, kw) in items:
        i = b.add(state, _eq(kw), _method(kw))
        b.start(i, run["t_final"], cfl=run.get("cfl", 0.2), dt=run.get("dt"), max_steps=run["max_steps"])
        slots.append(i)
    res = b.run()
    for k in (0, 1):
        u, t = b.download(slots[k])
        r_one, u_one, t_one = single[k]
        assert res[slots[k]]["status"] == r_one["status"] == "max_steps", k
        assert res[slots[k]]["n_steps"] == r_one["n_steps"], k
        assert t == t_one, k
        assert np.array_equal(u, u_one), (k, int(np.sum(u != u_one)), float(np.max(np.abs(u - u_one))))
    u, t = b.download(slots[2])
    assert res[slots[2]] == solo_small[0] and t == solo_small[2] and np.array_equal(u, solo_small[1])
    b.close()


def test_batched_instance_matches_oracle():
    # Sod P=2 Ne=64 with Persson AV to t = 0.2, inside a batch with a 2D case
    orc, state, solve = pair_1d(p=2, nel=64, method="persson", c_av=0.1)
    u0 = _sod(orc)
    r_ref = orc.integrate(0.2, cfl=0.15)
    o2, st2, _ = pair_2d(p=3, nx=12, ny=12, flux="hllc", method="persson", bcs=("transmissive",) * 4)
    st2.u[...] = four_quadrant_state(o2, jump_scale=0.25)
    b = Batch(capacity=2)
    state.u[...] = u0
    i = b.add(state, F.Euler1D(1.4), F.PerssonAVMethod(c_av=0.1))
    j = b.add(st2, F.Euler2D(1.4), F.PerssonAVMethod(c_av=0.1))
    b.start(i, 0.2, cfl=0.15)
    b.start(j, 1.0, cfl=0.1, max_steps=20)
    res = b.run()
    assert res[i]["status"] == "ok" and res[i]["n_steps"] == r_ref["n_steps"] == 950
    assert res[j]["status"] == "max_steps" and res[j]["n_steps"] == 20
    u, t = b.download(i)
    assert t == pytest.approx(0.2, abs=1e-15)
    assert np.sum(np.abs(u - orc.u)) / np.sum(np.abs(orc.u)) <= 1e-8
    b.close()


def test_continuous_batching_add_remove_midrun():
    # instances join and leave between runs; each still ends bit-identical to
    # its run alone
    cases = [MIX[0], MIX[1], MIX[4], MIX[7], MIX[3]]
    items = _setup(cases, seed0=31)
    solo = [_solo(state, kw, run) for (_, state, _, _, run, kw) in items]
    b = Batch(capacity=3)

    def add_start(k):
        orc, state, solve, u0, run, kw = items[k]
        i = b.add(state, _eq(kw), _method(kw))
        b.start(i, run["t_final"], cfl=run.get("cfl", 0.2), dt=run.get("dt"), max_steps=run["max_steps"])
        return i

    def check(k, i, res):
        r_solo, u_solo, t_solo = solo[k]
        assert res[i] == r_solo, k
        u, t = b.download(i)
        assert t == t_solo and np.array_equal(u, u_solo), k

    s0, s1 = add_start(0), add_start(1)
    res = b.run(max_steps=7)
    assert res[s0]["status"] == "running" and res[s0]["n_steps"] == 7
    s2 = add_start(2)  # joins a running batch
    res = b.run(max_steps=5)
    assert res[s2]["n_steps"] == 5 and res[s0]["n_steps"] == 12
    with pytest.raises(F.FRGError):
        add_start(3)  # capacity 3: full
    res = b.run()
    for k, i in ((0, s0), (1, s1), (2, s2)):
        check(k, i, res)
    b.remove(s1)
    s3 = add_start(3)  # reuses the freed slot
    assert s3 == s1
    b.remove(s0)
    s4 = add_start(4)
    res = b.run()
    check(3, s3, res)
    check(4, s4, res)
    check(2, s2, res)  # a finished instance is left untouched by later runs
    b.close()


def test_divergent_instance_does_not_disturb_others():
    items = _setup([MIX[0], MIX[7], MIX[4]], seed0=51)
    # poison instance 1 (1D Sod) with a NaN
    bad = items[1][3].copy()
    bad[1, 5, 0] = np.nan
    items[1] = items[1][:3] + (bad,) + items[1][4:]
    items[1][1].u[...] = bad
    single = [_run_alone(solve, u0, run) for (_, _, solve, u0, run, _) in items]
    assert single[1][0]["status"] == "diverged"
    solo = [_solo(state, kw, run) for (_, state, _, _, run, kw) in items]
    b = Batch(capacity=3)
    slots = []
    for (orc, state, solve, u0, run, kw) in items:
        i = b.add(state, _eq(kw), _method(kw))
        b.start(i, run["t_final"], cfl=run.get("cfl", 0.2), dt=run.get("dt"), max_steps=run["max_steps"])
        slots.append(i)
    res = b.run()
    for k, i in enumerate(slots):
        r_one = single[k][0]
        assert res[i]["status"] == r_one["status"] and res[i]["n_steps"] == r_one["n_steps"]
        assert res[i] == solo[k][0]
        u, t = b.download(i)
        assert t == solo[k][2]
        assert np.array_equal(u, solo[k][1], equal_nan=True)
        _close(u, single[k][1])
    b.close()


def test_hbm_budget_admission():
    orc, state, solve = pair_2d(p=3, nx=32, ny=32, method="persson")
    need = solve_bytes(state, F.Euler2D(1.4), F.PerssonAVMethod())
    assert need >= solve.info()["device_bytes"]
    b = Batch(capacity=8, hbm_budget=int(2.5 * need))
    b.add(state, F.Euler2D(1.4), F.PerssonAVMethod())
    b.add(state, F.Euler2D(1.4), F.PerssonAVMethod())
    with pytest.raises(F.FRGError) as e:
        b.add(state, F.Euler2D(1.4), F.PerssonAVMethod())
    assert e.value.code == L.FRG_ERR_OOM
    b.remove(0)
    b.add(state, F.Euler2D(1.4), F.PerssonAVMethod())  # room again
    b.close()


def test_start_without_state_and_bad_slot():
    orc, state, solve = pair_2d(p=2, nx=8, ny=8)
    b = Batch(capacity=2)
    with pytest.raises(ValueError):
        b.start(1, 1.0)
    with pytest.raises(ValueError):
        b.remove(0)
    i = b.add(state, F.Euler2D(1.4))
    with pytest.raises(ValueError):
        b.start(i, 1.0, cfl=0.0)
    res = b.run()  # nothing running: returns at once
    assert res[i]["status"] in ("ok", "max_steps") and b.n_running == 0
    b.close()


def test_autotune_table_selects_solve_and_group_variants():
    # a table entry for (P=3, HLLC, BR0, affine) sets the variant of a new
    # solve and of the batched group that runs such instances; results stay
    # within the batched bar of the oracle-checked single-solve path
    from frforge_b200 import autotune as T

    T.clear()
    try:
        T.set_variant(3, "hllc", "br0", False, 2)
        kw = dict(p=3, nx=20, ny=20, flux="hllc", method="persson", bcs=("transmissive",) * 4)
        orc, state, solve = pair_2d(**kw)
        assert solve.variant()[0] == 2
        u0 = four_quadrant_state(orc, jump_scale=0.25)
        run = dict(t_final=1.0, cfl=0.1, max_steps=20)
        r_ref, u_ref, t_ref = _run_alone(solve, u0, run)
        # the same run with the default batched tile
        T.clear()
        outs = []
        for v in (None, 2):
            if v is not None:
                T.set_variant(3, "hllc", "br0", False, v)
            b = Batch(capacity=2)
            i = b.add(state, F.Euler2D(1.4), F.PerssonAVMethod(c_av=0.1))
            b.upload(i, u0, 0.0)
            b.start(i, run["t_final"], cfl=run["cfl"], max_steps=run["max_steps"])
            res = b.run()
            assert b.group_of(i) == ((-1 if v is None else v), False)
            assert res[i]["status"] == r_ref["status"] and res[i]["n_steps"] == r_ref["n_steps"]
            outs.append(b.download(i)[0])
            b.close()
        for u in outs:
            assert rel_linf(u, u_ref) <= 1e-10
    finally:
        T.clear()
