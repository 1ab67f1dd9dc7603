"""Benchmark: FP64 DOF-stage updates/s of the FR residual + SSP-RK3 path.

Workload (default): 512^2 quads, GL P=3, HLLC, SSP-RK3, Persson AV (BR0,
c_av 0.1), transmissive, CFL 0.1, seeded four-quadrant IC (see
frforge_b200/workloads.py).  A "step" is one SSP-RK3 step = 3 stage
evaluations over all 512^2 x 16 x 4 = 16.8M degrees of freedom.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
  python bench.py --workload batched     # 64 mixed solves, batched vs one at a time
  python bench.py --workload served      # Poisson request trace, served vs one at a time
  python bench.py --workload c1          # the 1D 256-element case (launch-bound), steps/s
  python bench.py --ncu-target [--n 256] [--variant V] [--flux F] [--method M]
                                         # a few stage launches of the workload, for ncu

ours: value = DOF-stage/s with the state resident in HBM, timed with CUDA
events on the library's stream (max over ranks); e2e = the same metric through
the public C ABI with pinned host buffers (state upload + K steps + download
inside the timed region); roofline of the fused stage kernel from CUDA events
around every stage launch; cpu_baseline = the C oracle on a bounded sample.
reference: the reference algorithm on the host cores (the C oracle port, all
threads), each step one full SSP-RK3 step of the 512^2 workload.
Multi-GPU: replicas only (each rank runs its own solve, no data exchange).
The batched and served arms start from the committed B200 tile table
(frforge_b200/autotune_b200.json; --no-tune: default tiles).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "FP64 DOF-stage updates/s on 1 B200; batched solves/s + p99 latency vs plain"
UNIT = "DOF-stage/s"
# algorithmic HBM bytes per DOF per stage (SSP-RK3: 16, 24, 24 -> 64/3 avg)
STAGE_BYTES = (16.0, 24.0, 24.0)


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        time.sleep(0.15)
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.15)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = max(mx, float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def oracle_rate(n: int, steps: int, threads: int, min_seconds: float = 0.0):
    """DOF-stage/s of the C oracle on an n x n sample of the c3 workload."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from frforge_b200.workloads import C3, four_quadrant_ic, four_quadrant_states

    O.set_threads(threads)
    s = O.OracleSolver.two_d(p=C3.p, nx=n, ny=n, bcs=[O.make_bc("transmissive")] * 4, flux=C3.flux,
                             method="persson", c_av=C3.c_av)
    x, y = s.coords()
    s.set_state(four_quadrant_ic(x, y, four_quadrant_states(C3.seed, C3.jump_scale)))
    ndof = s.ndof
    s.integrate(1e9, cfl=C3.cfl, max_steps=1)  # warm the caches / thread pool
    done = 0
    t0 = time.perf_counter()
    while done < steps or (time.perf_counter() - t0) < min_seconds:
        r = s.integrate(1e9, cfl=C3.cfl, max_steps=1)
        if r["status"] == "diverged":
            raise RuntimeError("oracle sample diverged")
        done += 1
    dt = time.perf_counter() - t0
    return 3 * ndof * done / dt, done, dt


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    n = 512  # the workload itself: one full SSP-RK3 step of the 512^2 mesh per step
    oracle_rate(n, max(1, args.warmup), threads)
    rate, done, dt = oracle_rate(n, args.steps, threads)
    line = {
        "impl": "reference", "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * dt / done,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded four-quadrant Riemann IC)",
        "config": workload_config(args),
        "cpu_baseline": {"value": rate, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"{done} SSP-RK3 steps of the {n}^2 workload itself (one full step per "
                                   f"step); C oracle, OpenMP {threads} threads"},
        "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def workload_config(args):
    return {"workload": "2D Euler 512x512 quads, GL P=3, HLLC, SSP-RK3, Persson AV (BR0, c_av=0.1), "
                        "transmissive, CFL 0.1, seeded four-quadrant Riemann IC with each quadrant's "
                        "deviation from the four-state mean scaled by 0.25 (the unscaled draws make the "
                        "reference scheme diverge within 40 steps)",
            "ic_jump_scale": 0.25,
            "elements": 512 * 512, "p": 3, "dof": 512 * 512 * 16 * 4, "stages_per_step": 3,
            "l2": "inputs larger than L2 (3 x 134 MB state buffers)", "parallelism": f"replicas{args.gpus}"}


def _profile_summary():
    path = os.path.join(ROOT, "profiles", "stage2d_c3_traffic.json")
    if not os.path.exists(path):
        return {}
    with open(path) as f:
        return json.load(f)


def traffic_per_launch():
    """dram bytes per stage launch from the committed ncu summary, if any."""
    return _profile_summary().get("dram_bytes_per_launch_full_c3")


def issue_limiter():
    """The stage kernel's issue-side figures from the committed ncu summary:
    what bounds it below the HBM roofline."""
    d = _profile_summary().get("issue_256sq")
    if not d:
        return None
    return {"kind": "fp64 issue / latency", "fp64_pipe_busy": d["sm__pipe_fp64_cycles_active_pct"] / 100.0,
            "issue_active": d["smsp__issue_active_pct"] / 100.0,
            "warp_instructions_per_dof": d["warp_instructions_per_dof"],
            "source": "ncu, profiles/stage2d_c3_ncu.md"}


def max_over_ranks(ms: float, world: int, device: str) -> float:
    """The slowest rank's time (every rank gets it); device: where the
    process group's collectives run ("cuda" for NCCL, "cpu" for gloo)."""
    if world <= 1:
        return float(ms)
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def advance_launches(steps: int, ndof: int, loop1d: bool = False) -> int:
    """Kernels one frg_advance of `steps` SSP-RK3 steps launches: the prime
    pass, then graphs of K steps (K by state size, as run_steps picks it) of
    five kernels per step (begin, three stages, end); a 1D solve of at most 8
    tiles instead runs K steps per launch of the cluster loop kernel."""
    k = 4 if ndof > 4e6 else (16 if ndof > 2e5 else 64)
    return 1 + -(-steps // k) * (1 if loop1d else 5 * k)


def replica_rate(world: int, steps: int, ndof: int, ms_max: float) -> float:
    """Whole-job DOF-stage/s of `world` replicas that each ran `steps`
    SSP-RK3 steps (3 stages) of `ndof` DOF in at most ms_max."""
    return world * steps * 3 * ndof / (ms_max * 1e-3)


def run_ours(args):
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    import frforge_b200 as F
    from frforge_b200.workloads import C3

    ctx = F.Context(local)
    stream = torch.cuda.ExternalStream(ctx.stream_handle(), device=torch.device("cuda", local))
    st, method = C3.build(F)
    solve = F.GpuSolve(st, F.Euler2D(1.4), method, ctx=ctx)
    ndof = solve.ndof
    u_host = torch.empty(ndof, dtype=torch.float64, pin_memory=True)
    u_host.numpy()[:] = st.u.ravel(order="F")
    u_out = torch.empty(ndof, dtype=torch.float64, pin_memory=True)

    def barrier():
        if world > 1:
            dist.barrier()

    # warm-up (untimed): autotune the stage-kernel tile variant, then steps
    solve.upload(u_host.numpy().reshape(st.u.shape, order="F"), 0.0)
    variant, variant_ms = solve.autotune(reps=5)
    r = solve.advance(1e9, cfl=C3.cfl, max_steps=max(3, args.warmup))
    if r["status"] == "diverged":
        raise RuntimeError("warm-up diverged")

    # ---- device-resident timed region: K steps, events on the library stream
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        ev0.record(stream)
        r = solve.advance(1e9, cfl=C3.cfl, max_steps=args.steps)
        ev1.record(stream)
        torch.cuda.synchronize()
    barrier()
    if r["status"] != "max_steps" or r["n_steps"] != args.steps:
        raise RuntimeError(f"timed run ended early: {r}")
    ms_max = max_over_ranks(ev0.elapsed_time(ev1), world, "cuda")
    value = replica_rate(world, args.steps, ndof, ms_max)

    # ---- stage-kernel roofline: CUDA events around every stage launch
    nst = max(3, min(args.steps, 30))
    stage_ms, _ = solve.time_stages(nst, cfl=C3.cfl)
    alg_bytes = sum(STAGE_BYTES) / 3.0 * ndof  # per launch (average over the 3 stages)
    mean_stage_ms = float(np.mean(stage_ms))
    achieved_gbs = alg_bytes / (mean_stage_ms * 1e-3) / 1e9
    peak, peak_kind = measured_peaks()

    # ---- end-to-end through the public C ABI with pinned host buffers
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    barrier()
    torch.cuda.synchronize()
    e0.record(stream)
    solve.upload_ptr(u_host.data_ptr(), 0.0)
    r2 = solve.advance(1e9, cfl=C3.cfl, max_steps=args.steps)
    solve.download_ptr(u_out.data_ptr())
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    e2e_value = replica_rate(world, args.steps, ndof, max_over_ranks(e0.elapsed_time(e1), world, "cuda"))
    if not np.all(np.isfinite(u_out.numpy())) or r2["status"] != "max_steps":
        raise RuntimeError("e2e run produced a non-finite state")

    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            threads = os.cpu_count() or 1
            rate, done, dt = oracle_rate(512, 3, threads, min_seconds=5.0)
            srate, sdone, sdt = oracle_rate(512, 1, 1, min_seconds=3.0)
            cpu = {"value": rate, "unit": UNIT, "cores": threads, "kind": "port",
                   "sample": f"{done} SSP-RK3 steps of the 512^2 workload in {dt:.1f} s; C oracle, "
                             f"OpenMP {threads} threads",
                   "serial": {"value": srate, "unit": UNIT, "cores": 1,
                              "sample": f"{sdone} SSP-RK3 steps of the 512^2 workload in {sdt:.1f} s; "
                                        "C oracle, one thread (the reference's serial path)"}}
        tr = traffic_per_launch()
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded four-quadrant Riemann IC)", "config": workload_config(args),
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": ndof * 8 / args.steps,
                    "d2h_bytes_per_step": ndof * 8 / args.steps,
                    "note": "public C ABI: frg_upload_state (pinned host) + frg_advance(K) + "
                            "frg_download_state inside the timed region"},
            "roofline": {"bound": "hbm", "achieved": achieved_gbs, "peak": peak, "unit": "GB/s",
                         "frac": achieved_gbs / peak, "traffic": tr,
                         "kernel": "frg::stage2d_kernel<4,HLLC,BR0>",
                         "algorithmic_bytes_per_launch": alg_bytes,
                         "stage_ms": [float(x) for x in stage_ms], "peak_kind": peak_kind,
                         "tile_variant": int(variant),
                         "variant_ms": [float(x) for x in variant_ms],
                         "limiter": issue_limiter()},
            "cpu_baseline": cpu,
            "clocks": clk.summary(),
            "gpu_launches": advance_launches(args.steps, ndof),
        }
        print(json.dumps(line))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_c1(args):
    """The 1D case: 256 elements, P=3, Rusanov, Persson BR0, two-state
    Riemann IC, 2000 SSP-RK3 steps at CFL 0.1 (3,072 DOF).  It is launch- and
    latency-bound, not bandwidth-bound, so it reports steps/s and DOF-stage/s
    without a roofline.  One GPU (rank 0); other ranks exit."""
    import torch

    if int(os.environ.get("RANK", "0")) != 0:
        return 0
    import frforge_b200 as F
    from frforge_b200.workloads import C1

    ctx = F.Context(0)
    stream = torch.cuda.ExternalStream(ctx.stream_handle(), device=torch.device("cuda", 0))
    st, method = C1.build(F)
    solve = F.GpuSolve(st, F.Euler1D(1.4), method, ctx=ctx)
    ndof = solve.ndof
    u_host = torch.empty(ndof, dtype=torch.float64, pin_memory=True)
    u_host.numpy()[:] = st.u.ravel(order="F")
    u_out = torch.empty(ndof, dtype=torch.float64, pin_memory=True)
    steps = C1.steps
    for _ in range(max(3, args.warmup)):  # untimed: graph capture, caches
        solve.upload(st.u, 0.0)
        solve.advance(1e9, cfl=C1.cfl, max_steps=steps)
    times, e2e_times = [], []
    repeats = max(1, args.batch_reps)  # --batch-reps: timed repeats of the 2000 steps (median reported)
    with ClockSampler(0) as clk:
        for _ in range(repeats):
            solve.upload(st.u, 0.0)
            ev0 = torch.cuda.Event(enable_timing=True)
            ev1 = torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            ev0.record(stream)
            r = solve.advance(1e9, cfl=C1.cfl, max_steps=steps)
            ev1.record(stream)
            torch.cuda.synchronize()
            if r["status"] != "max_steps" or r["n_steps"] != steps:
                raise RuntimeError(f"C1 run ended early: {r}")
            times.append(ev0.elapsed_time(ev1))
            # end to end through the C ABI: upload, the 2000 steps, download
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(stream)
            solve.upload_ptr(u_host.data_ptr(), 0.0)
            solve.advance(1e9, cfl=C1.cfl, max_steps=steps)
            solve.download_ptr(u_out.data_ptr())
            e1.record(stream)
            torch.cuda.synchronize()
            e2e_times.append(e0.elapsed_time(e1))
    ms = float(np.median(times))
    ms_e2e = float(np.median(e2e_times))
    line = {
        "metric": "C1 1D solve: SSP-RK3 steps/s and DOF-stage/s (launch-bound, no roofline)",
        "value": steps / (ms * 1e-3), "unit": "steps/s", "n_gpus": 1, "steps": steps,
        "warmup": max(3, args.warmup), "ms_per_step": ms / steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded two-state Riemann IC)",
        "config": {"workload": "1D Euler, 256 elements on [0,1], GL P=3, Rusanov, SSP-RK3, Persson AV (BR0, "
                               "c_av=0.1), transmissive, CFL 0.1, 2000 steps, seeded two-state Riemann IC",
                   "dof": ndof, "repeats": len(times)},
        "dof_stage_per_s": 3 * ndof * steps / (ms * 1e-3),
        "e2e": {"value": steps / (ms_e2e * 1e-3), "unit": "steps/s", "h2d_bytes_per_step": ndof * 8 / steps,
                "d2h_bytes_per_step": ndof * 8 / steps},
        "clocks": clk.summary(),
        "gpu_launches": advance_launches(steps, ndof, loop1d=True),
    }
    print(json.dumps(line))
    return 0


def tune_table(F, ctx, keys, n: int = 256):
    """Fill the tile table (frg_autotune_table_*) as a deployment does before
    serving: from the committed table measured on a B200
    (frforge_b200/autotune_b200.json, frforge_b200.autotune.measure) when
    present, else for every (P, flux) key, Persson BR0 on an affine mesh, by
    timing the tile variants on an n^2 periodic density wave.  New solves and
    the batched groups of a key then use its variant.  Returns
    {"p<P>_<flux>": variant}."""
    from frforge_b200 import autotune as T
    from frforge_b200.workloads import Workload2D

    if T.load_default():
        return {f"p{p}_{flux}": T.get_variant(p, flux, "br0", False) for p, flux in keys}
    out = {}
    for p, flux in keys:
        w = Workload2D("c2", n, p, flux, "persson_av", 0.1, True, 0.1, 4)
        st, m = w.build(F)
        s = F.GpuSolve(st, F.Euler2D(1.4), m, ctx=ctx)
        s.upload(st.u, 0.0)
        best, _ = s.autotune(reps=3)
        out[f"p{p}_{flux}"] = int(best)
        s.close()
    return out


def run_batched(args):
    """64 independent mixed solves (frforge_b200.workloads.c4_instances), each
    200 SSP-RK3 steps: solves/s of the batched engine (frg_batch_*) against
    the same solves run one after another through frg_advance.  Both arms
    include the pinned-host upload of every initial state and the download of
    every final state; solve creation (mesh set-up) is outside both.  The
    batched results are checked bit-identical to the sequential ones."""
    import torch

    import frforge_b200 as F
    from frforge_b200.batch import Batch
    from frforge_b200.workloads import c4_instances

    local = int(os.environ.get("LOCAL_RANK", "0"))
    rank = int(os.environ.get("RANK", "0"))
    torch.cuda.set_device(local)
    ctx = F.Context(local)
    stream = torch.cuda.ExternalStream(ctx.stream_handle(), device=torch.device("cuda", local))
    inst = c4_instances(steps=args.batch_steps)
    built = [w.build(F) for w in inst]
    ndofs = [int(st.u.size) for st, _ in built]
    offs = np.concatenate([[0], np.cumsum(ndofs)])
    u_in = torch.empty(int(offs[-1]), dtype=torch.float64, pin_memory=True)
    out_seq = torch.empty_like(u_in, pin_memory=True)
    out_bat = torch.empty_like(u_in, pin_memory=True)
    for k, (st, _) in enumerate(built):
        u_in.numpy()[offs[k]:offs[k + 1]] = st.u.ravel(order="F")
    eq = F.Euler2D(1.4)
    steps = args.batch_steps
    cfl = inst[0].cfl
    esz = u_in.element_size()
    # tile table for both arms (solves read it at creation, batched groups
    # at grouping), outside the timed region
    tiles = {} if args.no_tune else tune_table(F, ctx, sorted({(w.p, w.flux) for w in inst}))

    # sequential arm: one GpuSolve per instance, run one after the other
    solves = [F.GpuSolve(st, eq, m, ctx=ctx) for st, m in built]

    def seq_pass(out):
        res = []
        for k, s in enumerate(solves):
            s.upload_ptr(u_in.data_ptr() + esz * int(offs[k]), 0.0)
            res.append(s.advance(1e9, cfl=cfl, max_steps=steps))
            s.download_ptr(out.data_ptr() + esz * int(offs[k]))
        return res

    # batched arm
    b = Batch(capacity=len(inst), ctx=ctx)
    slots = [b.add(st, eq, m) for st, m in built]

    def bat_pass(out):
        for k, i in enumerate(slots):
            b.upload_ptr(i, u_in.data_ptr() + esz * int(offs[k]), 0.0)
            b.start(i, 1e9, cfl=cfl, max_steps=steps)
        res = b.run()
        for k, i in enumerate(slots):
            b.download_ptr(i, out.data_ptr() + esz * int(offs[k]))
        return [res[i] for i in slots]

    def timed(fn, out):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        res = fn(out)
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1), res

    for _ in range(max(1, args.warmup // 3)):  # graphs captured, caches warm
        seq_pass(out_seq)
        bat_pass(out_bat)
    reps = max(1, args.batch_reps)
    seq_ms, bat_ms = [], []
    with ClockSampler(local) as clk:
        for _ in range(reps):
            ms, res_seq = timed(seq_pass, out_seq)
            seq_ms.append(ms)
            ms, res_bat = timed(bat_pass, out_bat)
            bat_ms.append(ms)
    # the batched and the single-solve kernels fuse a few multiply-adds
    # differently: results agree to rounding, statuses and step counts exactly
    a, c = out_seq.numpy(), out_bat.numpy()
    worst = 0.0
    for k in range(len(inst)):
        x, y = a[offs[k]:offs[k + 1]], c[offs[k]:offs[k + 1]]
        worst = max(worst, float(np.max(np.abs(x - y)) / max(np.max(np.abs(x)), 1e-300)))
    same = worst <= 1e-9 and all(
        p["status"] == q["status"] and p["n_steps"] == q["n_steps"] for p, q in zip(res_seq, res_bat))
    if not same:
        raise RuntimeError(f"batched results differ from the sequential ones (rel L-inf {worst:.3e})")
    t_seq, t_bat = float(np.median(seq_ms)), float(np.median(bat_ms))
    dof_stages = sum(3 * d * r["n_steps"] for d, r in zip(ndofs, res_bat))
    ngroups = len({(w.p, w.flux) for w in inst})
    # the packing bound: every instance's DOF-stages at the single-solve
    # stage kernel's own rate for its (P, flux) on a mesh that fills the GPU
    rates = single_solve_rates(F, ctx, sorted({(w.p, w.flux) for w in inst}))
    t_ideal = 1e3 * sum(3 * d * r["n_steps"] / rates[(w.p, w.flux)] for d, r, w in zip(ndofs, res_bat, inst))
    if rank == 0:
        line = {
            "metric": "batched solves/s (64 mixed 2D solves x 200 SSP-RK3 steps) vs one at a time",
            "value": len(inst) / (t_bat * 1e-3), "unit": "solves/s", "n_gpus": 1, "steps": steps,
            "warmup": args.warmup, "ms_per_step": t_bat / steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded ICs)",
            "config": {"workload": "batched: 64 instances, n=round(exp(U[ln16,ln256])), P~U{1..5}, "
                                   "HLLC/Rusanov, Persson AV c_av=0.1*U[0.5,2], half periodic density "
                                   "waves, half transmissive four-quadrant ICs, 200 SSP-RK3 steps, CFL 0.1",
                       "elements": int(sum(w.n * w.n for w in inst)), "dof": int(offs[-1]),
                       "groups": ngroups, "reps": reps,
                       "tile_table": tiles or "empty (default tiles)"},
            "sequential": {"value": len(inst) / (t_seq * 1e-3), "unit": "solves/s", "ms": t_seq},
            "speedup_vs_sequential": t_seq / t_bat,
            "ideal_speedup": t_seq / t_ideal,
            "ideal_ms": t_ideal,
            "packing_efficiency": t_ideal / t_bat,
            "single_solve_rates": {f"p{p}_{fl}": r for (p, fl), r in rates.items()},
            "ideal_note": "ideal_ms = sum over instances of DOF-stages / the single-solve stage kernel's rate for "
                          "that (P, flux) on a 512^2 (P<=3) or 384^2 (P>=4) periodic mesh, measured in this run: "
                          "the time of a perfectly packed batch; ideal_speedup = sequential ms / ideal_ms",
            "dof_stage_per_s": dof_stages / (t_bat * 1e-3),
            "statuses": sorted({r["status"] for r in res_bat}),
            "max_rel_linf_vs_sequential": worst,
            "e2e": {"value": len(inst) / (t_bat * 1e-3), "unit": "solves/s",
                    "h2d_bytes_per_step": int(offs[-1]) * 8 / steps,
                    "d2h_bytes_per_step": int(offs[-1]) * 8 / steps},
            "clocks": clk.summary(),
            "gpu_launches": steps * (2 + 3 * ngroups) + len(inst) + -(-steps // 4),
        }
        print(json.dumps(line))
    b.close()
    for s in solves:
        s.close()
    return 0


def single_solve_rates(F, ctx, keys, steps: int = 6):
    """DOF-stage/s of the single-solve stage kernels per (P, flux), Persson
    BR0, on a mesh that fills the GPU (512^2 for P <= 3, 384^2 above): the
    mean stage-kernel time of `steps` SSP-RK3 steps of a periodic density
    wave, CUDA events around every stage launch (frg_time_stages)."""
    from frforge_b200.workloads import Workload2D

    out = {}
    for p, flux in keys:
        n = 512 if p <= 3 else 384
        w = Workload2D("c2", n, p, flux, "persson_av", 0.1, True, 0.1, steps)
        st, m = w.build(F)
        s = F.GpuSolve(st, F.Euler2D(1.4), m, ctx=ctx)
        s.upload(st.u, 0.0)
        s.autotune(reps=3)
        stage_ms, _ = s.time_stages(steps, cfl=w.cfl)
        out[(p, flux)] = s.ndof / (float(np.mean(stage_ms)) * 1e-3)
        s.close()
    return out


def run_served(args):
    """A seeded Poisson request trace (frforge_b200.workloads.served_trace:
    1D and 2D solves, P 1..5, wavy 2D meshes, t_final U[0.05, 0.25]) served by
    frg_server_* against the same requests served one at a time (FIFO,
    frg_solve_create + device IC + frg_advance + download per request).
    Latency is arrival -> final state on the host, on the host clock; both
    arms include the device set-up of every solve and evaluate its initial
    condition on the device."""
    import torch

    import frforge_b200 as F
    from frforge_b200.serve import Server
    from frforge_b200.workloads import served_trace

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    ctx = F.Context(local)
    trace = served_trace(count=args.served_requests)
    # tile table for both arms (2D affine keys), outside the timed region
    tiles = {} if args.no_tune else tune_table(
        F, ctx, sorted({(r.p, r.flux) for r in trace if r.dim == 2 and not r.wavy}))
    # mesh and scheme only: both arms evaluate each request's IC on the device
    built = [req.build(F, fill=False) for req in trace]
    ics = [req.ic() for req in trace]
    arrivals = np.array([r.arrival for r in trace])

    def served_arm():
        srv = Server(slots=64, hbm_budget=64 << 30, steps_per_pump=8, ctx=ctx)
        done_at, ids, res = {}, [], {}
        nxt, t0 = 0, time.perf_counter()
        while len(done_at) < len(trace):
            now = time.perf_counter() - t0
            while nxt < len(trace) and arrivals[nxt] <= now:
                st, eq, m = built[nxt]
                ids.append(srv.submit_ic(st, eq, ics[nxt], m, t_final=trace[nxt].t_final, cfl=trace[nxt].cfl))
                nxt += 1
            _, q, a = srv.pump()
            now = time.perf_counter() - t0
            for rid in srv.take_completed():
                done_at[rid] = now
                res[rid] = srv.result(rid)
            if q == 0 and a == 0 and nxt < len(trace):
                time.sleep(max(0.0, arrivals[nxt] - (time.perf_counter() - t0)))
        srv.close()
        lat = np.array([done_at[rid] - arrivals[k] for k, rid in enumerate(ids)])
        return lat, max(done_at.values()), [res[rid] for rid in ids]

    def sequential_arm():
        lat, res = [], []
        t0 = time.perf_counter()
        for k, req in enumerate(trace):
            now = time.perf_counter() - t0
            if arrivals[k] > now:
                time.sleep(arrivals[k] - now)
            st, eq, m = built[k]
            s = F.GpuSolve(st, eq, m, ctx=ctx)
            s.set_initial_condition(**ics[k])
            r = s.advance(req.t_final, cfl=req.cfl)
            u, _ = s.download()
            s.close()
            r["u"] = u
            res.append(r)
            lat.append(time.perf_counter() - t0 - arrivals[k])
        return np.array(lat), time.perf_counter() - t0, res

    with ClockSampler(local) as clk:
        lat_s, span_s, res_s = served_arm()
        lat_q, span_q, res_q = sequential_arm()
    # The served path runs the batched kernels, the sequential one the
    # single-solve kernels: they fuse a few multiply-adds differently, and over
    # thousands of shocked steps that rounding grows.  Status and step count
    # must agree; the states are compared in relative L1 (and L-inf reported).
    worst, worst_l1 = 0.0, 0.0
    for k, (a, c) in enumerate(zip(res_s, res_q)):
        if a["status"] == c["status"] == "diverged":
            continue  # blow-up: the step it is detected at is rounding-sensitive
        if a["status"] != c["status"] or a["n_steps"] != c["n_steps"]:
            raise RuntimeError(f"served request {k} ({trace[k]}) ended {a['status']} after {a['n_steps']} "
                               f"steps, alone {c['status']} after {c['n_steps']}")
        d = np.abs(a["u"] - c["u"])
        worst = max(worst, float(d.max() / max(np.max(np.abs(c["u"])), 1e-300)))
        worst_l1 = max(worst_l1, float(d.sum() / max(np.sum(np.abs(c["u"])), 1e-300)))
    if worst_l1 > 1e-6:
        raise RuntimeError(f"served results differ from the sequential ones (rel L1 {worst_l1:.3e})")
    steps = sum(r["n_steps"] for r in res_s)
    dof_stages = sum(3 * req.ndof * r["n_steps"] for req, r in zip(trace, res_s))
    line = {
        "metric": f"served solves/s and latency ({len(trace)}-request Poisson trace at 200 req/s) vs one at a time",
        "value": len(trace) / span_s, "unit": "solves/s", "n_gpus": 1, "steps": int(steps),
        "warmup": 0, "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded request trace)",
        "config": {"workload": "served: Poisson arrivals 200/s; 1D Ne~U{128..4096} or 2D n~U{16..384} "
                               "(1/4 wavy, amplitude 0.05), P~U{1..5}, HLLC/Rusanov, density wave or "
                               "Riemann IC (jumps x0.25), periodic, t_final~U[0.05,0.25], Persson AV, "
                               "SSP-RK3, CFL 0.1",
                   "requests": len(trace), "slots": 64, "steps_per_pump": 8,
                   "tile_table": tiles or "empty (default tiles)"},
        "latency_s": {"p50": float(np.percentile(lat_s, 50)), "p99": float(np.percentile(lat_s, 99)),
                      "max": float(lat_s.max())},
        "sequential": {"value": len(trace) / span_q, "unit": "solves/s",
                       "latency_s": {"p50": float(np.percentile(lat_q, 50)),
                                     "p99": float(np.percentile(lat_q, 99)), "max": float(lat_q.max())}},
        "speedup_vs_sequential": span_q / span_s,
        "dof_stage_per_s": dof_stages / span_s,
        "max_rel_linf_vs_sequential": worst,
        "max_rel_l1_vs_sequential": worst_l1,
        "statuses": {st: sum(1 for r in res_s if r["status"] == st) for st in sorted({r["status"] for r in res_s})},
        "e2e": {"value": len(trace) / span_s, "unit": "solves/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 8 * sum(req.ndof for req in trace) / max(steps, 1),
                "note": "initial states evaluated on the device (frg_server_submit_ic); final states downloaded"},
        "clocks": clk.summary(),
    }
    print(json.dumps(line))
    return 0


def run_ncu_target(args):
    """A short, fixed launch sequence for ncu captures: the 512^2 workload
    (or --n elements per side, same P and IC; --flux / --method replace the
    workload's flux and capturing method), default tile variant, one prime
    launch (with Persson AV) then --steps SSP-RK3 steps with direct launches
    (begin, stage 1, 2, 3, end per step)."""
    import frforge_b200 as F
    from frforge_b200.workloads import C3, Workload2D

    w = Workload2D(C3.name, args.n, C3.p, args.flux or C3.flux, args.method or C3.method, C3.c_av, C3.periodic,
                   C3.cfl, C3.steps, seed=C3.seed, jump_scale=C3.jump_scale)
    st, method = w.build(F)
    solve = F.GpuSolve(st, F.Euler2D(1.4), method)
    if args.variant is not None:
        solve.set_variant(args.variant)
    solve.upload(st.u, 0.0)
    ms, r = solve.time_stages(args.steps, cfl=C3.cfl)
    print(json.dumps({"ncu_target": True, "n": args.n, "steps": args.steps, "variant": solve.variant()[0],
                      "stage_ms": [float(x) for x in ms], "status": r["status"]}))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="c3", choices=["c3", "c1", "batched", "served"])
    ap.add_argument("--served-requests", type=int, default=32)
    ap.add_argument("--ncu-target", action="store_true")
    ap.add_argument("--n", type=int, default=512)
    ap.add_argument("--variant", type=int, default=None,
                    help="--ncu-target: tile variant of the stage kernel (default: variant 0)")
    ap.add_argument("--flux", choices=["hllc", "rusanov"], default=None,
                    help="--ncu-target: numerical flux (default: the workload's, HLLC)")
    ap.add_argument("--method", choices=["persson_av", "null"], default=None,
                    help="--ncu-target: capturing method (default: the workload's, Persson AV)")
    ap.add_argument("--batch-steps", type=int, default=200)
    ap.add_argument("--batch-reps", type=int, default=3)
    ap.add_argument("--no-tune", action="store_true",
                    help="--workload batched/served: leave the autotune table empty (default tiles)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    if args.ncu_target:
        return run_ncu_target(args)
    if args.workload == "batched":
        return run_batched(args)
    if args.workload == "c1":
        return run_c1(args)
    if args.workload == "served":
        return run_served(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
