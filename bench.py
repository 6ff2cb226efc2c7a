#!/usr/bin/env python
"""Benchmark of the PD hot path: inverse-stiffness beam, forward + adjoint.

Workload (one bench step = one gradient evaluation of the inverse-stiffness
problem): 40x8x8 cubes of 0.05 m, 5 tets each (3,321 vertices, 12,800 tets),
per-tet E log-uniform in [1e4, 1e6] Pa (seed 1234), both ends pinned, gravity,
h = 1/100 s, 20 local-global iterations, 60 time steps.  A step refactors H
for the current moduli, runs the 60 steps forward, and the adjoint of all 60
steps back to dL/dE for L = |x_60 - x_60^target|^2 (target from the seed-5678
modulus field).  The metric is simulated time steps per second of
forward + adjoint (60 per bench step), summed over GPUs.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--precision fp64|mixed]
    python bench.py --impl reference ...   # CPU reference arm (FP64 oracle port)
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

SIM_STEPS = 60
METRIC = "fwd+adjoint sim steps/s (inverse stiffness 12,800 tets, K=20)"

# DRAM bytes per launch of the global solve on the inverse-stiffness workload,
# by solve form, from one ncu capture each (dram__bytes_read.sum +
# dram__bytes_write.sum; the persistent form's factor is largely L2-resident
# between solves, so its figure is below the algorithmic bytes; the dense
# form reads Hs^-1 from DRAM once per solve).  Not measured by a bench run.
SOLVE_DRAM_BYTES = {"persistent": 4.36e6, "dense": 88.51e6 + 2.93e6}
UNIT = "steps/s"


def pin_triangular(sc) -> bool:
    """Put a scene on the fastest of its supernodal triangular-solve forms (the
    plain form) when the autotune chose the dense inverse; True if it did."""
    info = sc.solve_mode()
    if info["mode"] != "dense":
        return False
    tri = {"levels": info["ms_levels"], "persistent": info["ms_persistent"], "split": info["ms_split"],
           "cluster": info["ms_cluster"], "resident": info["ms_resident"]}
    sc.solve_mode(min((v, k) for k, v in tri.items() if v > 0)[1])
    return True


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    p.add_argument("--sim-steps", type=int, default=None,
                   help="time steps per gradient evaluation (60 / 100 are the workloads; fewer only for profiler captures)")
    p.add_argument("--workload", default="inverse_stiffness", choices=["inverse_stiffness", "batch", "star", "cloth_ball"],
                   help="inverse_stiffness: one 12,800-tet scene; batch: 256 uneven scenes in one handle; "
                        "star: the muscle star on the ground, gradient w.r.t. all activations; "
                        "cloth_ball: a 64x64 cloth dropped on a ball, gradient w.r.t. the initial velocities")
    p.add_argument("--scenes", type=int, default=256, help="batch workload: number of scenes")
    p.add_argument("--no-comparison", action="store_true",
                   help="skip the mixed/FP64 and batched/one-at-a-time comparison of the default line")
    p.add_argument("--fp64-sample", type=int, default=-1,
                   help="batch workload: scenes stepped one at a time in FP64 for the plain-form rate "
                        "(-1: every scene of the batch, 0: skip)")
    a = p.parse_args()
    global SIM_STEPS
    SIM_STEPS = a.sim_steps if a.sim_steps is not None else {"batch": 100, "star": 200, "cloth_ball": 300}.get(a.workload, 60)
    return a


def workload_config(precision: str) -> dict:
    return {
        "workload": "inverse_stiffness beam 40x8x8 cubes x5 tets (12,800 tets, 3,321 vertices), "
                    "E~logU[1e4,1e6] seed 1234, both ends pinned, h=1/100, K=20, 60 steps, fwd+adjoint dL/dE",
        "tets": 12800, "vertices": 3321, "sim_steps_per_bench_step": SIM_STEPS, "pd_iterations": 20,
        **({} if SIM_STEPS == 60 else {"note": "reduced time steps: profiler capture only, not a bench value"}),
        "precision": precision, "parallelism": "replicas (one independent scene per GPU)",
    }


# ----------------------------------------------------------------- clocks ---

class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self.first = 0
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "50"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            # the timed region starts once sampling is live; samples before that are dropped
            t_end = time.time() + 3.0
            while not self.rows and time.time() < t_end:
                time.sleep(0.01)
            self.first = len(self.rows)
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self) -> dict:
        rows = self.rows[self.first:] if len(self.rows) > self.first else self.rows
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(r[1]) for r in rows if len(r) > 2 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if len(r) > 2 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in rows:
            for k, n in enumerate(names):
                if len(r) > 5 + k and r[5 + k].lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(rows)}


# ------------------------------------------------------------ CPU oracle ---

def oracle_sample(threads: int, sim_steps: int = 2) -> dict:
    """Time the FP64 oracle port on a bounded sample of the same workload:
    `sim_steps` steps forward + adjoint of the inverse-stiffness beam."""
    from diff_fem_b200 import scene as S
    from oracle import oracle as O
    d = S.inverse_stiffness()
    o = O.OracleScene(d)
    x = d.x0.reshape(-1).copy()
    v = np.zeros_like(x)
    t0 = time.perf_counter()
    o.set_materials(d.youngs, d.poisson)
    r = o.forward(x, v, n_steps=sim_steps, threads=threads)
    o.backward(2 * (r["x"] - x), np.zeros_like(x))
    dt = time.perf_counter() - t0
    return {"value": sim_steps / dt, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{sim_steps} of the 60 time steps, forward + adjoint incl. refactorisation, "
                      f"FP64 C++ oracle ({threads} host thread{'s' if threads > 1 else ''})",
            "seconds": dt}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    oracle_sample(threads, 1)  # warm-up (also builds the library if needed)
    vals = []
    for _ in range(max(1, args.warmup)):
        oracle_sample(threads, 1)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        vals.append(oracle_sample(threads, 2)["seconds"])
    total = sum(vals)
    value = 2 * args.steps / total
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config("fp64"),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": "each bench step = 2 of the 60 time steps forward + adjoint incl. "
                                       "refactorisation, FP64 C++ oracle, local step on all host threads"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# -------------------------------------------------------------------- GPU ---

def run_ours(args):
    import torch
    import torch.distributed as dist
    from diff_fem_b200 import scene as S
    from diff_fem_b200._capi import DFEM_PREC_FP64, DFEM_PREC_MIXED
    from diff_fem_b200.engine import Scene

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    prec = DFEM_PREC_FP64 if args.precision == "fp64" else DFEM_PREC_MIXED
    d = S.inverse_stiffness(precision=prec)
    sc = Scene(d, device=local)
    info = sc.info()
    N, T = d.n_vertices, d.n_tets
    E0 = torch.tensor(d.youngs, device=dev)
    nu = torch.tensor(d.poisson, device=dev)
    Et = torch.tensor(S.log_uniform_moduli(T, 5678), device=dev)
    x0 = torch.tensor(d.x0.reshape(-1), device=dev)
    v0 = torch.zeros_like(x0)
    sc.set_materials(Et, nu)
    target, _ = sc.forward(x0, v0, n_steps=SIM_STEPS)
    target = target.clone()
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)  # 256 MB > L2 (126 MB)

    def grad_eval(E):
        sc.set_materials(E, nu)
        x, v = sc.forward(x0, v0, n_steps=SIM_STEPS)
        gx = 2.0 * (x - target)
        g = sc.backward(gx, torch.zeros_like(gx))
        return g["E"]

    stream = torch.cuda.current_stream(dev)
    for _ in range(max(3, args.warmup)):
        grad_eval(E0)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    launches0 = sc.launch_count()
    elapsed = 0.0
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            grad_eval(E0)
            e1.record(stream)
            torch.cuda.synchronize()
            elapsed += e0.elapsed_time(e1) / 1e3
    launches = sc.launch_count() - launches0
    if world > 1:
        dist.barrier()
        t = torch.tensor([elapsed], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        elapsed = float(t.item())
    value = world * SIM_STEPS * args.steps / elapsed

    # forward-only rate (same scene, device-resident)
    torch.cuda.synchronize()
    ef0, ef1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ef0.record(stream)
    for _ in range(args.steps):
        sc.forward(x0, v0, n_steps=SIM_STEPS)
    ef1.record(stream)
    torch.cuda.synchronize()
    fwd_rate = SIM_STEPS * args.steps / (ef0.elapsed_time(ef1) / 1e3)
    iters = sc.iterations(SIM_STEPS)

    # end to end through the public API with host buffers (pinned), copies inside the timed region
    E_h = torch.tensor(d.youngs).pin_memory()
    nu_h = torch.tensor(d.poisson).pin_memory()
    x0_h = torch.tensor(d.x0.reshape(-1)).pin_memory()
    v0_h = torch.zeros(3 * N, dtype=torch.float64).pin_memory()
    tgt_h = target.cpu()
    t_e2e = 0.0
    for _ in range(args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        sc.set_materials(E_h, nu_h)
        xh, vh = sc.forward(x0_h, v0_h, n_steps=SIM_STEPS)
        gxh = 2.0 * (torch.from_numpy(xh) - tgt_h)
        gh = sc.backward(gxh.numpy(), np.zeros(3 * N))
        _ = float(np.sum(gh["E"]))
        t_e2e += time.perf_counter() - t0
    e2e = {"value": world * SIM_STEPS * args.steps / t_e2e if world == 1 else None, "unit": UNIT,
           "h2d_bytes_per_step": 8 * (2 * T + 3 * N * 4), "d2h_bytes_per_step": 8 * (3 * N * 4 + 2 * T)}
    if world > 1:
        t = torch.tensor([t_e2e], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e["value"] = world * SIM_STEPS * args.steps / float(t.item())

    # material update alone: moduli upload, Hs values and the numeric refactorisation
    torch.cuda.synchronize()
    tr0 = time.perf_counter()
    for _ in range(5):
        sc.set_materials(Et, nu)
    torch.cuda.synchronize()
    refactor_ms = (time.perf_counter() - tr0) / 5 * 1e3

    # roofline of the dominant kernel phase (CUDA events on the engine's stream)
    sc.forward(x0, v0, n_steps=1)
    ph = sc.profile_phases(reps=50)
    n_it = int(iters.sum())
    # the adjoint replays no step when every step's iterates fit the default adjoint budget (45 % of
    # the device memory): then one forward and one adjoint solve per PD iteration, else also a replay
    stored = 3 * N * 8 * (d.max_iterations + 1) * SIM_STEPS <= torch.cuda.get_device_properties(dev).total_memory * 45 // 100
    runs = 1 if stored else 2
    share = {"local": runs * n_it * ph["local"], "solve": (runs + 1) * n_it * ph["solve"],
             "adj_local": n_it * ph["adj_local"], "gather": (runs + 1) * n_it * ph["gather"]}
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    peak_note = "measured (MEASURED_PEAKS.json hbm_gbs, burst copy)" if "hbm_gbs" in peaks else "fallback 6650 GB/s"
    nnz = int(info["nnz_factor"])
    solve_info = sc.solve_mode()
    if solve_info["mode"] == "dense":
        # the dense-inverse form reads the N rows x N_p columns of Hs^-1 (FP64) once; rhs in, y out
        n_p = -(-N // 64) * 64
        solve_bytes = N * n_p * 8 + 48 * N
        solve_note = "per solve (the N x N_p FP64 rows of Hs^-1 once, rhs in, y out; k_dense_solve)"
    else:
        solve_bytes = 2 * nnz * 8 + 96 * N                   # 2 sweeps x the factor's FP64 values + in/out vectors
        solve_note = "per solve (both sweeps)"
    local_bytes = T * (16 + 72 + 16) + N * 72                 # tet tables + x, b, rhs per vertex
    dom = max(share, key=share.get)
    if dom == "solve":
        achieved = solve_bytes / (ph["solve"] * 1e-3) / 1e9
        traffic_note = solve_note
    else:
        achieved = local_bytes / (ph[dom] * 1e-3) / 1e9
        traffic_note = f"per {dom} launch"
    traffic = SOLVE_DRAM_BYTES.get(solve_info["mode"]) if (dom == "solve" and SIM_STEPS == 60) else None
    roofline = {"bound": "hbm", "kernel": dom, "solve_form": solve_info["mode"], "achieved": achieved, "peak": hbm,
                "unit": "GB/s", "frac": achieved / hbm, "traffic": traffic,
                "traffic_source": "dram__bytes_read.sum + dram__bytes_write.sum per launch from one earlier ncu "
                                  "capture of this solve form on this workload (not measured by this run)"
                if traffic else None, "peak_source": peak_note,
                "algorithmic_bytes": solve_bytes if dom == "solve" else local_bytes, "per": traffic_note,
                "phase_ms": ph, "phase_share_ms_per_bench_step": share}

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * elapsed / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "f32+f64",
            "data": "synthetic",
            "config": dict(workload_config(args.precision), l2="flushed between timed steps (256 MB write)",
                           factor={"supernodes": info["n_supernodes"], "levels": info["n_levels"], "nnz": nnz},
                           solve=sc.solve_mode()),
            "forward_only_steps_per_s": world * fwd_rate, "pd_iterations_total": n_it,
            "set_materials_ms": refactor_ms,
            "e2e": e2e, "roofline": roofline, "gpu_launches": launches, "clocks": clk.summary()}
    if rank == 0 and world == 1:
        try:
            line["cpu_baseline"] = oracle_sample(1, 2)
        except Exception as ex:  # the baseline must not kill the GPU line
            line["cpu_baseline"] = {"value": None, "error": str(ex)}
    sc.close()
    if rank == 0 and world == 1 and not args.no_comparison:
        try:
            line["comparison"] = comparison_extras(args, local)
        except Exception as ex:  # the comparison must not kill the GPU line
            line["comparison"] = {"error": f"{type(ex).__name__}: {ex}"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


# ------------------------------------------------------------ comparison ---

def _rel(a, b) -> float:
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def comparison_extras(args, local: int) -> dict:
    """The comparison the metric names: mixed FP32/FP64 against plain FP64,
    batched against one scene at a time, each with its error.
    (1) The 12,800-tet inverse-stiffness problem in both precisions, each
        against the FP64 oracle on the host (same moduli and target, 60 steps
        forward + adjoint): positions x_60 and dL/dE.
    (2) The 256-scene uneven batch (100 steps forward + adjoint): batched mixed,
        batched FP64, and plain FP64 one scene per handle on a stratified
        sample of 16 scenes; errors of the mixed batch against the FP64 batch.
    Timed with CUDA events on the engine's stream, L2 flushed between timed
    evaluations; a few evaluations each (the headline value above is the
    long-run number)."""
    import torch
    from diff_fem_b200 import scene as S
    from diff_fem_b200._capi import DFEM_PREC_FP64, DFEM_PREC_MIXED
    from diff_fem_b200.engine import Scene
    from oracle import oracle as O

    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream(dev)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)

    def timed(fn, reps, warm=1):
        out = None
        for _ in range(warm):
            out = fn()
        tot = 0.0
        for _ in range(reps):
            flush.zero_()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            out = fn()
            e1.record(stream)
            torch.cuda.synchronize()
            tot += e0.elapsed_time(e1) / 1e3
        return tot / max(1, reps), out

    res = {}
    # (1) inverse stiffness, FP64 and mixed against the oracle
    n = 60
    d64 = S.inverse_stiffness()
    T = d64.n_tets
    Et = S.log_uniform_moduli(T, 5678)
    x0 = d64.x0.reshape(-1).copy()
    v0 = np.zeros_like(x0)
    threads = os.cpu_count() or 1
    o = O.OracleScene(d64)
    o.set_materials(Et, d64.poisson)
    tgt = o.forward(x0, v0, n_steps=n, threads=threads)["x"]
    o.set_materials(d64.youngs, d64.poisson)
    ro = o.forward(x0, v0, n_steps=n, threads=threads)
    bo = o.backward(2.0 * (ro["x"] - tgt), np.zeros_like(x0))
    c2 = {}
    for name, prec in (("fp64", DFEM_PREC_FP64), ("mixed", DFEM_PREC_MIXED)):
        d = S.inverse_stiffness(precision=prec)
        sc = Scene(d, device=local)
        E0 = torch.tensor(d.youngs, device=dev)
        nu = torch.tensor(d.poisson, device=dev)
        xt, vt, tg = (torch.tensor(a, device=dev) for a in (x0, v0, tgt))

        def grad_eval():
            sc.set_materials(E0, nu)
            x, _ = sc.forward(xt, vt, n_steps=n)
            g = sc.backward(2.0 * (x - tg), torch.zeros_like(x))
            return x, g["E"]

        t, (x, gE) = timed(grad_eval, 10)
        c2[name] = {"value": n / t, "unit": "steps/s", "solve": sc.solve_mode()["mode"],
                    "pos_rel_err_vs_oracle": _rel(x.cpu().numpy(), ro["x"]),
                    "grad_E_rel_err_vs_oracle": _rel(gE.cpu().numpy(), bo["E"])}
        sc.close()
    c2["mixed_over_fp64"] = c2["mixed"]["value"] / c2["fp64"]["value"]
    c2["workload"] = "inverse stiffness 12,800 tets, 60 steps forward + adjoint dL/dE incl. refactorisation"
    c2["oracle"] = f"FP64 C++ oracle on the host ({threads} threads), same moduli and target"
    res["inverse_stiffness"] = c2

    # (2) the uneven batch: batched mixed, batched FP64, plain FP64 one at a time;
    #     as specified (stars on their grounds) and without the grounds
    def batch_block(ground):
        nb = 100
        dm, _ = S.uneven_batch(n_scenes=args.scenes, precision=DFEM_PREC_MIXED, ground=ground)
        dd, _ = S.uneven_batch(n_scenes=args.scenes, precision=DFEM_PREC_FP64, ground=ground)
        xb = torch.tensor(np.concatenate([d.x0.reshape(-1) for d in dm]), device=dev)
        vb = torch.zeros_like(xb)
        nseg = sum(d.n_segments for d in dm)
        act = torch.tensor(np.random.default_rng(42).uniform(0.0, 1.0, (nb, nseg)), device=dev)
        out = {}
        for name, descs, reps in (("mixed", dm, 2), ("fp64", dd, 1)):
            t0 = time.perf_counter()
            b = Scene.batch(descs, device=local)
            setup = time.perf_counter() - t0

            def batch_eval():
                x, _ = b.forward(xb, vb, n_steps=nb, act=act)
                return x, b.backward(2.0 * (x - xb), torch.zeros_like(x))

            t, (x, g) = timed(batch_eval, reps)
            out[name] = {"value": len(descs) * nb / t, "unit": "scene-steps/s", "setup_s": setup,
                         "x": x.cpu().numpy(), "E": g["E"].cpu().numpy(), "act": g["act"].cpu().numpy(),
                         "iters": b.iterations(nb), "offsets": b.offsets}
            b.close()
        # plain FP64, one scene per handle: a sample stratified by size
        order = np.argsort([d.n_tets for d in dd], kind="stable")
        sample = order[np.linspace(0, len(dd) - 1, min(16, len(dd))).astype(int)]
        vo, so = out["fp64"]["offsets"]["vertices"], out["fp64"]["offsets"]["segments"]
        # the plain form is the supernodal triangular solve (the fastest of its
        # forms per scene); the dense-inverse form small single scenes may
        # take instead is timed beside it
        tsum, tsum_auto, n_dense = 0.0, 0.0, 0
        for q in sample:
            sc = Scene(dd[q], device=local)
            xq = xb[3 * vo[q]:3 * vo[q + 1]].contiguous()
            aq = act[:, so[q]:so[q + 1]].contiguous() if so[q + 1] > so[q] else None

            def one():
                x, _ = sc.forward(xq, torch.zeros_like(xq), n_steps=nb, act=aq)
                return sc.backward(2.0 * (x - xq), torch.zeros_like(x))

            t, _ = timed(one, 1)
            tsum_auto += t
            if pin_triangular(sc):
                n_dense += 1
                t, _ = timed(one, 1)
            tsum += t
            sc.close()
        plain = len(sample) * nb / tsum
        plain_auto = len(sample) * nb / tsum_auto
        # errors of the mixed batch against the FP64 batch, per scene
        to = out["fp64"]["offsets"]["tets"]
        same = np.all(out["mixed"]["iters"] == out["fp64"]["iters"], axis=0)
        pe, ge = [], []
        for p in range(len(dd)):
            a0, a1 = 3 * vo[p], 3 * vo[p + 1]
            pe.append(_rel(out["mixed"]["x"][a0:a1], out["fp64"]["x"][a0:a1]))
            ge.append(_rel(out["mixed"]["E"][to[p]:to[p + 1]], out["fp64"]["E"][to[p]:to[p + 1]]))
        pe, ge = np.asarray(pe), np.asarray(ge)
        return {
            "workload": f"{len(dd)} uneven scenes (tets log-uniform in [1e3, 5e4], beams and muscle stars"
                        + (", the stars on their grounds" if ground else ", no grounds") + f"), {nb} steps forward + adjoint",
            "mixed_batched": {"value": out["mixed"]["value"], "unit": "scene-steps/s", "setup_s": out["mixed"]["setup_s"]},
            "fp64_batched": {"value": out["fp64"]["value"], "unit": "scene-steps/s", "setup_s": out["fp64"]["setup_s"]},
            "fp64_one_at_a_time": {"value": plain, "unit": "scene-steps/s", "scenes_sampled": int(len(sample)),
                                   "sample": "16 scenes evenly spaced in size order, one handle each",
                                   "solve": "supernodal triangular solve (fastest of its forms per scene)"},
            "fp64_one_at_a_time_any_form": {"value": plain_auto, "unit": "scene-steps/s",
                                            "scenes_with_dense_inverse": n_dense,
                                            "solve": "the autotuned form, the dense inverse included"},
            "mixed_batched_over_fp64_one_at_a_time_any_form": out["mixed"]["value"] / plain_auto,
            "mixed_batched_over_fp64_one_at_a_time": out["mixed"]["value"] / plain,
            "fp64_batched_over_fp64_one_at_a_time": out["fp64"]["value"] / plain,
            "mixed_over_fp64_batched": out["mixed"]["value"] / out["fp64"]["value"],
            "error_mixed_vs_fp64": {
                "scenes_with_equal_iteration_counts": int(same.sum()), "scenes": int(len(dd)),
                "pos_rel_max": float(pe[same].max()) if same.any() else None,
                "pos_rel_median": float(np.median(pe[same])) if same.any() else None,
                "grad_E_rel_max": float(ge[same].max()) if same.any() else None,
                "grad_E_rel_median": float(np.median(ge[same])) if same.any() else None,
                "grad_act_rel_max": _rel(out["mixed"]["act"], out["fp64"]["act"]),
                "other_scenes_pos_rel_max": float(pe[~same].max()) if (~same).any() else None},
            "target": ">= 10x batched mixed over plain FP64, at <= 1e-6 position and <= 1e-4 gradient error",
        }

    res["batch"] = batch_block(True)
    res["batch_without_ground"] = batch_block(False)
    res["batch_without_ground"]["note"] = ("the same scenes without obstacle contact: over 100 steps the contact "
                                           "phase's stick/slide and impact decisions amplify the mixed form's "
                                           "rounding, so the error target is met only without them")
    return res


# ------------------------------------------------------------ batch (C5) ---

BATCH_METRIC = "batched fwd+adjoint scene-steps/s (256 uneven scenes, 1k-50k tets, 100 steps)"


def batch_config(args, descs) -> dict:
    T = [d.n_tets for d in descs]
    return {
        "workload": f"{len(descs)} independent scenes, tets log-uniform in [1e3, 5e4] (seed 7): beams "
                    "(x=0 pinned, per-tet E~logU[1e4,1e6]) alternating with 8-arm muscle stars, each on its own "
                    "ground quad (mu=0.5, obstacle contact inside the batch), "
                    "h=1/60, K=15, random activations per segment per step (seed 42), "
                    f"{SIM_STEPS} steps forward + adjoint of L=|x_end - x_0|^2",
        "scenes": len(descs), "tets_total": int(sum(T)), "vertices_total": int(sum(d.n_vertices for d in descs)),
        "tets_min": int(min(T)), "tets_max": int(max(T)), "sim_steps_per_bench_step": SIM_STEPS,
        **({} if SIM_STEPS == 100 else {"note": "reduced time steps: profiler capture only, not a bench value"}),
        "precision": args.precision,
        "parallelism": "scenes split across the GPUs by longest-processing-time placement; one batch handle "
                       "per GPU holding its share (no collective inside a step)",
    }


def run_batch(args):
    import torch
    from diff_fem_b200 import scene as S
    from diff_fem_b200._capi import DFEM_PREC_FP64, DFEM_PREC_MIXED
    from diff_fem_b200.engine import Scene

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    from diff_fem_b200 import shard
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    prec = DFEM_PREC_FP64 if args.precision == "fp64" else DFEM_PREC_MIXED
    t0 = time.perf_counter()
    all_descs, _ = S.uneven_batch(n_scenes=args.scenes, precision=prec)
    # the scenes split across the ranks by longest-processing-time placement on
    # their tet counts (shard.assign_scenes: every rank computes the same split);
    # each rank builds one batch handle of its own share, no data-path collective
    costs = [d.n_tets for d in all_descs]
    placement = shard.assign_scenes(costs, world)
    mine = placement[rank]
    descs = [all_descs[i] for i in mine]
    b = Scene.batch(descs, device=local)
    t_setup = time.perf_counter() - t0
    n = SIM_STEPS
    x0 = torch.tensor(np.concatenate([d.x0.reshape(-1) for d in descs]), device=dev)
    v0 = torch.zeros_like(x0)
    # activations of every scene of the job (seed 42), then this rank's columns
    rng = np.random.default_rng(42)
    seg0 = np.concatenate([[0], np.cumsum([d.n_segments for d in all_descs])]).astype(int)
    act_all = rng.uniform(0.0, 1.0, (n, int(seg0[-1])))
    act_np = np.concatenate([act_all[:, seg0[i]:seg0[i + 1]] for i in mine], axis=1) if mine else act_all[:, :0]
    act = torch.tensor(np.ascontiguousarray(act_np), device=dev)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)

    def grad_eval():
        x, v = b.forward(x0, v0, n_steps=n, act=act)
        return x, b.backward(2.0 * (x - x0), torch.zeros_like(x))

    for _ in range(max(3, args.warmup)):
        grad_eval()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    launches0 = b.launch_count()
    elapsed = 0.0
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            xm, gm = grad_eval()
            e1.record(stream)
            torch.cuda.synchronize()
            elapsed += e0.elapsed_time(e1) / 1e3
    launches = b.launch_count() - launches0
    if world > 1:
        t = torch.tensor([elapsed], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        elapsed = float(t.item())
    value = len(all_descs) * n * args.steps / elapsed  # every rank's scenes over the slowest rank's time
    iters = b.iterations(n)
    loads = [float(sum(costs[i] for i in p)) for p in placement]

    # forward-only rate
    torch.cuda.synchronize()
    ef0, ef1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ef0.record(stream)
    b.forward(x0, v0, n_steps=n, act=act)
    ef1.record(stream)
    torch.cuda.synchronize()
    fwd_rate = len(descs) * n / (ef0.elapsed_time(ef1) / 1e3)  # this rank's

    # end to end with host buffers (pinned), copies inside the timed region
    x0_h = x0.cpu().pin_memory()
    v0_h = v0.cpu().pin_memory()
    act_h = act.cpu().pin_memory()
    t_e2e = 0.0
    for _ in range(args.steps):
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        xh, vh = b.forward(x0_h, v0_h, n_steps=n, act=act_h)
        gh = b.backward(2.0 * (xh - x0_h.numpy()), np.zeros_like(xh))
        _ = float(np.sum(gh["E"])) + float(np.sum(gh["act"]))
        t_e2e += time.perf_counter() - t1
    N3, T, nseg = 3 * b.N, b.T, b.nseg
    if world > 1:
        t = torch.tensor([t_e2e], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        t_e2e = float(t.item())
    e2e = {"value": len(all_descs) * n * args.steps / t_e2e, "unit": "scene-steps/s",
           "h2d_bytes_per_step": 8 * (2 * N3 + n * nseg + 2 * N3),
           "d2h_bytes_per_step": 8 * (2 * N3 + 2 * N3 + 2 * T + n * nseg)}

    binfo = b.info()
    b.forward(x0, v0, n_steps=1, act=act[:1].contiguous())
    phases = b.profile_phases(reps=20)

    # per-scene error of this run against the FP64 batch (same scenes, same inputs)
    errs = None
    if prec == DFEM_PREC_MIXED:
        d64_all, _ = S.uneven_batch(n_scenes=args.scenes, precision=DFEM_PREC_FP64)
        b64 = Scene.batch([d64_all[i] for i in mine], device=local)
        x64, v64 = b64.forward(x0, v0, n_steps=n, act=act)
        g64 = b64.backward(2.0 * (x64 - x0), torch.zeros_like(x64))
        vo, to, so = b.offsets["vertices"], b.offsets["tets"], b.offsets["segments"]
        xm_c, x64_c = xm.cpu().numpy(), x64.cpu().numpy()
        gEm, gE64 = gm["E"].cpu().numpy(), g64["E"].cpu().numpy()
        gAm, gA64 = gm["act"].cpu().numpy(), g64["act"].cpu().numpy()
        same_iters = np.all(iters == b64.iterations(n), axis=0)
        pe, ge, ae = [], [], []
        for p in range(b.nparts):
            a0, a1 = 3 * vo[p], 3 * vo[p + 1]
            pe.append(np.abs(xm_c[a0:a1] - x64_c[a0:a1]).max() / np.abs(x64_c[a0:a1]).max())
            e0_, e1_ = gEm[to[p]:to[p + 1]], gE64[to[p]:to[p + 1]]
            ge.append(np.abs(e0_ - e1_).max() / max(np.abs(e1_).max(), 1e-300))
            if so[p + 1] > so[p]:
                q0, q1 = gAm[:, so[p]:so[p + 1]], gA64[:, so[p]:so[p + 1]]
                ae.append(np.abs(q0 - q1).max() / max(np.abs(q1).max(), 1e-300))
        pe, ge = np.asarray(pe), np.asarray(ge)
        keep = same_iters
        errs = {"scenes_with_equal_iteration_counts": int(keep.sum()), "scenes": int(b.nparts),
                "pos_rel_max": float(pe[keep].max()) if keep.any() else None,
                "pos_rel_median": float(np.median(pe[keep])) if keep.any() else None,
                "grad_E_rel_max": float(ge[keep].max()) if keep.any() else None,
                "grad_E_rel_median": float(np.median(ge[keep])) if keep.any() else None,
                "grad_act_rel_max": float(max(ae)) if ae else None,
                "scenes_with_a_different_iteration_count": {
                    "count": int((~keep).sum()),
                    "pos_rel_max": float(pe[~keep].max()) if (~keep).any() else None,
                    "grad_E_rel_max": float(ge[~keep].max()) if (~keep).any() else None,
                    "note": "the early exit flipped at one step: the FP64 and mixed runs stop at different "
                            "iterations, and the scenes differ by up to one PD update (bounded by the "
                            "convergence tolerance 3N * 5e-7 in the 2-norm)"},
                "reference": "the same batch in the plain FP64 form; positions and E-gradients over the scenes "
                             "whose per-step iteration counts equal the FP64 run's"}
        b64.close()

    # plain FP64 form, scenes one at a time (a sample spread over the size range)
    plain = None
    if args.fp64_sample != 0:
        d64_all, _ = S.uneven_batch(n_scenes=args.scenes, precision=DFEM_PREC_FP64)
        d64 = [d64_all[i] for i in mine]
        k = len(d64) if args.fp64_sample < 0 else min(args.fp64_sample, len(d64))
        idx = np.linspace(0, len(d64) - 1, k).astype(int)
        tsum, tets = 0.0, 0
        vo, so = b.offsets["vertices"], b.offsets["segments"]
        for q in idx:
            sc = Scene(d64[q], device=local)
            pin_triangular(sc)
            xq = x0[3 * vo[q]:3 * vo[q + 1]].contiguous()
            aq = act[:, so[q]:so[q + 1]].contiguous() if so[q + 1] > so[q] else None
            xs, _ = sc.forward(xq, torch.zeros_like(xq), n_steps=n, act=aq)  # warm-up (graph build)
            sc.backward(2.0 * (xs - xq), torch.zeros_like(xs))
            torch.cuda.synchronize()
            ea, eb = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            ea.record(stream)
            xs, _ = sc.forward(xq, torch.zeros_like(xq), n_steps=n, act=aq)
            sc.backward(2.0 * (xs - xq), torch.zeros_like(xs))
            eb.record(stream)
            torch.cuda.synchronize()
            tsum += ea.elapsed_time(eb) / 1e3
            tets += d64[q].n_tets
            sc.close()
        rate = len(idx) * n / tsum
        plain = {"value": rate, "unit": "scene-steps/s", "scenes": int(len(idx)), "mean_tets": tets / len(idx),
                 "batch_mean_tets": b.T / b.nparts, "ratio_batch_over_plain": value / world / rate,
                 "form": "plain FP64 engine (supernodal triangular solve), one scene per handle, forward + "
                         "adjoint, CUDA-event timed"}

    # roofline of the dominant phase (the global solve, both sweeps), CUDA events on the engine's stream
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    solve_bytes = 2 * int(binfo["nnz_factor"]) * 8 + 96 * b.N
    achieved = solve_bytes / (phases["solve"] * 1e-3) / 1e9
    roofline = {"bound": "hbm", "kernel": "global solve (" + b.solve_mode()["mode"] + " form)", "achieved": achieved,
                "peak": hbm, "unit": "GB/s", "frac": achieved / hbm, "traffic": None,
                "traffic_note": "not captured: the full batch is beyond the ncu capture size; "
                                "the 32-scene capture is in profiles/",
                "peak_source": "measured (MEASURED_PEAKS.json hbm_gbs, burst copy)" if "hbm_gbs" in peaks
                else "fallback 6650 GB/s",
                "algorithmic_bytes": solve_bytes, "per": "per solve (both sweeps)"}

    line = {"metric": BATCH_METRIC, "value": value, "unit": "scene-steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * elapsed / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if args.precision == "fp64" else "f32+f64", "data": "synthetic",
            "config": dict(batch_config(args, all_descs), l2="flushed between timed steps (256 MB write)",
                           setup_s=t_setup),
            "forward_only_scene_steps_per_s": world * fwd_rate if world == 1 else None,
            "placement": {"scenes_per_rank": [len(p) for p in placement], "tets_per_rank": loads,
                          "imbalance_max_over_mean": max(loads) / (sum(loads) / world) if sum(loads) else 1.0,
                          "rule": "longest-processing-time on tet counts (diff_fem_b200.shard.assign_scenes)",
                          "measured_on_hardware": world == 1 or "yes (this run)"},
            "pd_iterations_total": int(iters.max(axis=1).sum()),
            "solve": b.solve_mode(), "phase_ms": phases, "factor": {"supernodes": binfo["n_supernodes"],
                                                                   "levels": binfo["n_levels"],
                                                                   "nnz": int(binfo["nnz_factor"])},
            "e2e": e2e, "error_vs_fp64": errs, "plain_fp64_one_at_a_time": plain, "roofline": roofline,
            "gpu_launches": launches, "clocks": clk.summary()}
    if rank == 0:
        print(json.dumps(line), flush=True)
    b.close()
    if world > 1:
        dist.destroy_process_group()


# --------------------------------------------------------- muscle star (C3) ---

STAR_METRIC = "fwd+adjoint sim steps/s (muscle star 9,840 tets on the ground, 384 segments, K=15)"


def run_contact_workload(args, d, metric, workload, act_np=None, grad_key="act"):
    """One scene with contact: n steps forward, then the adjoint of
    L = |x_n - x_0|^2 (the gradient of interest: grad_key)."""
    import torch
    from diff_fem_b200.engine import Scene

    local = int(os.environ.get("LOCAL_RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    sc = Scene(d, device=local)
    n = SIM_STEPS
    act = torch.tensor(act_np, device=dev) if act_np is not None else None
    x0 = torch.tensor(d.x0.reshape(-1), device=dev)
    v0 = torch.zeros_like(x0)
    stream = torch.cuda.current_stream(dev)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)

    def grad_eval():
        x, v = sc.forward(x0, v0, n_steps=n, act=act)
        return x, sc.backward(2.0 * (x - x0), torch.zeros_like(x))

    for _ in range(max(3, args.warmup)):
        grad_eval()
    torch.cuda.synchronize()
    launches0 = sc.launch_count()
    elapsed = 0.0
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            xg, gg = grad_eval()
            e1.record(stream)
            torch.cuda.synchronize()
            elapsed += e0.elapsed_time(e1) / 1e3
    launches = sc.launch_count() - launches0
    if world > 1:
        t = torch.tensor([elapsed], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        elapsed = float(t.item())
    value = world * n * args.steps / elapsed
    passes = sc.contact_passes(n)
    iters = sc.iterations(n)
    x0_h, v0_h = x0.cpu().pin_memory(), v0.cpu().pin_memory()
    act_h = act.cpu().pin_memory() if act is not None else None
    t1 = time.perf_counter()
    for _ in range(args.steps):
        xh, vh = sc.forward(x0_h, v0_h, n_steps=n, act=act_h)
        gh = sc.backward(2.0 * (xh - x0_h.numpy()), np.zeros_like(xh))
        _ = float(np.sum(gh[grad_key]))
    t_e2e = time.perf_counter() - t1
    n3 = 3 * d.n_vertices
    nact = 0 if act_np is None else act_np.size
    line = {"metric": metric, "value": value, "unit": "steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * elapsed / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "f32+f64",
            "data": "synthetic",
            "config": {"workload": workload, "precision": args.precision, "contact_steps": int((passes > 0).sum()),
                       "contact_passes_total": int(passes.sum()), "pd_iterations_total": int(iters.sum()),
                       "solve": sc.solve_mode(), "l2": "flushed between timed steps (256 MB write)"},
            "e2e": {"value": world * n * args.steps / t_e2e, "unit": "steps/s",
                    "h2d_bytes_per_step": 8 * (2 * n3 + nact + 2 * n3),
                    "d2h_bytes_per_step": 8 * (2 * n3 + 2 * n3 + 2 * d.n_tets + nact)},
            "grad_norm": float(torch.linalg.norm(gg[grad_key]).item()),
            "gpu_launches": launches, "clocks": clk.summary()}
    if rank == 0:
        print(json.dumps(line), flush=True)
    sc.close()
    if world > 1:
        dist.destroy_process_group()


def run_cloth_ball(args):
    from diff_fem_b200 import scene as S
    from diff_fem_b200._capi import DFEM_PREC_FP64, DFEM_PREC_MIXED
    prec = DFEM_PREC_FP64 if args.precision == "fp64" else DFEM_PREC_MIXED
    d = S.cloth_on_ball(precision=prec)
    run_contact_workload(args, d, "fwd+adjoint sim steps/s (64x64 cloth on a ball, K=20)",
                         f"cloth 64x64 (4,096 vertices, 12,033 springs, 3,844 bending stencils), membrane 1e3, "
                         f"bending 1e-3, 0.2 kg/m^2, dropped 0.3 m onto a static ball r=0.2 ({len(d.obstacle_faces) - 2} "
                         f"faces) above a ground quad, mu=0.3, h=1/120, K=20, {SIM_STEPS} steps, forward + adjoint dL/dv0",
                         grad_key="v")


def run_star(args):
    """Muscle star on a ground obstacle: 200 steps forward with random chain
    activations, then the gradient of L = |x_200 - x_0|^2 with respect to every
    segment activation of every step (contact phase included in the adjoint)."""
    import torch
    from diff_fem_b200 import scene as S
    from diff_fem_b200._capi import DFEM_PREC_FP64, DFEM_PREC_MIXED
    from diff_fem_b200.engine import Scene

    local = int(os.environ.get("LOCAL_RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    prec = DFEM_PREC_FP64 if args.precision == "fp64" else DFEM_PREC_MIXED
    import dataclasses
    # checkpoints every 20 steps, as the workload specifies (the adjoint regenerates each segment)
    d = dataclasses.replace(S.muscle_star(refine=2, ground=True, mu=0.5, precision=prec), checkpoint_every=20)
    sc = Scene(d, device=local)
    n = SIM_STEPS
    rng = np.random.default_rng(42)
    chains = d.n_segments // 6
    act_np = np.repeat(rng.uniform(0.0, 1.0, (n, chains)), 6, axis=1)  # one value per chain per step
    act = torch.tensor(act_np, device=dev)
    x0 = torch.tensor(d.x0.reshape(-1), device=dev)
    v0 = torch.zeros_like(x0)
    stream = torch.cuda.current_stream(dev)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)

    def grad_eval():
        x, v = sc.forward(x0, v0, n_steps=n, act=act)
        return x, sc.backward(2.0 * (x - x0), torch.zeros_like(x))

    for _ in range(max(3, args.warmup)):
        grad_eval()
    torch.cuda.synchronize()
    launches0 = sc.launch_count()
    elapsed = 0.0
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            xg, gg = grad_eval()
            e1.record(stream)
            torch.cuda.synchronize()
            elapsed += e0.elapsed_time(e1) / 1e3
    launches = sc.launch_count() - launches0
    if world > 1:
        t = torch.tensor([elapsed], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        elapsed = float(t.item())
    value = world * n * args.steps / elapsed
    passes = sc.contact_passes(n)
    iters = sc.iterations(n)
    # end to end with host buffers
    x0_h, v0_h, act_h = x0.cpu().pin_memory(), v0.cpu().pin_memory(), act.cpu().pin_memory()
    t1 = time.perf_counter()
    for _ in range(args.steps):
        xh, vh = sc.forward(x0_h, v0_h, n_steps=n, act=act_h)
        gh = sc.backward(2.0 * (xh - x0_h.numpy()), np.zeros_like(xh))
        _ = float(np.sum(gh["act"]))
    t_e2e = time.perf_counter() - t1
    n3 = 3 * d.n_vertices
    line = {"metric": STAR_METRIC, "value": value, "unit": "steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * elapsed / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "f32+f64",
            "data": "synthetic",
            "config": {"workload": f"muscle star refine 2 ({d.n_tets} tets, {d.n_vertices} vertices), "
                                   f"{chains} chains x 6 segments, ground quad mu=0.5, h=1/60, K=15, {n} steps, "
                                   "activations U[0,1] per chain per step (seed 42), forward + adjoint dL/da, "
                                   f"checkpoints every {d.checkpoint_every} steps",
                       "precision": args.precision, "contact_steps": int((passes > 0).sum()),
                       "contact_passes_total": int(passes.sum()), "pd_iterations_total": int(iters.sum()),
                       "l2": "flushed between timed steps (256 MB write)"},
            "e2e": {"value": world * n * args.steps / t_e2e, "unit": "steps/s",
                    "h2d_bytes_per_step": 8 * (2 * n3 + n * d.n_segments + 2 * n3),
                    "d2h_bytes_per_step": 8 * (2 * n3 + 2 * n3 + 2 * d.n_tets + n * d.n_segments)},
            "grad_act_norm": float(torch.linalg.norm(gg["act"]).item()),
            "gpu_launches": launches, "clocks": clk.summary()}
    if rank == 0:
        print(json.dumps(line), flush=True)
    sc.close()
    if world > 1:
        dist.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "batch":
        run_batch(args)
    elif args.workload == "star":
        run_star(args)
    elif args.workload == "cloth_ball":
        run_cloth_ball(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
