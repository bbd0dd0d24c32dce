"""Benchmark of the B200 engine on the 3-D compressible Navier-Stokes Taylor-Green vortex, 256^3 cells, one
periodic block (Roe = LMRoe with Mco = 1, MUSCL van Albada, central viscous fluxes, SSP-RK3, CFL 0.8):
cell-updates/s of the mixed form (FP32 flux arithmetic, FP64 state) beside the plain FP64 form, with the
L2 error of the mixed density against the FP64 form after the same steps.

  python bench.py [--gpus N --steps K --warmup W] [--impl reference] [--n 256]

One step = one time step (dt + 3 RK stages) of the whole 256^3 field. Under torchrun every rank runs its own
replica (the path shards by blocks; this config is one block: replicas only, weak scaling), timed with CUDA
events, max over ranks. --impl reference times the CPU restatement of the reference's path (the reference
itself is Fortran/OpenACC/CUDA Fortran and cannot be built here) on the host cores, on a bounded sample.
"""
import argparse
import datetime
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
for _p in (os.path.join(ROOT, "mose-gpu_b200"), os.path.join(ROOT, "oracle")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

METRIC = "cell-updates/s (FP64 vs mixed at stated L2 error)"
UNIT = "cell-updates/s"
B_STAGE = 320            # algorithmic bytes per cell per stage, 3-D NS, FP64 (state read/read/write + geometry)
N_STAGES = 3


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def instructions_per_cell(form):
    """Warp instructions per cell of one sweep launch from the committed ncu summary (None without one)."""
    p = os.path.join(ROOT, "profiles", "sweep_traffic.json")
    if not os.path.exists(p):
        return None
    d = json.load(open(p)).get(form)
    if not d or "warp_instructions" not in d:
        return None
    return float(d["warp_instructions"]) / float(d["cells"])


def traffic_per_launch(n, form):
    """DRAM bytes (read + write) of one sweep launch of `form` from the committed ncu summary, scaled from the
    captured case by the cells processed (the sweep's traffic grows in proportion to them)."""
    p = os.path.join(ROOT, "profiles", "sweep_traffic.json")
    if not os.path.exists(p):
        return None
    d = json.load(open(p)).get(form)
    if not d:
        return None
    return float(d["dram_bytes_per_launch"]) * (n ** 3) / float(d["cells"])


class Clocks:
    """nvidia-smi samples (every 100 ms) kept for the timed region only: the sampler starts before the warm-up,
    mark() and stop() bracket the timed region by host wall-clock, and samples are selected by their own
    timestamps."""

    def __init__(self, idx):
        self.f = os.path.join("/tmp", "mose_clocks_%d_%d.csv" % (os.getpid(), idx))
        q = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        self.t0 = self.t1 = None
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(idx), "--query-gpu=" + q, "--format=csv,noheader,nounits",
                                       "-lms", "100"], stdout=open(self.f, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None
            return
        deadline = time.time() + 5.0            # wait for the first sample so the timed region is covered
        while time.time() < deadline and os.path.getsize(self.f) == 0:
            time.sleep(0.02)

    def mark(self):
        self.t0 = time.time()

    def stop(self):
        self.t1 = time.time()
        if self.p is None:
            return None
        time.sleep(0.25)                         # let the sample that covers the end of the region arrive
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        rows = []
        for line in open(self.f):
            c = [x.strip() for x in line.split(",")]
            if len(c) < 10:
                continue
            try:
                ts = datetime.datetime.strptime(c[0], "%Y/%m/%d %H:%M:%S.%f").timestamp()
            except ValueError:
                continue
            rows.append((ts, c[1:]))
        inside = [r for t, r in rows if self.t0 - 0.1 <= t <= self.t1 + 0.1]
        if not inside and rows:                  # region shorter than the sampling period: nearest sample
            mid = 0.5 * (self.t0 + self.t1)
            inside = [min(rows, key=lambda tr: abs(tr[0] - mid))[1]]
        if not inside:
            return None
        sm = [float(r[1]) for r in inside if r[1].replace(".", "").isdigit()]
        mx = max(float(r[2]) for r in inside)
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[q] for r in inside for q in range(4) if r[5 + q].lower() == "active"})
        load = [v for v in sm if v > 0.5 * mx] or sm
        pw = [float(r[3]) for r in inside if r[3].replace(".", "").isdigit()]
        return {"sm_mhz": statistics.median(load) if load else None, "sm_max_mhz": mx, "reasons": reasons,
                "samples": len(inside), "power_w_median": statistics.median(pw) if pw else None}


def dist_setup(backend=None, timeout_s=600):
    """One process per GPU under torchrun (RANK / LOCAL_RANK / WORLD_SIZE / MASTER_* from the environment): the
    replicas share only the timing reductions. NCCL on GPUs; gloo where there is no GPU (the CPU tests)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        if backend is None:
            backend = "nccl" if torch.cuda.is_available() else "gloo"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
        pg = dist
    return world, rank, local, pg


def max_over_ranks(pg, x, dev):
    """The maximum of x over the ranks (a device time of every rank -> the job's time)."""
    if pg is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def barrier(pg, dev):
    import torch
    if dev.type == "cuda":
        torch.cuda.synchronize(dev)
    if pg is not None:
        pg.barrier()
        if dev.type == "cuda":
            torch.cuda.synchronize(dev)


def cpu_sample(case, min_seconds=10.0, max_steps=3):
    """The CPU restatement on the host cores over a bounded sample of the same workload: whole steps of the
    full field until min_seconds have passed (at most max_steps)."""
    import oracle
    o = oracle.Oracle(case)
    P = case.P0.copy()
    n, t0 = 0, time.perf_counter()
    while n < max_steps:
        rc = o.step(P, 1)
        if rc != 0:
            raise RuntimeError("oracle step failed: %d" % rc)
        n += 1
        if time.perf_counter() - t0 >= min_seconds:
            break
    dt = time.perf_counter() - t0
    return case.n_interior * n / dt, n, dt


def _err_norms(case, a, b):
    """L1 / L2 / Linf of the mixed state b against the FP64 state a, per primitive, relative to a's norms."""
    m = case.interior_mask()
    err = {}
    for q, nm in enumerate(["rho", "u", "v", "w", "p"]):
        x, y = b[q, m], a[q, m]
        d = x - y
        ny = np.abs(y).sum()
        err[nm] = {"L1": float(np.abs(d).sum() / ny) if ny > 0 else float(np.abs(d).sum()),
                   "L2": float(np.sqrt((d * d).sum() / max((y * y).sum(), 1e-300))) if ny > 0 else float(np.sqrt((d * d).sum())),
                   "Linf": float(np.abs(d).max() / max(np.abs(y).max(), 1e-300)) if ny > 0 else float(np.abs(d).max())}
    # the velocity vector against its own magnitude: a component that is near zero everywhere (w of a Taylor-Green
    # field) has a large error relative to its own norm even when the velocity error is small
    dv = np.sqrt(sum((b[q, m] - a[q, m]) ** 2 for q in (1, 2, 3)))
    vm = np.sqrt(sum(a[q, m] ** 2 for q in (1, 2, 3)))
    err["velocity"] = {"L1": float(dv.sum() / max(vm.sum(), 1e-300)),
                       "L2": float(np.sqrt((dv * dv).sum() / max((vm * vm).sum(), 1e-300))),
                       "Linf": float(dv.max() / max(vm.max(), 1e-300))}
    return err


def accuracy_at_config_steps(case, dev, stream, local):
    """The mixed form against both FP64 forms after the config's own step count (case.steps), each form on a fresh
    engine from the initial field, graph-replayed steps."""
    import torch
    from mosegpu import abi
    from mosegpu.engine import Engine
    st = {}
    for name, prec in (("fp64", abi.PREC_FP64), ("fp64_fast", abi.PREC_FP64_FAST), ("mixed", abi.PREC_MIXED)):
        eng = Engine(case, precision=prec, device=local, stream=stream)
        with torch.cuda.stream(stream):
            eng.step(case.steps, graph=True)
        torch.cuda.synchronize(dev)
        if eng.status().code != 0 or eng.status().steps != case.steps:
            raise RuntimeError("%s form did not complete %d steps" % (name, case.steps))
        st[name] = eng.state()
        eng.close()
        del eng
        torch.cuda.empty_cache()
    return _err_norms(case, st["fp64"], st["mixed"]), _err_norms(case, st["fp64_fast"], st["mixed"])


def run_fixed_steps(case, steps, warmup, dev, stream, args=None):
    """Both forms of one case for warmup + steps graph-replayed steps; device time of the timed steps
    (CUDA events on the launching stream), cell-updates/s, launches and the mixed-vs-FP64 error. A profiling run
    (args.tuning set) takes args' forms, steps, warm-up, fixed tile configuration and staging instead."""
    import torch
    from mosegpu import abi
    from mosegpu.engine import Engine
    out = {}
    states = {}
    forms = (("fp64", abi.PREC_FP64), ("mixed", abi.PREC_MIXED))
    prof = args is not None and bool(args.tuning)
    if prof:
        forms = [f for f in forms if f[0] in args.forms.split(",")]
        steps, warmup = args.steps, args.warmup
    for name, prec in forms:
        eng = Engine(case, precision=prec, device=dev.index, stream=stream)
        with torch.cuda.stream(stream):
            eng.step(1, graph=True)
            if prof:
                kc, pers = (int(x) for x in args.tuning.split(","))
                eng.set_tuning(kc, pers)
                tuning = (kc, pers)
                if prec == abi.PREC_MIXED and args.staging != "auto":
                    eng.set_staging(1 if args.staging == "tma" else 0)
            else:
                tuning = eng.autotune()      # k-chunk, queue and (mixed) staging, timed on this state
            eng.step(warmup - 1, graph=True)
        torch.cuda.synchronize(dev)
        l0 = eng.launches
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        with torch.cuda.stream(stream):
            eng.step(steps, graph=True)
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1)
        st = eng.status()
        if st.code != 0:
            raise RuntimeError("%s %s form: %s" % (case.name, name, abi.status_message(st.code)))
        out[name] = {"value": case.n_interior * steps / (ms * 1e-3), "ms_per_step": ms / steps,
                     "gpu_launches": eng.launches - l0, "time": st.time,
                     "tuning": {"k_chunk": tuning[0], "persistent": bool(tuning[1])}}
        if prec == abi.PREC_MIXED:
            out[name]["staging"] = eng.staging_label()
        states[name] = eng.state()
        eng.close()
        del eng
        torch.cuda.empty_cache()
    if "fp64" in out and "mixed" in out:
        out["mixed"]["speedup_vs_fp64"] = out["mixed"]["value"] / out["fp64"]["value"]
        out["mixed_vs_fp64_error_after_%d_steps" % (steps + warmup)] = _err_norms(case, states["fp64"], states["mixed"])
    return out


def run_c3(args, dev, stream):
    """The 2-D multi-block laminar batch: 8 x 6 blocks of seeded widths / heights in [64, 512], 405 inlet M 2,
    400 outlet, 301 walls, AUSM+ / van Leer, RK4, 200 steps, all 48 blocks in one sweep per stage."""
    from mosegpu import case as cs
    t0 = time.time()
    case = cs.multiblock_2d()
    setup = time.time() - t0
    r = run_fixed_steps(case, case.steps - 3, 3, dev, stream, args)
    r["config"] = {"workload": "mb2d_8x6_ns_ausm_vanleer_rk4", "cells": case.n_interior, "blocks": len(case.blocks),
                   "widths": case.meta["widths"], "heights": case.meta["heights"], "steps": case.steps,
                   "setup_s": round(setup, 1)}
    return r


def run_c5(args, dev, stream):
    """The large multi-block 3-D case: 4 x 4 x 4 blocks of 128^3 (134 M cells), TGV at Mach 0.3 with 1e-3 noise,
    HLLC / van Albada, SSP-RK3, 50 steps; the 64 blocks share one device copy of their (equal) geometry."""
    from mosegpu import case as cs
    t0 = time.time()
    case = cs.taylor_green_blocks(nb=4, nblk=128, steps=50)
    setup = time.time() - t0
    r = run_fixed_steps(case, case.steps - 3, 3, dev, stream, args)
    r["config"] = {"workload": "tgv_4x4x4_128_ns_hllc_vanalbada_ssprk3", "cells": case.n_interior,
                   "blocks": len(case.blocks), "steps": case.steps, "setup_s": round(setup, 1)}
    return r


def partition_requests(reqs, world, rank):
    """Serving cases are independent (no exchange between them): rank r of `world` serves requests r, r + world,
    r + 2 world, ... of the one seeded stream every rank builds."""
    return reqs[rank::world]


def merge_serving(parts):
    """One serving summary from every rank's part: (latencies, first arrival, last finish, cell-updates, cases
    completed, failed request ids); the ranks started their request loops together (after a barrier)."""
    lat = np.array(sorted(x for p in parts for x in p[0]))
    done = int(sum(p[4] for p in parts))
    firsts = [p[1] for p in parts if p[1] is not None]
    lasts = [p[2] for p in parts if p[2] is not None]
    span = (max(lasts) - min(firsts)) if (done and firsts and lasts) else float("nan")
    work = float(sum(p[3] for p in parts))
    return {"cases_completed": done, "failed": sorted(x for p in parts for x in p[5]),
            "cases_per_s": done / span if done else 0.0,
            "p50_s": float(np.percentile(lat, 50)) if done else None,
            "p99_s": float(np.percentile(lat, 99)) if done else None,
            "cell_updates_per_s": work / span if done else 0.0, "makespan_s": span}


def run_serving(args, dev, world=1, rank=0, pg=None):
    """A bounded sample of the seeded serving stream (1-D and 2-D Riemann cases, HLLC + minmod, SSP-RK3,
    CFL 0.5, mixed precision) through the continuous-batching server: p50 / p99 time-to-solution (arrival to
    result on the host), cases/s over the run, and the cell-updates/s the batch sustained. Under torchrun the
    cases are partitioned over the ranks (partition_requests) and the summary merges every rank's cases."""
    from mosegpu import abi
    from mosegpu import serving as sv
    t0 = time.time()
    stream = sv.request_stream(n_cases=args.serve_cases, rate=args.serve_rate, seed=20261203)
    reqs_all = [sv.riemann_request(q, d, n, st, te, arrival=t) for q, (t, d, n, st, te) in enumerate(stream)]
    reqs = partition_requests(reqs_all, world, rank)
    setup = time.time() - t0
    # lanes, each its own context and stream: 1-D cases (cheap steps, many of them) and 2-D cases; with three lanes
    # the 2-D cases of N >= serve_split go to a lane of their own, so that a small 2-D case does not advance at the
    # step time of the largest ones
    budget = int(args.serve_budget_gb * 2 ** 30)
    b1 = min(2 << 30, budget // 4)
    nl = 3 if args.serve_lanes == 3 else 2
    shares = [b1] + ([budget - b1] if nl == 2 else [(budget - b1) // 3, budget - b1 - (budget - b1) // 3])
    lanes = [sv.Server(reqs[0].case.scheme, reqs[0].case.thermo, budget_bytes=bb, max_cases=128,
                       precision=abi.PREC_MIXED, device=dev.index, poll_steps=args.serve_poll) for bb in shares]

    def route(r):
        n = r.case.blocks[0]["n"]
        if n[1] == 1:
            return 0
        return 2 if (nl == 3 and n[0] >= args.serve_split) else 1
    if pg is not None:
        barrier(pg, dev)
    done = sv.serve_lanes(lanes, route, reqs, max_wall=args.serve_max_s)
    for lane in lanes:
        lane.close()
    part = ([r.finish - r.arrival for r in done], min(r.arrival for r in reqs) if reqs else None,
            max(r.finish for r in done) if done else None, sum(r.case.n_interior * r.steps for r in done), len(done),
            [r.rid for r in done if r.error is not None or r.status.code != abi.MB_OK])
    parts = [part]
    if pg is not None:
        parts = [None] * world
        pg.all_gather_object(parts, part)
    out = {"cases_submitted": len(reqs_all), **merge_serving(parts), "arrival_rate_per_s": args.serve_rate,
           "poll_steps": args.serve_poll,
           "lanes": ("2 (1-D cases | 2-D cases)" if nl == 2 else
                     "3 (1-D cases | 2-D cases N < %d | 2-D cases N >= %d)" % (args.serve_split, args.serve_split))
           + ", one context and stream each",
           "budget_gb": args.serve_budget_gb, "precision": "mixed", "setup_s": round(setup, 1),
           "sample": "the first %d cases of the seeded 4096-case stream (half 1-D N in [256, 8192], half 2-D N^2 "
                     "with N in [128, 1024], log-uniform), Poisson arrivals" % len(reqs_all)}
    if world > 1:
        out["partition"] = "request q on rank q mod %d, no exchange" % world
    return out


def run_serving_sweep(args, dev, world=1, rank=0, pg=None):
    """The serving sample at each offered rate of --serve-rates: cases/s served, p50 / p99 time-to-solution. The
    sustained rate is the highest offered rate the server keeps up with (served >= 0.9 x offered, the p99 not
    growing by more than half over the previous rate's)."""
    out = {"rates": []}
    sustained, prev_p99 = None, None
    for rate in [float(x) for x in args.serve_rates.split(",")]:
        args.serve_rate = rate
        r = run_serving(args, dev, world, rank, pg)
        out["rates"].append({k: r[k] for k in ("arrival_rate_per_s", "cases_per_s", "p50_s", "p99_s",
                                                "cell_updates_per_s", "cases_completed", "makespan_s")})
        keeps = r["cases_per_s"] >= 0.9 * rate and (prev_p99 is None or r["p99_s"] <= 1.5 * prev_p99)
        if keeps:
            sustained = rate
        prev_p99 = r["p99_s"]
    out["sustained_rate_per_s"] = sustained
    out["sample"] = r["sample"]
    return out


def run_reference(args):
    world, rank, local, pg = int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")), 0, None
    if rank != 0:
        return 0
    from mosegpu import case as cs
    case = cs.taylor_green(n=args.n)
    cores = os.cpu_count()
    vals = []
    nwarm, t0 = 0, time.perf_counter()
    for _ in range(max(1, args.warmup)):      # the requested warm-up steps, stopped after ~30 s of CPU work
        cpu_sample(case, min_seconds=0.0, max_steps=1)
        nwarm += 1
        if time.perf_counter() - t0 > 30.0:
            break
    total_n, total_t = 0, 0.0
    for _ in range(max(1, args.steps)):
        v, n, t = cpu_sample(case, min_seconds=0.0, max_steps=1)
        vals.append(v)
        total_n += n
        total_t += t
        if total_t > 120.0:
            break
    value = case.n_interior * total_n / total_t
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": total_n, "warmup": nwarm, "ms_per_step": 1e3 * total_t / total_n, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded Taylor-Green field)",
            "config": {"workload": "tgv%d_ns_roe_vanalbada_ssprk3" % args.n, "cells": case.n_interior,
                       "steps_timed": total_n},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": "%d whole time step(s) of the %d^3 field, %.1f s, OpenMP over %d threads "
                                       "(the reference's own host build needs nvfortran + FiNeR: unavailable)"
                                       % (total_n, args.n, total_t, cores)},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=60)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--forms", default="fp64,fp64_fast,mixed",
                    help="c2: the forms to time (the headline needs mixed; profiling runs take one form)")
    ap.add_argument("--tuning", default="", help="K,P: k-chunk K and persistent queue P (0/1) instead of the "
                                                  "autotuner (profiling runs)")
    ap.add_argument("--staging", default="auto", choices=["auto", "tma", "plain"],
                    help="the mixed sweep's tile staging: auto = the autotuner's choice")
    ap.add_argument("--serve-rates", default="1.0,1.5,2.0,2.5,3.0",
                    help="serving-sweep: the offered rates (cases/s), each served with --serve-cases cases")
    ap.add_argument("--workload", default="default", choices=["default", "c2", "c3", "c5", "serving", "serving-sweep"],
                    help="default: the 256^3 Taylor-Green headline plus the serving sample and the 2-D batch; "
                         "c2 / c3 / c5 / serving: that workload alone")
    ap.add_argument("--serve-cases", type=int, default=256)
    ap.add_argument("--serve-rate", type=float, default=3.0, help="Poisson arrivals per second")
    ap.add_argument("--serve-budget-gb", type=float, default=32.0)
    ap.add_argument("--serve-poll", type=int, default=16, help="steps between reads of the case clocks")
    ap.add_argument("--serve-lanes", type=int, default=3, choices=[2, 3],
                    help="2: 1-D | 2-D cases; 3: 1-D | small 2-D | large 2-D cases")
    ap.add_argument("--serve-split", type=int, default=512, help="the N of the 2-D cases of the third lane")
    ap.add_argument("--serve-max-s", type=float, default=240.0)
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    args.warmup = max(3, args.warmup)

    import torch
    from mosegpu import abi
    from mosegpu import case as cs
    from mosegpu.engine import Engine
    world, rank, local, pg = dist_setup()
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    if args.workload in ("c3", "c5", "serving", "serving-sweep"):
        stream = torch.cuda.Stream(dev)
        r = {"c3": lambda: run_c3(args, dev, stream), "c5": lambda: run_c5(args, dev, stream),
             "serving": lambda: run_serving(args, dev, world, rank, pg),
             "serving-sweep": lambda: run_serving_sweep(args, dev, world, rank, pg)}[args.workload]()
        if rank == 0:
            print(json.dumps({"workload": args.workload, "n_gpus": world, **r}), flush=True)
        if pg is not None:
            pg.destroy_process_group()
        return 0
    t0 = time.time()
    case = cs.taylor_green(n=args.n)
    setup_s = time.time() - t0
    cells = case.n_interior
    stream = torch.cuda.Stream(dev)
    forms = {}
    forms_run = [f for f in (("fp64", abi.PREC_FP64), ("fp64_fast", abi.PREC_FP64_FAST), ("mixed", abi.PREC_MIXED))
                 if f[0] in args.forms.split(",")]
    for name, prec in forms_run:
        eng = Engine(case, precision=prec, device=local, stream=stream)
        clk = Clocks(local)
        with torch.cuda.stream(stream):
            eng.step(1, graph=True)
            if args.tuning:                  # a fixed tile configuration (profiling runs: no autotuner launches)
                kc, pers = (int(x) for x in args.tuning.split(","))
                eng.set_tuning(kc, pers)
                tuning = (kc, pers)
            else:
                tuning = eng.autotune()      # the sweep's tile configuration, timed on this state
            if prec == abi.PREC_MIXED and args.staging != "auto":
                eng.set_staging(1 if args.staging == "tma" else 0)
            eng.step(args.warmup - 1, graph=True)
        barrier(pg, dev)
        l0 = eng.launches
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        barrier(pg, dev)
        clk.mark()
        e0.record(stream)
        with torch.cuda.stream(stream):
            eng.step(args.steps, graph=True)
        e1.record(stream)
        e1.synchronize()
        barrier(pg, dev)
        ms = max_over_ranks(pg, e0.elapsed_time(e1), dev)
        clocks = clk.stop()
        st = eng.status()
        if st.code != 0:
            raise RuntimeError("%s form: %s" % (name, abi.status_message(st.code)))
        # the dominant kernel alone: the fused sweep of a middle stage, CUDA events on its stream
        with torch.cuda.stream(stream):
            g_ms, s_ms = eng.profile_stage(2, 5)
        forms[name] = dict(eng=eng, ms=ms, launches=eng.launches - l0, clocks=clocks, sweep_ms=s_ms, ghost_ms=g_ms,
                           tuning={"k_chunk": tuning[0], "persistent": bool(tuning[1])})
        if name != "mixed":                  # the mixed form's engine is kept for the e2e leg
            eng.close()
            forms[name]["eng"] = None
            torch.cuda.empty_cache()
    if len(forms) < 3:  # a profiling run of some forms: their times only, no headline line
        out = {"workload": "c2 (%s)" % ",".join(forms), "cells": cells, "steps": args.steps,
               "forms": {k: {"ms_per_step": v["ms"] / args.steps, "sweep_ms": v["sweep_ms"], "tuning": v["tuning"]}
                         for k, v in forms.items()}}
        if "mixed" in forms:
            out["forms"]["mixed"]["staging"] = forms["mixed"]["eng"].staging_label()
        for fm in forms.values():
            if fm["eng"] is not None:
                fm["eng"].close()
        if rank == 0:
            print(json.dumps(out), flush=True)
        if pg is not None:
            pg.destroy_process_group()
        return 0
    # accuracy of the mixed form at the config's step count (100), against the FP64 parity form (the oracle's
    # arithmetic bit for bit, tests/test_gpu_fullsize_oracle.py) and the FP64 production form, from the same field
    err, err_fast = accuracy_at_config_steps(case, dev, stream, local)
    l2_rho = err["rho"]["L2"]
    head = "mixed" if l2_rho <= 1e-5 else "fp64"
    f = forms[head]
    value = world * cells * args.steps / (f["ms"] * 1e-3)
    fp64_value = world * cells * args.steps / (forms["fp64"]["ms"] * 1e-3)
    fast_value = world * cells * args.steps / (forms["fp64_fast"]["ms"] * 1e-3)
    mixed_value = world * cells * args.steps / (forms["mixed"]["ms"] * 1e-3)

    # e2e through the C ABI with host buffers: the initial field uploaded from pinned host memory, each step
    # driven by the reference-facing calls (begin_step, stage 1..3) with the status (dt, time, checks) read
    # back to the host, the final field downloaded to pinned host memory.
    eng = forms[head]["eng"]
    if eng is None:
        eng = forms[head]["eng"] = Engine(case, precision=abi.PREC_FP64, device=local, stream=stream)
    host_in = torch.from_numpy(case.P0).pin_memory()
    host_out = torch.empty_like(host_in).pin_memory()
    barrier(pg, dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    with torch.cuda.stream(stream):
        eng.P.copy_(host_in, non_blocking=True)
        for _ in range(args.steps):
            eng.begin_step()
            for irk in range(1, 4):
                eng.stage(irk)
            st = eng.status()
        host_out.copy_(eng.P, non_blocking=True)
    e1.record(stream)
    e1.synchronize()
    barrier(pg, dev)
    e2e_ms = max_over_ranks(pg, e0.elapsed_time(e1), dev)
    e2e_value = world * cells * args.steps / (e2e_ms * 1e-3)
    state_bytes = case.P0.nbytes

    peak, peak_kind = peaks()
    bytes_launch = cells * B_STAGE
    achieved = bytes_launch / (f["sweep_ms"] * 1e-3) / 1e9
    tkey = head
    if head == "mixed" and f["eng"] is not None and f["eng"].staging_mode() == 1 and f["eng"].staging()[0] > 0:
        tkey = "mixed_tma"               # the capture of the staging the timed sweep used
    tr = traffic_per_launch(args.n, tkey)
    # the bound that holds: instruction issue (ncu warp instructions per cell of the same kernel x cells / the sweep's
    # CUDA-event time, against 4 schedulers x 148 SMs x the SM clock sampled during the timed steps)
    ipc = instructions_per_cell(tkey)
    sm_mhz = (f["clocks"] or {}).get("sm_mhz") if isinstance(f.get("clocks"), dict) else None
    issue = None
    if ipc and sm_mhz:
        nsm = torch.cuda.get_device_properties(dev).multi_processor_count
        rate = ipc * cells / (f["sweep_ms"] * 1e-3)
        issue = {"warp_instructions_per_cell": ipc, "achieved_per_s": rate,
                 "peak_per_s": 4.0 * nsm * sm_mhz * 1e6, "frac": rate / (4.0 * nsm * sm_mhz * 1e6),
                 "source": "ncu smsp__inst_executed.sum at 160^3 (profiles/k_sweep_mixed_tgv160_ncu.md)"}
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": f["ms"] / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 flux / f64 state" if head == "mixed" else "f64",
            "data": "synthetic (seeded Taylor-Green field, dimensional: T0 300 K, Mach 0.1, Re 1600)",
            "config": {"workload": "tgv%d_ns_roe_vanalbada_ssprk3" % args.n, "cells": cells,
                       "block": "1 periodic block", "parallelism": "replicas only (dp%d)" % world,
                       "form": head, "l2_flush": "inputs larger than L2 (state 3 x %.0f MB + geometry)" %
                       (state_bytes / 1e6), "dt_rule": "additive", "setup_s": round(setup_s, 1)},
            "forms": {"fp64": {"value": fp64_value, "ms_per_step": forms["fp64"]["ms"] / args.steps,
                               "sweep_ms": forms["fp64"]["sweep_ms"], "ghost_ms": forms["fp64"]["ghost_ms"],
                               "tuning": forms["fp64"]["tuning"], "clocks": forms["fp64"]["clocks"],
                               "build": "parity form: the reference's statements, no FMA (bit-identical to the oracle)"},
                      "fp64_fast": {"value": fast_value, "ms_per_step": forms["fp64_fast"]["ms"] / args.steps,
                                    "sweep_ms": forms["fp64_fast"]["sweep_ms"],
                                    "ghost_ms": forms["fp64_fast"]["ghost_ms"], "tuning": forms["fp64_fast"]["tuning"],
                                    "clocks": forms["fp64_fast"]["clocks"],
                                    "build": "production form: FP64 values, simplified flux path, FMA (within the "
                                             "1e-12 / 1e-9 gates of the oracle)"},
                      "mixed": {"value": mixed_value, "ms_per_step": forms["mixed"]["ms"] / args.steps,
                                "sweep_ms": forms["mixed"]["sweep_ms"], "ghost_ms": forms["mixed"]["ghost_ms"],
                                "tuning": forms["mixed"]["tuning"], "speedup_vs_fp64": mixed_value / fp64_value,
                                "speedup_vs_fp64_fast": mixed_value / fast_value,
                                "speedup_vs_faster_fp64": mixed_value / max(fp64_value, fast_value)},
                      "mixed_vs_fp64_error_after_%d_steps" % case.steps: err,
                      "mixed_vs_fp64_fast_error_after_%d_steps" % case.steps: err_fast},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": tr, "peak_source": peak_kind,
                         "kernel": "k_sweep<%s> (stage 2)" % ("float" if head == "mixed" else "double"),
                         "staging": f["eng"].staging_label() if head == "mixed" and f["eng"] is not None else None,
                         "algorithmic_bytes_per_launch": bytes_launch, "issue": issue},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": state_bytes / args.steps,
                    "d2h_bytes_per_step": state_bytes / args.steps + 48,
                    "copies": "once per run: the state is uploaded before the first step and downloaded after the "
                              "last (the per-step bytes are those copies divided by the steps), as the reference's "
                              "host loop keeps the field on the device between output iterations "
                              "(Mod_Explicit.f90:300-305); the status (dt, time, checks) is read every step",
                    "path": "C ABI: upload once, per step mb_begin_step + 3 x mb_stage + mb_get_status, download"},
            "gpu_launches": f["launches"], "clocks": f["clocks"]}
    for fm in forms.values():
        if fm["eng"] is not None:
            fm["eng"].close()
    forms.clear()
    torch.cuda.empty_cache()
    if args.workload == "default":
        line["workloads"] = {"serving": run_serving(args, dev, world, rank, pg), "mb2d": run_c3(args, dev, torch.cuda.Stream(dev))}
    if rank == 0 and world == 1 and not args.no_cpu:
        v, n, t = cpu_sample(case, min_seconds=10.0, max_steps=2)
        line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
                                "sample": "%d whole time step(s) of the %d^3 field (%.1f s), OpenMP" % (n, args.n, t)}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if pg is not None:
        pg.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
