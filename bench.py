#!/usr/bin/env python
"""SIMP iterations/s of the mixed-precision path on the 192x96x96 bridge (1,769,472 Hex8 elements, 5.4M DOFs).

The timed path (--precision, default "mixed-mg") is the mixed-precision form with the multigrid preconditioner:
FP32 inner flexible CG (FP32 K.u and FP32 V-cycle) inside FP64 iterative refinement, FP64 dot products. The
other solver forms run beside it on the same iterations: the plain FP64 path (reference arithmetic), "mixed"
(FP32 inner Jacobi-PCG, the reference's preconditioner), "fp64f" and "mg".

One step = one SIMP iteration (filter, E/DiagA, warm-started PCG to the tolerance, compliance, sensitivities,
adjoint filter, OC bisection) on the device-resident state. Prints one JSON line.

  value      SIMP iter/s with the state resident in HBM (CUDA events on the library's stream, max over ranks)
  e2e        the same metric for a whole job through the C ABI from host buffers: problem upload, W+K
             iterations each followed by the density snapshot read-back (what the App consumes), final u
  roofline   the FP32 stiffness matvec (the dominant kernel), timed live by events captured in the PCG graph
  fp64       the plain FP64 path (bit-exact drop-in) on the same workload, and the timed path's compliance error
  cpu_baseline  the CPU oracle (C++ restatement, all host threads) on a bounded sample of the same iteration
  serving    a bounded sample of the served job stream (p50/p99 latency, aggregate SIMP iter/s)
  batched    the 48 batched instances: packed whole runs (solves in shared launches) against the serving loop

--impl reference runs only the CPU restatement of the reference path (rank 0) on the same workload.
Multi-GPU (torchrun): each rank runs its own replica of the workload (no collective on the data path).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
# the headline metric (the same for both arms)
METRIC = "SIMP iter/s (mixed FP32-inner/FP64-refined, 192x96x96 bridge)"
sys.path.insert(0, ROOT)

# PCG iterations per SIMP iteration of the plain FP64 path on this workload: the mean over SIMP iterations
# 6-25 (the timed iterations of a `--steps 20 --warmup 5` run), 1,810, measured on B200 by the default run's
# fp64 arm, which runs those same iterations (the FP64 path reproduces the reference's iteration counts). Used
# only to scale the CPU sample of the reference arm; the default run uses its own fp64 counts.
FP64_PCG_PER_SIMP_ITER = {"bridge_192x96x96": 1810}

# DRAM bytes per launch of the FP32 matvec (MODE 1) from one ncu capture (dram__bytes_read.sum +
# dram__bytes_write.sum), keyed by (solver form, matvec variant, workload). Jacobi-PCG form (`--probe mixed
# --probe-grid 192x96x96 --probe-variant 3`): 53.47 MB read, 5.53 MB written (K p and p_t mostly stay in the
# 126 MB L2 during the launch).
# Mixed multigrid form (`--probe mixed-mg --probe-grid 192x96x96 --probe-variant 3`, third MODE-1 launch):
# 53.52 MB read, 4.88 MB written.
# Multigrid level-1 residual product (`--probe mixed-mg --probe-grid 192x96x96 --probe-variant 3`, fifth
# k_mg_apply_nodes_tma launch): 127.11 MB read, 5.62 MB written.
NCU_DRAM_BYTES = {("mixed", 3, "bridge_192x96x96"): 53.47e6 + 5.53e6,
                  ("mixed-mg", 3, "bridge_192x96x96"): 53.52e6 + 4.88e6,
                  ("mg-level1", "mixed-mg", "bridge_192x96x96"): 127.11e6 + 5.62e6}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="mycel", choices=["mycel", "reference"])
    ap.add_argument("--workload", default="bridge_192x96x96", choices=["bridge_192x96x96", "cantilever_40x20x10"])
    ap.add_argument("--fp64-steps", type=int, default=-1,
                    help="iterations after the warm-up of the plain FP64 arm run beside the timed form (-1: --steps, "
                         "0: none)")
    ap.add_argument("--profile-steps", type=int, default=5,
                    help="SIMP iterations after the timed ones during which the roofline kernels are timed")
    ap.add_argument("--others-steps", type=int, default=2,
                    help="iterations after the warm-up of the other solver forms (fp64f, mg, mixed)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cpu-sample-iters", type=int, default=6)
    ap.add_argument("--precision", choices=["mixed-mg", "mixed", "mg", "fp64f"], default="mixed-mg",
                    help="solver form of the timed path (value, e2e, roofline, serving sample, batched)")
    ap.add_argument("--probe", choices=["mixed", "fp64", "fp64f", "mg", "mixed-mg"], default=None,
                    help="kernel probe for profilers: one PCG solve of --probe-iters iterations on a bridge grid")
    ap.add_argument("--probe-grid", default="96x48x48")
    ap.add_argument("--probe-iters", type=int, default=40)
    ap.add_argument("--probe-variant", type=int, default=0,
                    help="FP32 matvec variant for --probe mixed (0 autotune, 1 dense, 2 tensor, 3 factored)")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving sample of the default run")
    ap.add_argument("--no-batched-sample", action="store_true", help="skip the batched sample of the default run")
    ap.add_argument("--mv32-variant", type=int, default=0,
                    help="FP32 matvec variant of the timed mixed run (0 autotune; for profiler runs)")
    ap.add_argument("--serve-sample-jobs", type=int, default=12)
    ap.add_argument("--serve-sample-max-elems", type=int, default=250_000)
    ap.add_argument("--serve", action="store_true",
                    help="served job stream only (Poisson arrivals, log-uniform sizes, HBM-budget admission)")
    ap.add_argument("--serve-jobs", type=int, default=500)
    ap.add_argument("--serve-rate", type=float, default=20.0)
    ap.add_argument("--serve-max-elems", type=int, default=1_000_000)
    ap.add_argument("--serve-slots", type=int, default=6)
    ap.add_argument("--serve-budget-gb", type=float, default=150.0)
    ap.add_argument("--serve-precisions", default="mixed-mg,fp64")
    ap.add_argument("--serve-fp64-jobs", type=int, default=None, help="prefix of the stream run in FP64 (default all)")
    ap.add_argument("--static", action="store_true",
                    help="static solve of the sphere-carved 96x48x24 box (about 98k active elements) to 1e-8: plain "
                         "FP64, mixed and fast FP64 paths, and the CPU oracle")
    ap.add_argument("--batched", action="store_true", help="48 independent problems submitted at once")
    ap.add_argument("--surface", action="store_true",
                    help="iso-surface (Surface Nets) of the bridge's physical density after --surface-iters SIMP "
                         "iterations: device time vs the CPU oracle, identical meshes")
    ap.add_argument("--surface-iters", type=int, default=20)
    ap.add_argument("--batched-count", type=int, default=48)
    ap.add_argument("--batched-skip-fp64", action="store_true", help="time only the timed form of --batched")
    ap.add_argument("--batched-iters", type=int, default=4)
    ap.add_argument("--batched-steady-extra", type=int, default=4,
                    help="--batched: also run each form with this many more iterations per problem (steady "
                         "SIMP iter/s from the difference; 0: off)")
    ap.add_argument("--batched-warmup", type=int, default=1,
                    help="--batched: SIMP iterations per problem of an untimed warm-up batch (0: none)")
    ap.add_argument("--batched-lockstep", action="store_true",
                    help="packed batched form: one SIMP iteration of every problem per call (mycel_simp_step_many) "
                         "instead of whole runs in which each problem goes on by itself (mycel_simp_run_many)")
    ap.add_argument("--batched-packs", type=int, default=4,
                    help="packs of the packed batched form (each on its own context and host thread)")
    ap.add_argument("--batched-mode", choices=("packed", "served", "both"), default="both",
                    help="batched timed form: packed launches of all problems (one context), the serving loop's "
                         "slots, or both (FP64 always through the serving loop)")
    ap.add_argument("--batched-cases", choices=("separate", "summed"), default="separate",
                    help="load cases of a batched problem: one solve per case on the shared stiffness (objective "
                         "the sum of the cases' compliances), or summed into one right-hand side as the reference")
    ap.add_argument("--job-tol", type=float, default=1e-8,
                    help="PCG relative residual of the served and batched jobs (every SIMP iteration)")
    return ap.parse_args()


def workload(name):
    from mycel_b200 import workloads as W
    if name == "bridge_192x96x96":
        m, o = W.bridge_192x96x96()
    else:
        m, o = W.simp_cantilever_40x20x10()
    return m, o


def dist_init():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime

        import torch
        import torch.distributed as dist
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    return ws, rank, local


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(ws, v):
    if ws == 1:
        return v
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


class Clocks:
    """nvidia-smi clocks/throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.flush()
        rows = [r.split(",") for r in open(self.f.name).read().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm = [float(r[1]) for r in rows if len(r) >= 9 and r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if len(r) >= 9 and r[2].strip().replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            if len(r) < 9:
                continue
            for k, nm in enumerate(names):
                if "Active" in r[5 + k] and "Not" not in r[5 + k]:
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        return None


def matvec_bytes_fp32(model):
    """Algorithmic bytes of one fused FP32 matvec launch of the inner PCG: read z and p_{t-1}, write p_t and
    K p_t (4 x 12 B per node), E and the domain byte per element (5 B), the node flag byte (1 B)."""
    nn = model.total_nodes
    ne = model.total_elements
    return 48 * nn + 5 * ne + nn


def serve_stream(jobs, precision, slots, budget_bytes, tol, rate_scale=1.0, device=0, ws=1):
    """Submit the jobs at their arrival times to a server and wait for all; returns the stats, per-job
    compliance histories and the wall time. Arrival times are the stream's (seconds from the first)."""
    from mycel_b200 import api
    from mycel_b200 import workloads as W
    specs = [W.served_job(nx, ny, nz, it, seed, precision=precision, tol=tol) for (_t, nx, ny, nz, it, seed) in jobs]
    hist = []
    lat = []
    with api.Server(slots=slots, hbm_budget_bytes=int(budget_bytes), device=device) as srv:
        barrier(ws)
        t0 = time.perf_counter()
        ids = []
        for (arr, *_rest), (m, o) in zip(jobs, specs):
            dt = arr * rate_scale - (time.perf_counter() - t0)
            if dt > 0:
                time.sleep(dt)
            ids.append(srv.submit(m, o))
        srv.wait()
        wall = time.perf_counter() - t0
        st = srv.stats()
        for jid in ids:
            info = srv.info(jid)
            r = srv.result(jid) if info["state"] == "done" else None
            hist.append([h.compliance for h in r["history"]] if r else None)
            if r:
                lat.append(info["finish_s"] - info["submit_s"])
    elems = sum(nx * ny * nz for (_t, nx, ny, nz, _i, _s) in jobs)
    span = st["last_finish_s"] - st["first_submit_s"]
    return {"jobs": len(jobs), "completed": st["completed"], "failed": st["failed"],
            "simp_iterations": st["simp_iterations"], "simp_iter_s": st["simp_iterations"] / span if span > 0 else None,
            "p50_latency_s": st["p50_latency_s"], "p99_latency_s": st["p99_latency_s"],
            "mean_latency_s": st["mean_latency_s"], "p50_queue_s": st["p50_queue_s"], "p99_queue_s": st["p99_queue_s"],
            "peak_admitted_gb": st["peak_admitted_bytes"] / 1e9, "elements_total": elems, "wall_s": wall,
            "_latencies": lat}, hist


def compare_histories(h_mixed, h_fp64):
    """Relative compliance differences, mixed vs FP64, of the same jobs iteration by iteration. Iteration 1
    starts both from the same state (the solver's precision alone); later iterations also carry the
    divergence of the two SIMP trajectories."""
    errs, first = [], []
    for a, b in zip(h_mixed, h_fp64):
        if not a or not b:
            continue
        first.append(abs(a[0] - b[0]) / abs(b[0]))
        for x, y in zip(a, b):
            errs.append(abs(x - y) / abs(y))
    if not errs:
        return None
    return {"max": max(errs), "median": float(np.median(errs)), "iteration1_max": max(first)}


def serving_report(args, n_jobs, max_elems, rate, slots, budget_gb, precisions, fp64_jobs=None):
    from mycel_b200 import workloads as W
    jobs = W.job_stream(n_jobs=n_jobs, rate=rate, seed=11, max_elems=max_elems)
    out = {"stream": {"jobs": n_jobs, "rate_jobs_s": rate, "elements": [8000, max_elems], "iterations": [20, 60],
                      "slots": slots, "hbm_budget_gb": budget_gb, "seed": 11, "pcg_tol": args.job_tol}}
    hists = {}
    for prec in precisions:
        sel = jobs if (prec != "fp64" or fp64_jobs is None) else jobs[:fp64_jobs]
        out[prec], hists[prec] = serve_stream(sel, prec, slots, budget_gb * 1e9, args.job_tol)
        out[prec].pop("_latencies", None)
    if "fp64f" in hists and "fp64" in hists:
        out["rel_compliance_err_fp64f_vs_fp64"] = compare_histories(hists["fp64f"], hists["fp64"])
        if out["fp64"]["simp_iter_s"]:
            out["speedup_fp64f_vs_fp64"] = out["fp64f"]["simp_iter_s"] / out["fp64"]["simp_iter_s"]
    for prec in ("mixed", "mixed-mg", "mg"):
        if prec in hists and "fp64" in hists:
            out[f"rel_compliance_err_{prec}_vs_fp64"] = compare_histories(hists[prec], hists["fp64"])
            n = min(len(hists[prec]), len(hists["fp64"]))
            if out["fp64"]["simp_iter_s"]:
                out[f"speedup_{prec}_vs_fp64"] = out[prec]["simp_iter_s"] / out["fp64"]["simp_iter_s"] \
                    if n == len(hists[prec]) else None
    return out


def run_serve(args):
    """The served stream on this node's GPUs: one process per GPU (torchrun), rank r serves jobs r, r+N, ...
    on its own GPU; the per-job results are merged once at the end (no collective while jobs run)."""
    from mycel_b200 import replicas
    from mycel_b200 import workloads as W
    ws, rank, local = dist_init()
    precisions = [p for p in args.serve_precisions.split(",") if p]
    jobs = W.job_stream(n_jobs=args.serve_jobs, rate=args.serve_rate, seed=11, max_elems=args.serve_max_elems)
    if ws == 1:
        out = {"metric": "served SIMP job stream: p50/p99 job latency and aggregate SIMP iter/s",
               **serving_report(args, args.serve_jobs, args.serve_max_elems, args.serve_rate, args.serve_slots,
                                args.serve_budget_gb, precisions, args.serve_fp64_jobs)}
        for prec in precisions:
            out.get(prec, {}).pop("_latencies", None)
        print(json.dumps(out), flush=True)
        return
    mine = replicas.partition(jobs, rank, ws)
    out = {"metric": "served SIMP job stream: p50/p99 job latency and aggregate SIMP iter/s", "n_gpus": ws,
           "scaling": "strong", "stream": {"jobs": args.serve_jobs, "rate_jobs_s": args.serve_rate,
                                           "pcg_tol": args.job_tol, "slots_per_gpu": args.serve_slots}}
    for prec in precisions:
        r, _h = serve_stream(mine, prec, args.serve_slots, args.serve_budget_gb * 1e9, args.job_tol, device=local,
                             ws=ws)
        out[prec] = replicas.merge({"latencies": r["_latencies"], "simp_iterations": r["simp_iterations"],
                                    "first_submit_s": 0.0, "last_finish_s": r["wall_s"]})
    for prec in precisions:
        if prec != "fp64" and "fp64" in out and out["fp64"]["simp_iter_s"]:
            out[f"speedup_{prec}_vs_fp64"] = out[prec]["simp_iter_s"] / out["fp64"]["simp_iter_s"]
    if rank == 0:
        print(json.dumps(out), flush=True)
    import torch.distributed as dist
    dist.destroy_process_group()


def run_static(args):
    """Static solve to relative residual 1e-8 on the sphere-carved 96x48x24 box: PCG solve time (median of three
    solves from u = 0 on a prepared problem, CUDA events), iterations and the stiffness matvec time per path,
    u and compliance against the plain FP64 result; the CPU oracle (all host threads) on the same solve."""
    import torch
    from mycel_b200 import api
    from mycel_b200 import workloads as W
    model = W.sphere_carved_box()
    ctx = api.Context(0)
    stream = torch.cuda.ExternalStream(ctx.stream, device=torch.device("cuda", 0))
    out = {"metric": "static solve to 1e-8 (sphere-carved 96x48x24 box)", "active_elements": model.active_element_count,
           "dofs": model.total_dofs}
    ref = None
    for prec, slot in (("fp64", 1), ("mixed", 0), ("fp64f", 2), ("mg", 2), ("mixed-mg", 0)):
        pr = api.Problem(model, ctx)
        b = pr.forces()
        pr.pcg_solve(b, tol=1e-8, max_iterations=20000, precision=prec)  # set-up, autotune, graph capture
        times = []
        for rep in range(3):
            ctx.set_profiling(rep == 2)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            u, r = pr.pcg_solve(b, tol=1e-8, max_iterations=20000, precision=prec)
            e1.record(stream)
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1))
        tm = ctx.kernel_timing(slot)
        ctx.set_profiling(False)
        comp = float(np.dot(b, u))
        entry = {"solve_ms": statistics.median(times), "pcg_iterations": r.iterations,
                 "fallback_iterations": r.fallback_iterations, "final_residual": r.final_residual,
                 "matvec_us": 1000.0 * tm["total_ms"] / tm["launches"] if tm["launches"] else None,
                 "compliance": comp}
        if ref is None:
            ref = (u, comp)
        else:
            entry["rel_compliance_err_vs_fp64"] = abs(comp - ref[1]) / abs(ref[1])
            entry["rel_u_err_vs_fp64"] = float(np.abs(u - ref[0]).max() / np.abs(ref[0]).max())
        out[prec] = entry
        pr.close()
    if not args.no_cpu:
        from oracle import oracle as O
        O.set_modes(0, threads=os.cpu_count() or 1)
        t0 = time.perf_counter()
        cres = O.static_run(model, 1e-8, 20000)
        out["cpu_baseline"] = {"solve_ms": (time.perf_counter() - t0) * 1000.0, "cores": os.cpu_count() or 1,
                               "kind": "port", "pcg_iterations": cres.solver_info.iterations,
                               "note": "oracle StaticAnalysis.Run (set-up, solve, post-processing)"}
    print(json.dumps(out), flush=True)


def run_surface(args):
    """Surface Nets of a SIMP design: the 192x96x96 bridge's physical density after --surface-iters iterations of
    the timed form, extracted at threshold 0.5 on the device (median of 3 calls through the C ABI from host
    buffers) and by the CPU oracle (the reference's sequential algorithm, one thread); meshes compared."""
    import torch
    from mycel_b200 import api
    from mycel_b200 import workloads as W
    from mycel_b200.model import GridSpec
    model, opts = W.bridge_192x96x96()
    ctx = api.Context(0)
    prob = api.Problem(model, ctx)
    sess = api.SimpSession(prob, opts.replace(precision=args.precision, max_iterations=args.surface_iters))
    for _ in range(args.surface_iters):
        sess.step()
    rho = sess.read(u=False, densities=True)["physical"]
    sess.close()
    prob.close()
    g = model.grid
    grid = GridSpec(g.nx, g.ny, g.nz, g.h)
    api.SurfaceNetsExtractor.extract(grid, rho, 0.5, ctx=ctx)  # warm-up
    ts = []
    for _ in range(3):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        m = api.SurfaceNetsExtractor.extract(grid, rho, 0.5, ctx=ctx)
        ts.append((time.perf_counter() - t0) * 1000.0)
    out = {"metric": "Surface Nets iso-surface of the bridge design (192x96x96, threshold 0.5)",
           "simp_iterations": args.surface_iters, "vertices": m.vertex_count, "triangles": m.triangle_count,
           "well_composed_passes": m.passes, "resolutions": m.changes,
           "device_ms": statistics.median(ts), "includes": "host density upload, all kernels, mesh read-back"}
    if not args.no_cpu:
        from oracle import oracle as O
        t0 = time.perf_counter()
        pos, idx, info = O.surface_nets(g.nx, g.ny, g.nz, rho, h=float(g.h), threshold=0.5)
        out["cpu_baseline"] = {"ms": (time.perf_counter() - t0) * 1000.0, "cores": 1, "kind": "port",
                               "sample": "the same extraction, oracle restatement of the reference's sequential code"}
        out["identical_to_oracle"] = bool(np.array_equal(pos.view(np.uint32), m.positions.view(np.uint32)) and
                                          np.array_equal(idx, m.indices) and info["passes"] == m.passes)
        out["speedup_vs_cpu"] = out["cpu_baseline"]["ms"] / out["device_ms"]
    # the same grid with a saddle-rich density: every pass of the well-composedness sweep runs
    sd = W.saddle_density(g.nx, g.ny, g.nz, seed=1)
    api.SurfaceNetsExtractor.extract(grid, sd, 0.5, ctx=ctx)
    ts = []
    for _ in range(3):
        t0 = time.perf_counter()
        ms = api.SurfaceNetsExtractor.extract(grid, sd, 0.5, ctx=ctx)
        ts.append((time.perf_counter() - t0) * 1000.0)
    sad = {"vertices": ms.vertex_count, "triangles": ms.triangle_count, "well_composed_passes": ms.passes,
           "resolutions": ms.changes, "device_ms": statistics.median(ts)}
    if not args.no_cpu:
        t0 = time.perf_counter()
        pos, idx, info = O.surface_nets(g.nx, g.ny, g.nz, sd, h=float(g.h), threshold=0.5)
        sad["cpu_ms"] = (time.perf_counter() - t0) * 1000.0
        sad["identical_to_oracle"] = bool(np.array_equal(pos.view(np.uint32), ms.positions.view(np.uint32)) and
                                          np.array_equal(idx, ms.indices) and info["passes"] == ms.passes and
                                          info["changes"] == ms.changes)
    out["saddle_field"] = sad
    print(json.dumps(out), flush=True)


def batched_measure(args):
    """Batched instances: all problems at once; aggregate SIMP iter/s of the timed form in packs (solves in
    shared launches) and through the serving loop's slots, vs FP64. Each form is also run with
    --batched-steady-extra more iterations per problem: the extra iterations over the extra wall time give the
    steady SIMP iter/s, without the one-time problem set-up and tear-down."""
    import threading
    from mycel_b200 import api
    from mycel_b200 import workloads as W
    probs = W.batched_instances(count=args.batched_count)
    sep = args.batched_cases == "separate"
    head = args.precision
    out = {"metric": "batched instances: aggregate SIMP iter/s", "problems": len(probs),
           "iterations_each": args.batched_iters, "pcg_tol": args.job_tol, "load_cases": args.batched_cases,
           "load_cases_total": int(sum(len(bp.load_cases) for bp in probs)),
           "elements_total": int(sum(bp.model.total_elements for bp in probs)),
           "cases_together": os.environ.get("MYCEL_CASES_TOGETHER", "1") != "0"}

    def opts(bp, iters, prec):
        return bp.options.replace(max_iterations=iters, precision=prec, solver_tolerance_initial=args.job_tol,
                                  solver_tolerance_final=args.job_tol, separate_load_cases=sep)

    def packed_run(iters):
        """Packs of problems, each on its own context and host thread; within a pack every problem's session is
        stepped together (mycel_simp_step_many). Problems go largest first (elements x load cases) to the
        lightest pack. Returns (wall s, SIMP iterations, compliance histories, per-pack info)."""
        G = max(1, min(args.batched_packs, len(probs)))
        load = [0] * G
        member = [[] for _ in range(G)]
        for k in sorted(range(len(probs)), key=lambda k: -probs[k].model.total_elements * len(probs[k].load_cases)):
            g = min(range(G), key=lambda q: load[q])
            member[g].append(k)
            load[g] += probs[k].model.total_elements * len(probs[k].load_cases)
        ph = [[] for _ in probs]
        info = [None] * G
        errs = []

        def run_pack(g):
            try:
                ctx = api.Context(0)
                made = []
                for k in member[g]:
                    pr = api.Problem(probs[k].model, ctx)
                    made.append((k, pr, api.SimpSession(pr, opts(probs[k], iters, head))))
                packed0 = ctx.packed_count
                if args.batched_lockstep:  # every SIMP iteration of the pack a barrier (mycel_simp_step_many)
                    while not all(x[2].done for x in made):
                        live = [x for x in made if not x[2].done]
                        for x, r in zip(live, api.SimpSession.step_many([x[2] for x in live])):
                            if r is not None:
                                ph[x[0]].append(r.compliance)
                else:  # whole runs (mycel_simp_run_many): each problem goes on as soon as its own solve ends
                    for x, recs in zip(made, api.SimpSession.run_many([x[2] for x in made])):
                        ph[x[0]].extend(r.compliance for r in recs)
                info[g] = {"problems": len(made), "rhs_solved_packed": ctx.packed_count - packed0}
                for _, pr, se in made:
                    se.close()
                    pr.close()
                ctx.close()
            except Exception as e:  # reported by the caller
                errs.append(repr(e))

        t0 = time.perf_counter()
        ths = [threading.Thread(target=run_pack, args=(g,)) for g in range(G)]
        for t in ths:
            t.start()
        for t in ths:
            t.join()
        wall = time.perf_counter() - t0
        if errs:
            raise RuntimeError("packed batch failed: " + "; ".join(errs))
        return wall, sum(len(h) for h in ph), ph, info

    def served_run(iters, prec):
        """All problems submitted at once to the serving loop (one slot per context and host thread)."""
        with api.Server(slots=args.serve_slots, hbm_budget_bytes=int(args.serve_budget_gb * 1e9)) as srv:
            ids = [srv.submit(bp.model, opts(bp, iters, prec)) for bp in probs]
            srv.wait()
            st = srv.stats()
            hist = [[h.compliance for h in srv.result(j)["history"]] for j in ids]
        return st["last_finish_s"] - st["first_submit_s"], st["simp_iterations"], hist, st

    extra = args.batched_steady_extra
    hists = {}
    if args.batched_warmup > 0:  # one-time costs of the process (matvec autotune per grid, module loads) first
        t0 = time.perf_counter()
        served_run(args.batched_warmup, head)
        out["warmup_s"] = time.perf_counter() - t0

    def measured(name, run):
        wall, n_it, hist, more = run(args.batched_iters)
        rec = {"simp_iter_s": n_it / wall, "wall_s": wall, "simp_iterations": n_it}
        if extra > 0:
            wall2, n_it2, hist2, _ = run(args.batched_iters + extra)
            rec["steady_simp_iter_s"] = (n_it2 - n_it) / (wall2 - wall) if wall2 > wall else None
            rec["wall_s_longer_run"] = wall2
            rec["histories_prefix_consistent"] = all(h2[:len(h)] == h for h, h2 in zip(hist, hist2))
        hists[name] = hist
        return rec, more

    if args.batched_mode in ("packed", "both"):
        rec, info = measured("packed", packed_run)
        rec.update({"packs": len(info), "rhs_solved_packed": sum(x["rhs_solved_packed"] for x in info),
                    "form": head, "note": "packs of problems whose solves share launches (mycel_simp_run_many, or "
                                          "mycel_simp_step_many with --batched-lockstep), the packs on concurrent "
                                          "contexts"})
        out["packed"] = rec
    if args.batched_mode in ("served", "both"):
        rec, st = measured(head, lambda it: served_run(it, head))
        rec.update({"completed": st["completed"], "p50_latency_s": st["p50_latency_s"],
                    "p99_latency_s": st["p99_latency_s"], "slots": args.serve_slots})
        out[head] = rec
    if not args.batched_skip_fp64:
        wall, n_it, hist, st = served_run(args.batched_iters, "fp64")
        out["fp64"] = {"simp_iter_s": n_it / wall, "wall_s": wall, "completed": st["completed"],
                       "p50_latency_s": st["p50_latency_s"], "p99_latency_s": st["p99_latency_s"]}
        hists["fp64"] = hist
    if "packed" in out and head in out:
        out["packed"]["same_histories_as_served"] = hists["packed"] == hists[head]
        out["packed"]["rel_compliance_err_vs_served"] = compare_histories(hists["packed"], hists[head])
        out["packed"]["speedup_vs_served"] = out["packed"]["simp_iter_s"] / out[head]["simp_iter_s"]
        if out["packed"].get("steady_simp_iter_s") and out[head].get("steady_simp_iter_s"):
            out["packed"]["steady_speedup_vs_served"] = (out["packed"]["steady_simp_iter_s"] /
                                                         out[head]["steady_simp_iter_s"])
    if "fp64" in out:
        fast = "packed" if "packed" in out else head
        out[f"speedup_{head}_vs_fp64"] = out[fast]["simp_iter_s"] / out["fp64"]["simp_iter_s"]
        out[f"rel_compliance_err_{head}_vs_fp64"] = compare_histories(hists[fast], hists["fp64"])
    return out


def run_batched(args):
    print(json.dumps(batched_measure(args)), flush=True)


def run_mycel(args):
    import torch
    from mycel_b200 import api
    ws, rank, local = dist_init()
    ctx = api.Context(local)
    model, opts = workload(args.workload)
    head = opts.replace(precision=args.precision)
    stream = torch.cuda.ExternalStream(ctx.stream, device=torch.device("cuda", local))

    # ---------------- value: device-resident SIMP iterations ----------------
    prob = api.Problem(model, ctx)
    if args.mv32_variant:
        prob.set_matvec32(args.mv32_variant)
    sess = api.SimpSession(prob, head)
    for _ in range(args.warmup):
        sess.step()
    launches0 = ctx.launch_count
    clocks = Clocks(local)
    barrier(ws)
    torch.cuda.synchronize(local)
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    recs = [sess.step() for _ in range(args.steps)]
    e1.record(stream)
    torch.cuda.synchronize(local)
    clk = clocks.stop()
    barrier(ws)
    t_ms = e0.elapsed_time(e1)
    gpu_launches = ctx.launch_count - launches0
    t_max = max_over_ranks(ws, t_ms)
    value = ws * args.steps / (t_max / 1000.0)
    # kernel timings for the roofline: the next --profile-steps iterations of the same session, with CUDA
    # event-record nodes around one matvec and one level-1 product per chunk graph (kept out of the timed steps
    # above, whose graphs carry no events)
    ctx.set_profiling(True)
    p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    p0.record(stream)
    n_prof = 0
    for _ in range(args.profile_steps):
        if sess.done:
            break
        sess.step()
        n_prof += 1
    p1.record(stream)
    torch.cuda.synchronize(local)
    timing = ctx.kernel_timing(0)
    timing_l1 = ctx.kernel_timing(3)
    ctx.set_profiling(False)
    prof_window = {"iterations": n_prof, "simp_iter_s": 1000.0 * n_prof / p0.elapsed_time(p1) if n_prof else None}
    # the same kernels timed back to back in one CUDA graph (20 launches between two events, after a warm-up
    # launch): their device time without the event nodes' own cost inside the solver's graphs
    kb_mv = prob.kernel_bench(0, 20)
    kb_l1 = prob.kernel_bench(3, 20) if args.precision in ("mixed-mg", "mg") else None
    pcg_inner = [r.solver_iterations for r in recs]
    comp_head = [r.compliance for r in recs]
    mv_variant = prob.matvec32()
    sess.close()
    prob.close()

    # ---------------- roofline of the FP32 matvec ----------------
    pk = peaks()
    in_solve_ms = timing["total_ms"] / max(1, timing["launches"])
    per_launch_ms = kb_mv / 1000.0
    mv_bytes = matvec_bytes_fp32(model)
    achieved = mv_bytes / (per_launch_ms / 1000.0) / 1e9
    hbm = (pk or {}).get("hbm_gbs") or 6650.0
    kname = {1: "k_mv32 (dense KE rows, FMA pipe)", 2: "k_mv32tc (dense KE, tcgen05 3xTF32)",
             3: "k_mv32f (factorised Hex8 operator, TMA-fed)"}.get(mv_variant, "FP32 matvec")
    traffic = NCU_DRAM_BYTES.get((args.precision, mv_variant, args.workload))
    roof = {"kernel": kname + ": FP32 Hex8 K.p with fused p update + p.Ap partials", "bound": "hbm",
            "achieved": achieved, "peak": hbm, "unit": "GB/s",
            "frac": (achieved / hbm) if achieved else None, "traffic": traffic,
            "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum, one MODE-1 launch of this kernel in "
                              "this solver form on this workload (192x96x96)" if traffic else None,
            "peak_source": "measured" if pk else "fallback", "avg_launch_us": per_launch_ms * 1000.0,
            "timing": "CUDA events around 20 launches back to back in one graph on the library's stream",
            "in_solve_event_us": in_solve_ms * 1000.0 if timing["launches"] else None,
            "in_solve_note": "event-record nodes around one launch per chunk graph during --profile-steps "
                             "iterations; includes the event nodes' own cost",
            "timed_launches": timing["launches"], "algorithmic_bytes_per_launch": mv_bytes,
            "flops_per_launch": 1152 * model.active_element_count, "flops_note": "dense-KE equivalent",
            "tflops": 1152 * model.active_element_count / (per_launch_ms / 1000.0) / 1e12 if timing["launches"] else None}

    # the multigrid level-1 residual product (y = r - A x on the 96x48x48 level, 27-point stencil of 3x3 blocks in
    # half storage): 14 blocks x 9 floats of the node's own rows + x, r, 1/diag read + y written = 552 B per node
    roof_l1 = None
    if kb_l1:
        l1_nodes = (model.grid.nx // 2 + 1 + model.grid.nx % 2) * (model.grid.ny // 2 + 1 + model.grid.ny % 2) * \
            (model.grid.nz // 2 + 1 + model.grid.nz % 2)  # nodes of the level-1 grid (element counts halved, rounded up)
        l1_bytes = 552.0 * l1_nodes
        l1_ach = l1_bytes / (kb_l1 * 1e-6) / 1e9
        roof_l1 = {"kernel": "k_mg_apply_nodes_tma (multigrid level-1 residual product, stencil staged by TMA)",
                   "bound": "hbm",
                   "achieved": l1_ach, "peak": hbm, "unit": "GB/s", "frac": l1_ach / hbm,
                   "traffic": NCU_DRAM_BYTES.get(("mg-level1", args.precision, args.workload)),
                   "peak_source": "measured" if pk else "fallback", "avg_launch_us": kb_l1,
                   "timing": "CUDA events around 20 launches back to back in one graph on the library's stream",
                   "in_solve_event_us": 1000.0 * timing_l1["total_ms"] / timing_l1["launches"]
                   if timing_l1["launches"] else None,
                   "nodes_per_launch": l1_nodes, "algorithmic_bytes_per_launch": l1_bytes, "bytes_per_node": 552}

    out = {"metric": METRIC, "value": value,
           "unit": "SIMP iter/s", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": t_max / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
           "dtype": "f32 inner PCG + f64 refinement/reductions", "data": "synthetic",
           "config": {"workload": args.workload, "elements": model.total_elements, "dofs": model.total_dofs,
                      "precision": args.precision, "volfrac": opts.volume_fraction, "rmin": opts.filter_radius_mm,
                      "penal": opts.penal, "emin_ratio": model.material.emin_ratio,
                      "pcg_tol": opts.solver_tolerance_final, "inputs_vs_l2": "inputs > L2 (126 MB); no flush",
                      "parallelism": f"replicas x{ws}"},
           "roofline": roof, "roofline_mg_level1": roof_l1, "roofline_window": prof_window,
           "gpu_launches": gpu_launches, "clocks": clk,
           "pcg_inner_iters_per_step": pcg_inner, "compliance": comp_head}

    # ---------------- plain FP64 path over the same iterations; the timed form's errors against it ----------------
    # Both forms run from iteration 1 side by side for the timed run's W + K iterations (or W + --fp64-steps):
    # per iteration the relative compliance error, the max-norm relative error of u and the largest absolute
    # difference of the physical densities (values in [0, 1]) of the timed form against the plain FP64 path.
    if args.fp64_steps != 0 and rank == 0:
        n_acc = args.warmup + (args.steps if args.fp64_steps < 0 else args.fp64_steps)
        pa, pb = api.Problem(model, ctx), api.Problem(model, ctx)
        if args.mv32_variant:
            pa.set_matvec32(args.mv32_variant)
        sa = api.SimpSession(pa, head)
        sb = api.SimpSession(pb, opts.replace(precision="fp64"))
        ctx.set_profiling(True)
        f_recs, t64, err_c, err_u, err_d = [], [], [], [], []
        for i in range(n_acc):
            ra = sa.step()
            f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            f0.record(stream)
            rb = sb.step()
            f1.record(stream)
            torch.cuda.synchronize(local)
            f_recs.append(rb)
            if i >= args.warmup:
                t64.append(f0.elapsed_time(f1))
            xa = sa.read(u=True, densities=False, active=True)
            xb = sb.read(u=True, densities=False, active=True)
            err_c.append(abs(ra.compliance - rb.compliance) / abs(rb.compliance))
            err_u.append(float(np.abs(xa["u"] - xb["u"]).max() / np.abs(xb["u"]).max()))
            err_d.append(float(np.abs(xa["rho_phys_active"] - xb["rho_phys_active"]).max()))
        tm64 = ctx.kernel_timing(1)
        ctx.set_profiling(False)
        for q in (sa, sb, pa, pb):
            q.close()
        per64 = tm64["total_ms"] / max(1, tm64["launches"])
        out["fp64"] = {"simp_iter_s": 1000.0 * len(t64) / sum(t64) if t64 else None,
                       "ms_per_step": statistics.mean(t64) if t64 else None,
                       "iterations_timed": f"{args.warmup + 1}..{n_acc}",
                       "pcg_iters_per_step": [r.solver_iterations for r in f_recs[args.warmup:]],
                       "matvec_us": per64 * 1000.0,
                       "matvec_gbs": (48 * model.total_nodes + 9 * model.total_elements) / (per64 / 1000.0) / 1e9 if tm64["launches"] else None}
        out["rel_err_vs_fp64"] = {"iterations": list(range(1, n_acc + 1)), "compliance": err_c, "u": err_u,
                                  "density": err_d, "max_compliance": max(err_c), "max_u": max(err_u),
                                  "max_density": max(err_d),
                                  "definition": "per SIMP iteration from 1, timed form vs plain FP64 run side by side: "
                                                "|C - C64|/|C64|, max|u - u64|/max|u64|, max|rho_phys - rho_phys64|"}
        out["speedup_vs_fp64"] = (value / ws) / out["fp64"]["simp_iter_s"] if out["fp64"]["simp_iter_s"] else None
        # the other solver forms on the first W + --others-steps iterations: speed and compliance error
        others = [("fp64f", "fp64_factored"), ("mg", "fp64_multigrid"), ("mixed", "mixed_jacobi"),
                  ("mixed-mg", "mixed_multigrid")]
        n_oth = min(n_acc, args.warmup + args.others_steps)
        for prec, key in [o for o in others if o[0] != args.precision and args.others_steps > 0]:
            prob = api.Problem(model, ctx)
            sess = api.SimpSession(prob, opts.replace(precision=prec))
            q_recs, tq = [], []
            for i in range(n_oth):
                f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                f0.record(stream)
                q_recs.append(sess.step())
                f1.record(stream)
                torch.cuda.synchronize(local)
                if i >= args.warmup:
                    tq.append(f0.elapsed_time(f1))
            sess.close()
            prob.close()
            qerr = [abs(a.compliance - b.compliance) / abs(b.compliance) for a, b in zip(q_recs, f_recs)]
            out[key] = {"simp_iter_s": 1000.0 * len(tq) / sum(tq) if tq else None,
                        "ms_per_step": statistics.mean(tq) if tq else None,
                        "pcg_iters_per_step": [r.solver_iterations for r in q_recs[args.warmup:]],
                        "max_rel_compliance_err_vs_fp64": max(qerr) if qerr else None,
                        "rel_compliance_err_vs_fp64": qerr}

    # ---------------- e2e: whole job through the C ABI from host buffers ----------------
    if not args.no_e2e:
        barrier(ws)
        torch.cuda.synchronize(local)
        n_it = args.warmup + args.steps
        h2d = model.domain.nbytes + model.element_density.nbytes + model.fixed_dofs.nbytes + \
            sum(lc.patch.nodes.nbytes + lc.patch.node_area.nbytes for lc in model.loads)
        d2h_step = 2 * 4 * model.total_elements + 112
        # the App's buffers for the per-iteration density read-backs: pinned host memory, allocated once
        pin = {k: torch.empty(model.total_elements, dtype=torch.float32, pin_memory=True).numpy()
               for k in ("physical", "design")}
        t0 = time.perf_counter()
        prob = api.Problem(model, ctx)
        sess = api.SimpSession(prob, head.replace(max_iterations=n_it))
        for _ in range(n_it):
            sess.step()
            sess.read(u=False, densities=True, out=pin)
        final = sess.read(u=True, densities=False)
        torch.cuda.synchronize(local)
        t_e2e = time.perf_counter() - t0
        sess.close()
        prob.close()
        t_e2e = max_over_ranks(ws, t_e2e)
        out["e2e"] = {"value": ws * n_it / t_e2e, "unit": "SIMP iter/s",
                      "h2d_bytes_per_step": int(h2d / n_it), "d2h_bytes_per_step": int(d2h_step + final["u"].nbytes / n_it),
                      "iterations": n_it, "includes": "problem upload, set-up, W+K SIMP iterations from iteration 1, "
                                                      "per-iteration float density snapshots into pinned host "
                                                      "buffers, final u"}

    # ---------------- CPU baseline (rank 0, bounded sample) ----------------
    if rank == 0 and not args.no_cpu:
        pcg_per_it = (statistics.mean(out["fp64"]["pcg_iters_per_step"]) if "fp64" in out else
                      FP64_PCG_PER_SIMP_ITER.get(args.workload) or statistics.mean(pcg_inner))
        out["cpu_baseline"] = cpu_sample(model, opts, pcg_per_it, args.cpu_sample_iters)

    # ---------------- serving sample (rank 0): Poisson job stream through the serving loop ----------------
    if rank == 0 and not args.no_serve:
        out["serving"] = serving_report(args, args.serve_sample_jobs, args.serve_sample_max_elems, 20.0,
                                        args.serve_slots, 150.0, [args.precision, "fp64"])
        out["serving"]["note"] = ("bounded sample of the served stream: first jobs of the Poisson(20/s) stream, "
                                  "sizes log-uniform up to serve_sample_max_elems; full stream: bench.py --serve")

    # ---------------- batched sample (rank 0): the 48 batched instances, packed and through the serving loop ---
    if rank == 0 and not args.no_batched_sample:
        ns = argparse.Namespace(**vars(args))
        ns.batched_skip_fp64, ns.batched_steady_extra, ns.batched_mode = True, 0, "both"
        out["batched"] = batched_measure(ns)
        out["batched"]["note"] = ("48 batched instances x 4 SIMP iterations, load cases kept apart, after a "
                                  "one-iteration warm-up batch: packed whole runs (mycel_simp_run_many, 4 packs) "
                                  "against the serving loop; FP64 and steady figures: bench.py --batched")

    if rank == 0:
        print(json.dumps(out), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def cpu_sample(model, opts, pcg_per_simp_iter, sample_iters):
    """Oracle (C++ restatement, OpenMP over all host threads) on a bounded sample of one SIMP iteration:
    the density filter, E/DiagA, `sample_iters` PCG iterations, sensitivities + adjoint filter, OC update.
    One SIMP iteration is estimated as the non-PCG part + pcg_per_simp_iter * (time per PCG iteration)."""
    from oracle import oracle as O
    threads = os.cpu_count() or 1
    O.set_modes(0, threads=threads)
    m = O.Model(model)
    act = model.active_elements
    t = time.perf_counter()
    f = O.Filter(model.grid, model.domain, act, max(1.5, opts.filter_radius_mm / model.grid.h))
    t_setup = time.perf_counter() - t
    rho = np.full(act.size, opts.volume_fraction)
    t = time.perf_counter()
    rb = f.apply(rho)
    dens = np.ones(model.total_elements)
    dens[act] = rb
    m.update_densities(dens, opts.penal)
    t_filter = time.perf_counter() - t
    b = m.forces() * (m.constrained() == 0)
    t = time.perf_counter()
    m.pcg_solve(b, tol=1e-30, max_iter=1)
    t1 = time.perf_counter() - t
    t = time.perf_counter()
    u, res = m.pcg_solve(b, tol=1e-30, max_iter=1 + sample_iters)
    t_pcg = (time.perf_counter() - t - t1) / sample_iters
    t = time.perf_counter()
    dcb = m.sensitivities(u, rb, opts.penal)
    dc = f.adjoint(dcb)
    t_sens = time.perf_counter() - t
    t = time.perf_counter()
    O.oc_update(rho, dc, f.s, None, opts.volume_fraction, opts.move_limit, opts.rho_min, 1.0)
    t_oc = time.perf_counter() - t
    t_iter = t_filter + t_sens + t_oc + pcg_per_simp_iter * t_pcg
    return {"value": 1.0 / t_iter, "unit": "SIMP iter/s", "cores": threads, "kind": "port",
            "sample": (f"oracle on the same workload: filter, E/DiagA, {sample_iters} PCG iterations "
                       f"({t_pcg * 1e3:.1f} ms each), sensitivities + adjoint, OC; SIMP iteration = non-PCG part + "
                       f"{pcg_per_simp_iter:.0f} PCG iterations (the FP64 path's count per iteration)"),
            "pcg_iter_ms": t_pcg * 1e3, "filter_setup_s": t_setup}


def run_reference(args):
    ws, rank, local = dist_init()
    if rank != 0:
        return
    model, opts = workload(args.workload)
    pcg_per_it = FP64_PCG_PER_SIMP_ITER.get(args.workload, 1000)
    vals = []
    for i in range(args.warmup + args.steps):
        t = time.perf_counter()
        r = cpu_sample(model, opts, pcg_per_it, 2)
        if i >= args.warmup:
            vals.append(r["value"])
    v = statistics.mean(vals)
    out = {"impl": "reference", "metric": METRIC,
           "value": v, "unit": "SIMP iter/s", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": {"workload": args.workload},
           "cpu_baseline": {"value": v, "unit": "SIMP iter/s", "cores": r["cores"], "kind": "port",
                            "sample": r["sample"]},
           "e2e": {"value": v, "unit": "SIMP iter/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def run_probe(args):
    """A short PCG solve (fixed iteration count) on a bridge grid: the case the ncu captures in profiles/ use."""
    from mycel_b200 import api, workloads as W
    nx, ny, nz = (int(v) for v in args.probe_grid.split("x"))
    ctx = api.Context(0)
    pr = api.Problem(W.bridge(nx, ny, nz), ctx)
    if args.probe in ("mixed", "mixed-mg", "mg") and args.probe_variant:
        pr.set_matvec32(args.probe_variant)
    u, r = pr.pcg_solve(pr.forces(), tol=1e-30, max_iterations=args.probe_iters, precision=args.probe)
    print(json.dumps({"probe": args.probe, "grid": args.probe_grid, "iterations": r.iterations,
                      "elapsed_ms": r.elapsed_ms, "final_residual": r.final_residual,
                      "matvec32": pr.matvec32() if args.probe in ("mixed", "mixed-mg", "mg") else None}))


if __name__ == "__main__":
    a = parse()
    if a.probe:
        run_probe(a)
    elif a.serve and a.impl != "reference":
        run_serve(a)
    elif a.batched and a.impl != "reference":
        run_batched(a)
    elif a.static and a.impl != "reference":
        run_static(a)
    elif a.surface and a.impl != "reference":
        run_surface(a)
    elif a.impl == "reference":
        run_reference(a)
    else:
        run_mycel(a)
