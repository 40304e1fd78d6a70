#!/usr/bin/env python
"""Benchmark of the B200 tangent-point path (one JSON line on rank 0).

Workload (the configuration the headline metric is quoted on): torus R=1, r=0.4,
160 x 120 vertex grid (19,200 vertices, 38,400 triangles), normal jitter N(0, 0.002^2),
q=6, p=12, theta=0.5. A step is one energy + differential evaluation of the mesh at the
current coordinates: SemiStaticUpdate (simplex data + cluster-moment upsweep) followed
by TangentPointEnergy0::Differential (near- and far-field pair kernels, collection,
chain rule, vertex scatter). Synthetic seeded inputs stand in for user meshes.

Timing: W warm-up steps, then K steps, each bracketed by CUDA events on the mesh's
stream; before every timed step a 256 MiB device buffer is overwritten (outside the
events) so no step starts with the mesh resident in L2. Multi-GPU runs (torchrun) are
independent replicas, one mesh per GPU (weak scaling); the reported time is the max
over ranks.

--impl reference times the CPU restatement of the reference path (oracle/, FP64,
std::thread) on this host's cores on the same workload.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "energy+grad evals/s; metric-solve ms to 1e-6 res, learned vs plain precond, 1 GPU"
Q, P = 6.0, 12.0
# algorithmic flops per unique pair of the energy+differential traversal with q/2 = 3,
# p/2 = 6 (TP0_Kernel_FF/NF::Compute and the loop bodies around them), counted by the
# oracle's operation-counting scalar (oracle.pair_opcounts; tests/test_opcounts.py keeps
# these equal): far field 56 add + 96 mul + 1 div, near field (triangles) 74 add + 123 mul
# + 1 div
FLOPS_FAR_PAIR = 153.0
FLOPS_NEAR_PAIR = 198.0
# geometry (primitive data + in-block scans), block scan, cluster moments, near and far
# pairs (one launch), collect + chain rule, vertex gather
LAUNCHES_PER_STEP = 6


def max_over_ranks(x, dist, device):
    """The slowest rank's time (replicas run the same work; the job ends with the slowest)."""
    if not dist:
        return x
    import torch

    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(world, steps_per_rank, max_ms):
    """Whole-job evaluations per second: every rank evaluates its own mesh `steps_per_rank`
    times; the job takes the slowest rank's `max_ms`."""
    return world * steps_per_rank / (max_ms * 1e-3)


def pair_traffic_from_profile():
    """DRAM bytes (read + write) of the merged pair launch of one evaluation, from the ncu
    capture summarised in profiles/k_tp0_pairs_tiled_both_torus160x120.md (null if absent)."""
    import re
    path = os.path.join(ROOT, "profiles", "k_tp0_pairs_tiled_both_torus160x120.md")
    if not os.path.exists(path):
        return None
    m = re.search(r"DRAM bytes per evaluation[^:]*:\s*([0-9,]+)", open(path).read(), re.IGNORECASE)
    return int(m.group(1).replace(",", "")) if m else None


def stage_rooflines(st, ms):
    """HBM roofline of the two non-pair stages of a step (triangles): algorithmic bytes,
    each array read or written once, divided by the stage's CUDA-event time.
    geometry + upsweep: perm, simplices, coordinates and the written primitive data and
    in-block prefix rows, then the prefix rows read back, the cluster ranges and the
    written cluster data: N (4 + 12 + 64 + 80 + 80) + nV 24 + NC (8 + 64) bytes.
    collection + gather: perm, simplices, coordinates, leaf index, near rows, far rows, the
    clusters' data and tree links, the written and re-read per-corner derivatives, the
    vertex-to-corner lists and the output: N (4 + 12 + 4 + 80 + 72 + 72 + 12) +
    NC (80 + 64 + 8) + nV (24 + 4 + 24) bytes."""
    N, NC, nV = st["simplex_count"], st["cluster_count"], st["vertex_count"]
    peak = measured_hbm_gbs()
    out = {}
    for name, nbytes, t in (("geometry_upsweep", N * 240 + nV * 24 + NC * 72, ms[0]),
                            ("collect_chain_gather", N * 256 + NC * 152 + nV * 52, ms[3])):
        gbs = nbytes / (t * 1e-3) / 1e9
        out[name] = {"bytes": nbytes, "ms": t, "achieved_gbs": gbs, "peak_gbs": peak,
                     "frac": gbs / peak if peak else None}
    return out


def measured_hbm_gbs():
    """HBM copy bandwidth measured on this pool's B200s (MEASURED_PEAKS.json), else the
    pool's earlier measurement."""
    try:
        return float(json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"])
    except (OSError, KeyError, ValueError):
        return 6650.0


def workload_mesh():
    from repulsor_b200 import meshes
    return meshes.torus(R=1.0, r=0.4, n_major=160, n_minor=120, jitter=0.002, seed=1002)


WORKLOAD = {"workload": "torus R=1 r=0.4 160x120 (19,200 vertices, 38,400 triangles), q=6 p=12 theta=0.5",
            "step": "SemiStaticUpdate + Differential (energy + dE, FP32 pair kernels with FP64 near-field projections), "
                    "one CUDA graph per step",
            "l2": "256 MiB buffer overwritten before every timed step"}
REFERENCE_STEP = ("SemiStaticUpdate + Differential in FP64 on host threads: the CPU restatement of the reference "
                  "path (oracle/tp0_oracle.cpp built with the reference's flags -O3 -ffast-math -fno-math-errno), "
                  "rows split over std::threads as the reference's FMM traversor splits them")


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    FIELDS = ["index", "clocks.sm", "clocks.max.sm", "power.draw", "clocks_event_reasons.active",
              "clocks_event_reasons.hw_slowdown", "clocks_event_reasons.hw_thermal_slowdown",
              "clocks_event_reasons.sw_thermal_slowdown", "clocks_event_reasons.sw_power_cap"]

    def __init__(self, device_index):
        self.path = tempfile.mktemp(suffix=".csv")
        self.proc = None
        self.device_index = device_index

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={','.join(self.FIELDS)}", "--format=csv,noheader,nounits",
                 "-i", str(self.device_index), "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        self.proc.wait()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_baseline(V, S, budget_s=20.0, max_evals=30):
    """CPU restatement of the reference path (oracle port, FP64, std::thread over all
    host cores) on the same mesh: SemiStaticUpdate + Differential per evaluation."""
    import numpy as np

    import oracle

    oracle.use_timed_build()
    threads = os.cpu_count() or 1
    O = oracle.OracleMesh(2, V, S, threads=threads)
    Y = np.zeros_like(V)
    O.semistatic_update(V)
    O.differential(Q, P, 1.0, 0.0, Y)   # warm-up
    n = 0
    t0 = time.perf_counter()
    while n < max_evals and time.perf_counter() - t0 < budget_s:
        O.semistatic_update(V)
        O.differential(Q, P, 1.0, 0.0, Y)
        n += 1
    dt = time.perf_counter() - t0
    return {"value": n / dt, "unit": "evals/s", "cores": threads, "kind": "port",
            "sample": f"{n} full evaluations (SemiStaticUpdate + Differential) of the benchmark mesh, "
                      f"{dt:.1f} s, oracle/tp0_oracle.cpp FP64 (-O3 -ffast-math, the reference's flags) with "
                      f"{threads} std::threads"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    V, S = workload_mesh()
    import numpy as np

    import oracle

    oracle.use_timed_build()
    threads = os.cpu_count() or 1
    O = oracle.OracleMesh(2, V, S, threads=threads)
    Y = np.zeros_like(V)
    for _ in range(max(1, args.warmup)):
        O.semistatic_update(V)
        O.differential(Q, P, 1.0, 0.0, Y)
    steps = max(1, min(args.steps, 50))
    t0 = time.perf_counter()
    for _ in range(steps):
        O.semistatic_update(V)
        O.differential(Q, P, 1.0, 0.0, Y)
    dt = time.perf_counter() - t0
    value = steps / dt
    out = {"impl": "reference", "metric": METRIC, "value": value, "unit": "evals/s", "n_gpus": args.gpus,
           "steps": steps, "warmup": args.warmup, "ms_per_step": 1e3 * dt / steps, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded torus)",
           "config": dict(WORKLOAD, step=REFERENCE_STEP, parallelism="host threads"),
           "cpu_baseline": {"value": value, "unit": "evals/s", "cores": threads, "kind": "port",
                            "sample": f"{steps} evaluations of the benchmark mesh (steps capped at 50)"},
           "e2e": {"value": value, "unit": "evals/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true")
    ap.add_argument("--no-solve", action="store_true", help="skip the Solve timings on the icosphere level-6 mesh")
    ap.add_argument("--no-graph", action="store_true", help="time direct launches instead of a captured CUDA graph")
    ap.add_argument("--flow-max-iter", type=int, default=100000, help="iteration limit of the full-flow Solve")
    ap.add_argument("--flow", action="store_true",
                    help="only the full flow step on two linked tori (1,228,800 triangles) with an obstacle")
    ap.add_argument("--learned", action="store_true",
                    help="only configuration 4: train the learned preconditioner on seeded icospheres of levels 5-7 "
                         "and evaluate it on held-out meshes")
    ap.add_argument("--learned-train", type=int, default=256, help="training meshes (configuration 4: 256)")
    ap.add_argument("--learned-rhs", type=int, default=8, help="right-hand sides per training mesh (8)")
    ap.add_argument("--learned-heldout", type=int, default=32, help="held-out meshes (32)")
    ap.add_argument("--learned-steps", type=int, default=30, help="unrolled CG iterations of the training loss")
    ap.add_argument("--learned-lr", type=float, default=1e-3, help="Adam learning rate")
    ap.add_argument("--learned-hybrid", action="store_true",
                    help="train the network as the learned part of the hybrid preconditioner P_ref + w M")
    ap.add_argument("--learned-hard", type=int, default=0,
                    help="train on the residuals left after this many flexible-CG iterations with the untrained "
                         "operator (repulsor_b200.learned.slow_residual) instead of N(0,1) right-hand sides")
    ap.add_argument("--sharded", action="store_true",
                    help="strong scaling: one mesh (the two linked tori) row-sharded over the ranks, one NCCL "
                         "all-reduce of the derivative buffers per evaluation")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        return run_reference(args)
    if args.flow:
        return run_flow(args)
    if args.learned:
        return run_learned(args)
    if args.sharded:
        return run_sharded(args)

    import numpy as np
    import torch

    import repulsor_b200 as rpb

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))

    V, S = workload_mesh()
    M = rpb.SimplicialMesh(V, S, device=local_rank)
    tpe = rpb.TangentPointEnergy0(Q, P)
    st = M.stats()
    Vd = torch.tensor(V, device="cuda")
    Yd = torch.zeros((V.shape[0], 3), dtype=torch.float64, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    # the mesh works on a torch stream so that a step can be captured into a CUDA graph
    ext = torch.cuda.Stream()
    M.set_stream(ext.cuda_stream)

    def step():
        # the energy stays on the device (no host read per step); e2e below reads it back
        M.SemiStaticUpdateDevice(Vd.data_ptr())
        tpe.DifferentialDevice(M, Yd.data_ptr(), 3, 1.0, 0.0, want_energy=False)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    # one step as a CUDA graph (7 nodes: the coordinate copy and the six kernels), replayed
    # per timed step; direct launches if capture is not possible
    graph = None
    if not args.no_graph:
        try:
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g, stream=ext):
                step()
            torch.cuda.synchronize()
            graph = g
        except Exception as exc:   # noqa: BLE001 - capture is an optimisation only
            print(f"CUDA graph capture failed ({exc}); timing direct launches", file=sys.stderr)
            graph = None
        M.set_stream(ext.cuda_stream)
    run_step = graph.replay if graph is not None else step
    for _ in range(args.warmup):
        with torch.cuda.stream(ext):
            run_step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    sampler = ClockSampler(local_rank)
    sampler.start()
    time.sleep(0.3)
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    torch.cuda.synchronize()
    for k in range(args.steps):
        with torch.cuda.stream(ext):
            flush.fill_(k & 0xFF)
            starts[k].record(ext)
            run_step()
            ends[k].record(ext)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    time.sleep(0.3)
    clocks = sampler.stop()
    total_ms = max_over_ranks(sum(s.elapsed_time(e) for s, e in zip(starts, ends)), dist, "cuda")
    value = replica_throughput(world, args.steps, total_ms)

    # end to end through the public API with pinned host buffers (H2D of V, D2H of dE and E)
    Vh = torch.tensor(V).pin_memory()
    Yh = torch.zeros((V.shape[0], 3), dtype=torch.float64).pin_memory()
    Vn, Yn = Vh.numpy(), Yh.numpy()
    e2e_steps = max(10, min(args.steps, 500))
    for _ in range(3):
        M.SemiStaticUpdate(Vn)
        tpe.Differential(M, 1.0, 0.0, Yn)
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        M.SemiStaticUpdate(Vn)
        tpe.Differential(M, 1.0, 0.0, Yn)
    e2e_s = max_over_ranks(time.perf_counter() - t0, dist, "cuda")
    e2e = {"value": replica_throughput(world, e2e_steps, e2e_s * 1e3), "unit": "evals/s", "h2d_bytes_per_step": V.nbytes,
           "d2h_bytes_per_step": Yn.nbytes + 8,
           "how": "SimplicialMesh.SemiStaticUpdate(host V) + TangentPointEnergy0.Differential(M, 1, 0, host Y), "
                  "pinned host buffers, wall clock per step"}

    out = None
    if rank == 0:
        # roofline of the dominant kernel (pair kernels), timed on the launching stream
        import ctypes

        lib = rpb._capi.load()
        ms = np.zeros(5)
        rpb._capi.check(lib.rpb_tpe0_stage_times(M._h, Q, P, 50, 256 << 20, rpb._capi.dptr(ms)), "stage_times")
        peak = ctypes.c_double()
        rpb._capi.check(lib.rpb_measure_fp32_peak(local_rank, ctypes.byref(peak)), "fp32_peak")
        near_pairs = st["near_nnz"] / 2
        far_pairs = st["far_nnz"] / 2
        pair_ms = ms[1] + ms[2]
        flops = FLOPS_NEAR_PAIR * near_pairs + FLOPS_FAR_PAIR * far_pairs
        achieved = flops / (pair_ms * 1e-3) / 1e12
        traffic = pair_traffic_from_profile()
        roofline = {"bound": "fp32", "achieved": achieved, "peak": peak.value, "unit": "TFLOP/s",
                    "frac": achieved / peak.value, "traffic": traffic,
                    "kernel": "k_tp0_pairs_tiled (near and far patterns timed as separate launches; one "
                              "k_tp0_pairs_tiled_both launch in the step)",
                    "peak_source": "measured FP32 FMA throughput (rpb_measure_fp32_peak); MEASURED_PEAKS.json "
                                   "has no FP32 figure",
                    "flops_per_evaluation": flops,
                    "stage_ms": {"geometry_upsweep": ms[0], "near_pairs": ms[1], "far_pairs": ms[2],
                                 "collect_chain_gather": ms[3], "total": ms[4]},
                    "stages": stage_rooflines(st, ms)}
        out = {"metric": METRIC, "value": value, "unit": "evals/s", "n_gpus": world, "steps": args.steps,
               "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
               "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
               "data": "synthetic (seeded torus; no dataset involved)",
               "config": dict(WORKLOAD, parallelism=f"replicas x{world}", near_nnz=st["near_nnz"],
                              far_nnz=st["far_nnz"], clusters=st["cluster_count"]),
               "clocks": clocks, "e2e": e2e, "gpu_launches": LAUNCHES_PER_STEP * args.steps,
               "roofline": roofline}
        if not args.no_cpu_baseline:
            out["cpu_baseline"] = cpu_baseline(V, S)
        if not args.no_extras:
            out["extras"] = extras(rpb, torch, not args.no_solve)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if out is not None:
        print(json.dumps(out))
    return 0


def extras(rpb, torch, with_solve):
    """Metric matvecs/s and Solve time on the icosphere level-6 configuration."""
    from repulsor_b200 import meshes

    V, S = meshes.icosphere_sh(level=6, seed=1003)
    M = rpb.SimplicialMesh(V, S)
    tpm = rpb.TangentPointMetric0(Q, P)
    X = torch.randn((V.shape[0], 3), dtype=torch.float64, device="cuda")
    Y = torch.zeros_like(X)
    ext = torch.cuda.ExternalStream(M.stream())
    for _ in range(5):
        tpm.MultiplyMetricDevice(M, 1.0, X.data_ptr(), 0.0, Y.data_ptr())
    torch.cuda.synchronize()
    n = 200
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(ext)
    for _ in range(n):
        tpm.MultiplyMetricDevice(M, 1.0, X.data_ptr(), 0.0, Y.data_ptr())
    b.record(ext)
    torch.cuda.synchronize()
    mv_ms = a.elapsed_time(b) / n
    st = M.stats()
    N, NC, nV = st["simplex_count"], st["cluster_count"], st["vertex_count"]
    # algorithmic bytes of one product: per full-pattern nonzero two FP32 values and a column
    # index; row pointers; the FP64 12-wide primitive and cluster buffers read and written;
    # the Pre/Post operator (3 indices + 12 FP64 coefficients per primitive) applied twice;
    # the input, output and one intermediate vertex vector
    mv_bytes = ((st["near_nnz"] + st["far_nnz"]) * 12 + (N + NC) * 8 + (N + NC) * 96 * 2
                + N * (3 * 4 + 12 * 8) * 2 + nV * 24 * 3)
    peak = measured_hbm_gbs()
    achieved = mv_bytes / (mv_ms * 1e-3) / 1e9
    out = {"metric_matvec": {"workload": "icosphere level 6 (81,920 triangles), nrhs=3",
                             "matvecs_per_s": 1e3 / mv_ms, "ms": mv_ms,
                             "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                                          "frac": achieved / peak if peak else None, "bytes_per_product": mv_bytes,
                                          "note": "the block SpMM is bound by L1 request throughput on the "
                                                  "96-byte input gathers, not by HBM"}}}
    # collision-free step size along the negative differential of the same mesh, scaled so
    # that the fastest vertex moves by 5 mean edge lengths at t = 1
    import numpy as np

    Dd = rpb.TangentPointEnergy0(Q, P).Differential(M)
    edge = float(np.linalg.norm(V[S[:, 1]] - V[S[:, 0]], axis=1).mean())
    vel = -Dd * (5.0 * edge / max(float(np.abs(Dd).max()), 1e-300))
    M.MaximumSafeStepSize(vel, 1.0)
    t0 = time.perf_counter()
    reps = 5
    for _ in range(reps):
        t_step = M.MaximumSafeStepSize(vel, 1.0)
    out["step_size"] = {"workload": "icosphere level 6, velocities -dE scaled to 5 mean edge lengths, max_time 1, "
                                    "TOL 1/16", "ms": 1e3 * (time.perf_counter() - t0) / reps, "t": t_step,
                        "how": "host candidate traversal + GPU bisections, wall clock per call"}
    if not with_solve:
        return out
    out["solve"] = solve_extras(rpb, M, tpm, V)
    return out


def train_learned_small(rpb, tpm, epochs=3, steps=30, lr=1e-3):
    """The learned preconditioner trained on GPU for the default extras and the flow:
    six seeded spherical-harmonic icospheres (levels 4 and 5, seeds 3001-3006), two N(0,1)
    right-hand sides each, `epochs` passes of the unrolled-CG energy loss over `steps`
    preconditioned CG iterations (repulsor_b200.learned.train_unrolled), starting from the
    multilevel operator (output layer zero: every gain 1). Returns (net, prior, info)."""
    from repulsor_b200 import meshes
    from repulsor_b200.learned import NPARAM_OUTPUT_OFFSET, LearnedPreconditioner, train_unrolled

    t0 = time.perf_counter()
    samples = []
    for lvl, seed in ((4, 3001), (4, 3002), (5, 3003), (5, 3004), (4, 3005), (5, 3006)):
        Vt, St = meshes.icosphere_sh(level=lvl, seed=seed)
        Mt = rpb.SimplicialMesh(Vt, St)
        for j in range(2):
            samples.append((Mt, meshes.random_rhs(Vt.shape[0], seed=10 * seed + j, project=True)))
    t1 = time.perf_counter()
    net = LearnedPreconditioner(seed=1)
    th = net.get_params()
    th[NPARAM_OUTPUT_OFFSET:] = 0.0
    net.set_params(th)
    prior = LearnedPreconditioner(params=th.copy())
    hist = train_unrolled(net, tpm, samples, epochs=epochs, lr=lr, steps=steps, seed=0)
    t2 = time.perf_counter()
    info = {"meshes": "icosphere_sh levels 4 and 5 (seeds 3001-3006), 2 RHS each", "samples": len(samples),
            "loss": "unrolled CG energy -sum log(-phi(x_K)), K = %d" % steps, "epochs": epochs,
            "mesh_setup_s": t1 - t0, "training_s": t2 - t1, "loss_first_epoch": hist[0], "loss_last_epoch": hist[-1]}
    return net, prior, info


def run_learned(args):
    """Configuration 4: the learned preconditioner trained on seeded icospheres of levels
    5, 6 and 7 (spherical-harmonic displacement, 20,480-327,680 triangles) with
    args.learned_rhs N(0,1) right-hand sides each, by the unrolled-CG energy loss, and
    evaluated on args.learned_heldout held-out meshes (the same family, other seeds) by
    iterations and ms to the 1e-6 true residual: flexible CG with the trained network,
    the same with the untrained multilevel operator (every gain 1), plain CG, CG with the
    reference preconditioner (its H1 factorization timed apart), and flexible CG with the
    hybrid preconditioner (reference plus network) for both networks. Training time is
    reported separately. One JSON line."""
    import numpy as np
    import torch

    import repulsor_b200 as rpb
    from repulsor_b200 import meshes
    from repulsor_b200.learned import NPARAM_OUTPUT_OFFSET, LearnedPreconditioner, slow_residual, train_unrolled

    torch.cuda.set_device(0)
    tpm = rpb.TangentPointMetric0(Q, P)
    levels = (5, 6, 7)
    net = LearnedPreconditioner(seed=1)
    th = net.get_params()
    th[NPARAM_OUTPUT_OFFSET:] = 0.0
    net.set_params(th)
    prior = LearnedPreconditioner(params=th.copy())
    t0 = time.perf_counter()
    setup_s, losses = 0.0, []
    for i in range(args.learned_train):
        ts = time.perf_counter()
        V, S = meshes.icosphere_sh(level=levels[i % 3], seed=5000 + i)
        M = rpb.SimplicialMesh(V, S)
        samples = [(M, meshes.random_rhs(V.shape[0], seed=100 * (5000 + i) + j)) for j in range(args.learned_rhs)]
        if args.learned_hard > 0:
            samples = [(M, slow_residual(prior, M, tpm, rhs, args.learned_hard)) for _, rhs in samples]
        setup_s += time.perf_counter() - ts
        losses += train_unrolled(net, tpm, samples, epochs=1, lr=args.learned_lr, steps=args.learned_steps, seed=i,
                                 hybrid=args.learned_hybrid)
        del M, samples
    train_s = time.perf_counter() - t0 - setup_s
    rows = []
    for j in range(args.learned_heldout):
        V, S = meshes.icosphere_sh(level=levels[j % 3], seed=9000 + j)
        M = rpb.SimplicialMesh(V, S)
        b = meshes.random_rhs(V.shape[0], seed=9000 + j)
        row = {"level": levels[j % 3], "seed": 9000 + j}
        for name, pc, n in (("plain_cg", rpb.PRECOND_NONE, None), ("untrained_fcg", rpb.PRECOND_LEARNED, prior),
                            ("trained_fcg", rpb.PRECOND_LEARNED, net), ("reference_cg", rpb.PRECOND_REFERENCE, None),
                            ("untrained_hybrid_fcg", rpb.PRECOND_HYBRID, prior),
                            ("trained_hybrid_fcg", rpb.PRECOND_HYBRID, net)):
            if n is not None:
                n.attach(M)
            if pc == rpb.PRECOND_REFERENCE:
                t = time.perf_counter()
                tpm.MultiplyPreconditioner(M, 1.0, b)
                row["reference_setup_ms"] = 1e3 * (time.perf_counter() - t)
            torch.cuda.synchronize()
            t = time.perf_counter()
            tpm.Solve(M, 1.0, b, max_iter=40000, tolerance=1e-6, precond=pc, strict=False)
            ms = 1e3 * (time.perf_counter() - t)
            rr = max(float(x) for x in tpm.Solver_RelativeResiduals())
            row[name] = {"iterations": tpm.Solver_IterationCount(), "ms": ms, "rel_residual": rr,
                         "fallback_iteration": tpm.SolveInfo(M)["fallback_iteration"]}
        rows.append(row)
        del M

    SOLVERS = ("plain_cg", "untrained_fcg", "trained_fcg", "reference_cg", "untrained_hybrid_fcg",
               "trained_hybrid_fcg")

    def mean(name, key, lvl=None):
        v = [r[name][key] for r in rows if lvl is None or r["level"] == lvl]
        return float(np.mean(v)) if v else None

    summary = {name: {"iterations": mean(name, "iterations"), "ms": mean(name, "ms"),
                      "per_level": {lvl: {"iterations": mean(name, "iterations", lvl), "ms": mean(name, "ms", lvl)}
                                    for lvl in levels}}
               for name in SOLVERS}
    out = {"metric": "learned preconditioner: held-out solve iterations and ms to 1e-6 true residual", "unit": "ms",
           "workload": f"icosphere_sh levels 5-7: {args.learned_train} training meshes x {args.learned_rhs} RHS "
                       f"(seeds 5000+), {args.learned_heldout} held-out meshes (seeds 9000+), q=6 p=12 theta=0.5",
           "training": {"loss": f"unrolled CG energy, K = {args.learned_steps} iterations", "lr": args.learned_lr,
                        "preconditioner_trained": "hybrid P_ref + w M" if args.learned_hybrid else "M alone",
                        "rhs": (f"residuals after {args.learned_hard} untrained flexible-CG iterations"
                                if args.learned_hard > 0 else "N(0,1), mean-free"),
                        "samples": args.learned_train * args.learned_rhs, "training_s": train_s,
                        "mesh_setup_s": setup_s, "loss_first_mesh": float(np.mean(losses[:args.learned_rhs])),
                        "loss_last_mesh": float(np.mean(losses[-args.learned_rhs:]))},
           "summary": summary, "all_converged": all(r[n]["rel_residual"] <= 1e-6 for r in rows for n in SOLVERS),
           "held_out": rows}
    print(json.dumps(out))
    return 0


def solve_extras(rpb, M, tpm, V):
    """Solve to 1e-6 relative residual on the icosphere level-6 mesh: plain CG, CG with the
    reference preconditioner, flexible CG with the multilevel operator before and after
    training (train_learned_small: unrolled-CG energy loss on GPU, training time reported
    separately), and flexible CG with the hybrid (reference preconditioner plus the trained
    network's output; its H1 factorization is already in place). The reference preconditioner's H1 factorization (host Cholesky and upload,
    cached until the geometry changes) is timed apart as setup_ms; its ms is the Solve with
    the factor in place."""
    from repulsor_b200 import meshes

    net, prior, training = train_learned_small(rpb, tpm)
    B = meshes.random_rhs(V.shape[0], seed=1003)
    res = {"workload": "icosphere level 6 (40,962 vertices), RHS N(0,1) projected off translations, tol 1e-6 "
                       "(true residual of the plain metric operator)",
           "training": training}
    for name, pc, max_iter in (("plain_cg", rpb.PRECOND_NONE, 20000),
                               ("multilevel_prior_fcg", rpb.PRECOND_LEARNED, 20000),
                               ("learned_fcg", rpb.PRECOND_LEARNED, 20000),
                               ("reference_precond_cg", rpb.PRECOND_REFERENCE, 2000),
                               ("hybrid_fcg", rpb.PRECOND_HYBRID, 2000)):
        if name == "multilevel_prior_fcg":
            prior.attach(M)
        elif name in ("learned_fcg", "hybrid_fcg"):
            net.attach(M)
        setup_ms = None
        if pc == rpb.PRECOND_REFERENCE:
            # the H1 factorization (host Cholesky + upload), cached until the geometry changes
            t = time.perf_counter()
            tpm.MultiplyPreconditioner(M, 1.0, B)
            setup_ms = 1e3 * (time.perf_counter() - t)
        t = time.perf_counter()
        tpm.Solve(M, 1.0, B, max_iter=max_iter, tolerance=1e-6, precond=pc, strict=False)
        ms = 1e3 * (time.perf_counter() - t)
        rr = [float(x) for x in tpm.Solver_RelativeResiduals()]
        info = tpm.SolveInfo(M)
        res[name] = {"ms": ms, "iterations": tpm.Solver_IterationCount(), "rel_residual": rr,
                     "converged": bool(max(rr) <= 1e-6), "ms_per_iteration": ms / max(1, info["iterations"]),
                     "fallback_iteration": info["fallback_iteration"]}
        if pc == rpb.PRECOND_REFERENCE:
            res[name].update(setup_ms=setup_ms, ms_with_setup=setup_ms + ms, h1_factor_seconds=info["factor_seconds"],
                             h1_factor_nnz=info["factor_nnz"], supernode_levels=info["supernode_levels"])
    return res


def run_flow(args):
    """Full flow step at scale: two linked tori (R=1, r=0.3, 480 x 640 grids, 1,228,800
    triangles) with an icosphere level-5 obstacle of radius 0.3 at (0, 0, 2): energy +
    differential (TangentPointEnergy0 + TangentPointObstacleEnergy), the metric Solve of the
    differential to 1e-6 by flexible CG with the hybrid preconditioner (the reference
    preconditioner plus the learned network's output; network trained on seeded icospheres,
    time reported separately) with the reference preconditioner alone as fallback, and the
    collision-free step size along the solution (MaximumSafeStepSize). One step; times are
    wall clock around each public call. With the learned operator alone the flexible CG
    stalls near iteration 860 and falls back; with the reference preconditioner alone the
    solve takes 67,140 iterations."""
    import numpy as np
    import torch

    import repulsor_b200 as rpb
    from repulsor_b200 import meshes

    torch.cuda.set_device(0)
    out = {"metric": "full flow step (energy+grad, hybrid learned FCG solve to 1e-6)", "unit": "s",
           "workload": "two linked tori 480x640 (614,400 vertices, 1,228,800 triangles) + icosphere L5 obstacle "
                       "r=0.3 at (0,0,2), q=6 p=12 theta=0.5"}
    t = time.perf_counter()
    V, S = meshes.linked_tori()
    M = rpb.SimplicialMesh(V, S)
    Vo, So = meshes.icosphere(level=5, radius=0.3, centre=(0.0, 0.0, 2.0))
    M.LoadObstacle(rpb.SimplicialMesh(Vo, So))
    out["setup_s"] = time.perf_counter() - t
    st = M.stats()
    out["mesh"] = {k: st[k] for k in ("cluster_count", "near_nnz", "far_nnz", "tree_build_seconds", "device_bytes")}
    out["obstacle"] = M.obstacle_stats()
    tpe, tpo = rpb.TangentPointEnergy0(Q, P), rpb.TangentPointObstacleEnergy(Q, P)
    tpm = rpb.TangentPointMetric0(Q, P)
    D = np.zeros_like(V)
    for _ in range(2):
        torch.cuda.synchronize()
        t = time.perf_counter()
        E = tpe.Differential(M, 1.0, 0.0, D)
        E += tpo.Differential(M, 1.0, 1.0, D)
        out["energy_grad_s"] = time.perf_counter() - t
    out["energy"] = E
    net, _, training = train_learned_small(rpb, tpm)
    out["training"] = training
    net.attach(M)
    B = D - D.mean(0)
    t = time.perf_counter()
    X = tpm.Solve(M, 1.0, B, max_iter=args.flow_max_iter, tolerance=1e-6, precond=rpb.PRECOND_HYBRID, strict=False)
    out["solve_s"] = time.perf_counter() - t
    # the flow's next call: the collision-free step along the descent direction -X, scaled so
    # that the fastest vertex moves by at most the mean edge length at t = 1
    edge = float(np.linalg.norm(V[S[:, 1]] - V[S[:, 0]], axis=1).mean())
    vel = -X * (edge / max(float(np.abs(X).max()), 1e-300))
    t = time.perf_counter()
    out["step_size"] = M.MaximumSafeStepSize(vel, 1.0)
    out["step_size_s"] = time.perf_counter() - t
    info = tpm.SolveInfo(M)
    out["solve"] = {"iterations": info["iterations"], "fallback_iteration": info["fallback_iteration"],
                    "rel_residual": [float(x) for x in tpm.Solver_RelativeResiduals()],
                    "h1_factor_s": info["factor_seconds"], "h1_factor_nnz": info["factor_nnz"],
                    "precond": "hybrid: reference H1^-1 L H1^-1 + w x learned multilevel"}
    out["value"] = out["energy_grad_s"] + out["solve_s"] + out["step_size_s"]
    print(json.dumps(out))
    return 0


def run_sharded(args):
    """One evaluation (SemiStaticUpdate + Differential) of the two linked tori (1,228,800
    triangles) per step, its row tiles split over the ranks (repulsor_b200/sharding.py):
    each GPU evaluates its shard, one NCCL all-reduce sums the (N + N_C) x 10 derivative
    buffer, every GPU collects. Total work is fixed as N grows (strong scaling); the step
    time is the slowest rank's CUDA-event time."""
    import datetime

    import torch

    import repulsor_b200 as rpb
    from repulsor_b200 import meshes
    from repulsor_b200.sharding import ShardedDifferential

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local_rank)
    import torch.distributed as dist
    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    os.environ.setdefault("MASTER_PORT", "29512")
    dist.init_process_group("nccl", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120),
                            device_id=torch.device("cuda", local_rank))
    try:
        V, S = meshes.linked_tori()
        M = rpb.SimplicialMesh(V, S, device=local_rank)
        tpe = rpb.TangentPointEnergy0(Q, P)
        sd = ShardedDifferential(M, tpe)
        Vd = torch.tensor(V, device="cuda")
        Yd = torch.zeros((V.shape[0], 3), dtype=torch.float64, device="cuda")
        ext = torch.cuda.ExternalStream(M.stream())

        def step():
            M.SemiStaticUpdateDevice(Vd.data_ptr())
            sd(Yd.data_ptr(), want_energy=False)

        for _ in range(args.warmup):
            step()
        torch.cuda.synchronize()
        dist.barrier()
        steps = max(1, min(args.steps, 50))
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(ext)
        for _ in range(steps):
            step()
        b.record(ext)
        torch.cuda.synchronize()
        ms = max_over_ranks(a.elapsed_time(b) / steps, dist, "cuda")
        E = sd(Yd.data_ptr())
        st = M.stats()
        if rank == 0:
            print(json.dumps({"metric": "energy+grad evals/s of one mesh, row-sharded", "value": 1e3 / ms,
                              "unit": "evals/s", "n_gpus": world, "steps": steps, "warmup": args.warmup,
                              "ms_per_step": ms, "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
                              "dtype": "f32+f64", "data": "synthetic (seeded linked tori)",
                              "config": {"workload": "two linked tori 480x640 (1,228,800 triangles), q=6 p=12 "
                                                     "theta=0.5", "parallelism": f"row shards x{world}",
                                         "near_nnz": st["near_nnz"], "far_nnz": st["far_nnz"],
                                         "allreduce_bytes": 8 * sd.buf.numel()},
                              "energy": E}))
        del sd
    finally:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
