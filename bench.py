#!/usr/bin/env python
"""Benchmark: time-to-solution of the 1M-node P1 wave-equation CG solve.

Workload (one step): SOLVE of A x = b on the 1001 x 1001-node mesh
(1,002,001 nodes, 2,000,000 triangles; A = M + dt*g*h_e*K_e, smooth depth,
b = A x_true), diagonal preconditioning, relative residual 1e-8, x0 = 0.
`value` is the mixed-precision solve (binary32 inner CG with binary64
refinement) in solves/s over all ranks, with the inputs resident in HBM;
the plain binary64 GRACJG solve, the standalone EBE matvec bandwidth and
the end-to-end (host buffers through the C ABI) time are reported beside it.

Multi-GPU: each rank solves its own replica (the path does not shard in
this build), so scaling is weak; times are the max over ranks.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np


def quiet(fn):
    """Run fn with the process's stdout (fd 1, C stdio included) discarded,
    so that the one JSON line stays the only output."""
    import ctypes
    libc = ctypes.CDLL(None)
    sys.stdout.flush()
    libc.fflush(None)
    saved = os.dup(1)
    null = os.open(os.devnull, os.O_WRONLY)
    os.dup2(null, 1)
    try:
        return fn()
    finally:
        libc.fflush(None)
        os.dup2(saved, 1)
        os.close(saved)
        os.close(null)

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "1M-node P1 CG time-to-1e-8 relres: mixed vs FP64 on 1 B200; matvec HBM GB/s"
UNIT = "solves/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--n", type=int, default=1001, help="nodes per side of the mesh")
    ap.add_argument("--eps", type=float, default=1e-8)
    ap.add_argument("--storage", default="ebe", choices=["ebe", "seg"],
                    help="matrix storage: ebe (element by element, STO=1) or seg (edge "
                         "segments, STO=3, built from the EBE matrix by ASSEX3)")
    ap.add_argument("--depth", default="smooth", choices=["smooth", "loguniform"],
                    help="smooth: h = 5 + 4 sin(2 pi x) cos(2 pi y); loguniform: h log-uniform "
                         "in [0.5, 500] m, 3 passes of neighbour averaging")
    ap.add_argument("--inner-tol", type=float, default=None,
                    help="refinement threshold of the mixed solve: the binary32 residual is "
                         "refreshed from a binary64 one after dropping by this factor "
                         "(default 0.1 for wave1m, 1e-4 for batch256)")
    ap.add_argument("--cpu-seconds", type=float, default=12.0,
                    help="target CPU time of the bounded CPU-baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-large-matvec", action="store_true",
                    help="skip the MATVEC measurements on the 2001x2001-node mesh")
    ap.add_argument("--no-extras", action="store_true",
                    help="wave1m: skip the 2001x2001 log-uniform solves (config2) and the "
                         "256-mesh batch (batch256) reported beside the headline")
    ap.add_argument("--batch-shape", default=None,
                    help="batch256: nodes per thread, threads per block and optionally "
                         "blocks per SM as NPT,TPB[,BPS] (default: the autotuner's choice)")
    ap.add_argument("--max-inner", type=int, default=200,
                    help="mixedcap: inner iterations of each bounded mixed solve")
    ap.add_argument("--batch-max-inner", type=int, default=1000000,
                    help="batch256: stop every instance after this many inner iterations "
                         "(the launch then covers only the first cycles: time against cycles)")
    ap.add_argument("--nitmax", type=int, default=1000000,
                    help="fp64: NITMAX of the binary64 solves (a small value bounds the "
                         "launch for profiling)")
    ap.add_argument("--workload", default="wave1m",
                    choices=["wave1m", "batch256", "matvec", "mixedcap", "fp64"],
                    help="wave1m: the 1M-node solve (default); batch256: 256 independent "
                         "meshes of 2,000-200,000 nodes in one persistent launch per rank; "
                         "matvec: the binary64 and binary32 MATVEC 'X=AY' alone on the "
                         "--n x --n mesh; mixedcap: mixed solves capped at --max-inner "
                         "inner iterations on the --n x --n mesh (a bounded profiling target); "
                         "fp64: the binary64 GRACJG alone on the --n x --n mesh (--depth, "
                         "--eps, --nitmax)")
    args = ap.parse_args()
    if args.inner_tol is None:
        args.inner_tol = 1e-4 if args.workload == "batch256" else 0.1
    return args


def algorithmic_bytes(npoin, nelem, nseg=None):
    """Algorithmic bytes (each input read once, each output written once)."""
    if nseg is not None:   # segment storage: XA 8 B + GLOSEG 2x4 B per segment
        return dict(mv64=16 * nseg + 24 * npoin, mv32=12 * nseg + 12 * npoin,
                    it64=16 * nseg + 88 * npoin,
                    it32=12 * nseg + 48 * npoin, upd=16 * nseg + 48 * npoin)
    return dict(
        # EBE matvec 'X=AY' with a full diagonal, binary64: XM 3x8 + IKLE 3x4
        # per element; DM, Y in, X out per node
        mv64=36 * nelem + 24 * npoin,
        # the same in binary32: XM 3x4 + IKLE 3x4 per element; DM, Y, X
        mv32=24 * nelem + 12 * npoin,
        # one binary64 GRACJG iteration on the scaled system: matvec without
        # diagonal (36/elem + 16/node) + 9 node-vector accesses (72/node)
        it64=36 * nelem + 88 * npoin,
        # one binary32 inner iteration: matvec 12+12 per element, row sum +
        # p in + q out (12/node) + 9 binary32 node-vector accesses (36/node)
        it32=24 * nelem + 48 * npoin,
        # reliable update: binary64 matvec on x + b, r32, x and z updates
        upd=36 * nelem + 48 * npoin,
    )


class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.f = None

    def __enter__(self):
        try:
            self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if self.proc is None or self.f is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.f.flush()
        rows = []
        with open(self.f.name) as fh:
            for line in fh:
                p = [c.strip() for c in line.split(",")]
                if len(p) >= 9:
                    rows.append(p)
        os.unlink(self.f.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(rows)}


def depth_field(depth, x, y, ik):
    from opentelemac_b200 import meshgen as mg
    return mg.depth_loguniform(ik) if depth == "loguniform" else mg.depth_smooth(x, y, ik)


def build_problem(n, device, depth="smooth", storage="ebe"):
    """Mesh, operator (assembled on the device), manufactured solution."""
    import torch
    from opentelemac_b200 import bief, meshgen as mg
    x, y, ik = mg.square_mesh(n)
    coef = mg.wave_coef(depth_field(depth, x, y, ik))
    npoin = x.size
    mesh = bief.Mesh(ik, npoin, device=device)
    A = bief.Matrix(mesh)
    t = lambda a: torch.tensor(a, device=f"cuda:{device}", dtype=torch.float64)
    A.assemble_wave(t(x), t(y), t(coef))
    nseg = None
    if storage == "seg":
        g1, g2, _, _ = mg.segments(ik, npoin)
        mesh.set_segments(g1, g2)
        A.to_segments()
        nseg = int(g1.size)
    xt = t(mg.random_solution(npoin))
    b = torch.zeros_like(xt)
    bief.matvec("X=AY    ", b, A, xt)
    return dict(x=x, y=y, ik=ik, coef=coef, mesh=mesh, A=A, xt=xt, b=b, npoin=npoin,
                nelem=ik.shape[0], nseg=nseg)


def cpu_baseline(n, eps, nit_full, seconds, depth="smooth"):
    """The oracle's reference-order binary64 SOLVE on one host core, timed on
    a bounded number of CG iterations and extrapolated to a full solve."""
    import oracle
    from opentelemac_b200 import meshgen as mg
    oracle.build()
    x, y, ik = mg.square_mesh(n)
    coef = mg.wave_coef(depth_field(depth, x, y, ik))
    dm, xm = oracle.wave_matrix(x, y, ik, coef)
    b = oracle.matvec("X=AY    ", ik, dm, "Q", xm, "S", mg.random_solution(x.size))
    args = (ik, dm, "Q", xm, "S", b)
    k1 = 5
    t0 = time.perf_counter()
    oracle.solve(*args, nitmax=k1, eps=1e-300)
    t1 = time.perf_counter() - t0
    k2 = 25
    t0 = time.perf_counter()
    oracle.solve(*args, nitmax=k2, eps=1e-300)
    t2 = time.perf_counter() - t0
    per_it = max((t2 - t1) / (k2 - k1), 1e-9)
    k3 = int(min(max(k2 + 10, seconds / per_it), nit_full))
    t0 = time.perf_counter()
    oracle.solve(*args, nitmax=k3, eps=1e-300)
    t3 = time.perf_counter() - t0
    per_it = (t3 - t1) / (k3 - k1)
    setup = max(t1 - k1 * per_it, 0.0)
    full = setup + per_it * nit_full
    return {"value": 1.0 / full, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": (f"binary64 reference-order C restatement of SOLVE/GRACJG, 1 thread, "
                       f"{k3} of {nit_full} CG iterations timed ({t3:.1f} s) on the "
                       f"{x.size}-node mesh, extrapolated: {per_it * 1e3:.2f} ms/iteration, "
                       f"{full:.1f} s per solve"),
            "seconds_per_solve": full, "ms_per_iteration": per_it * 1e3}


def dist_init():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    return ws, rank, local


def max_over_ranks(v, ws):
    from opentelemac_b200 import replicas
    return replicas.max_over_ranks(v) if ws > 1 else v


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def solve_config(args, npoin, nelem, nseg, ws):
    """`config` of the wave-equation SOLVE line, the same dict in both arms."""
    return {"workload": f"wave-equation SOLVE (CG, diagonal precon, relres {args.eps:g}) on "
                        f"the {args.n}x{args.n}-node P1 mesh",
            "npoin": npoin, "nelem": nelem, "nseg": nseg,
            "storage": "segments (STO=3)" if args.storage == "seg" else "EBE (STO=1)",
            "depth": args.depth, "inner_tol": args.inner_tol, "parallelism": f"replicas x{ws}",
            "l2": "1 GiB written then 256 MB read before every timed step"}


def run_reference(args, ws, rank):
    """--impl reference: the reference algorithm's CPU implementation on the
    host cores (the Fortran cannot be compiled on these machines, so the
    oracle's port of SOLVE/GRACJG, run on every host thread with OpenMP as
    the reference would run with one MPI rank per core), rank 0 only.  Every
    step, warm-up included, is one whole solve of the workload from x = 0 to
    the relative residual, timed with the host clock."""
    if rank != 0:
        return
    import oracle
    from opentelemac_b200 import meshgen as mg
    oracle.build()
    nthreads = os.cpu_count() or 1
    x, y, ik = mg.square_mesh(args.n)
    coef = mg.wave_coef(depth_field(args.depth, x, y, ik))
    dm, xm = oracle.wave_matrix(x, y, ik, coef)
    b = oracle.matvec("X=AY    ", ik, dm, "Q", xm, "S", mg.random_solution(x.size))
    times, full = [], None
    for s in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        full = oracle.solve_omp(ik, dm, xm, b, eps=args.eps, nthreads=nthreads)
        dt = time.perf_counter() - t0
        if s >= args.warmup:
            times.append(dt)
    per_solve = sum(times) / len(times)
    val = 1.0 / per_solve
    line = {"impl": "reference", "metric": METRIC, "value": val, "unit": UNIT,
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": per_solve * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": solve_config(args, int(x.size), int(ik.shape[0]),
                                   int(x.size + ik.shape[0] - 1) if args.storage == "seg"
                                   else None, ws),
            "solver": "binary64 GRACJG, every step a whole solve from x = 0",
            "iterations": full["nit"], "relres": full["relres"],
            "cpu_baseline": {"value": val, "unit": UNIT, "cores": nthreads, "kind": "port",
                             "sample": f"binary64 port of SOLVE/GRACJG on {nthreads} threads; "
                                       f"every step one whole solve ({full['nit']} CG "
                                       f"iterations, {per_solve:.2f} s)"},
            "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def hbm_peak():
    """Measured HBM copy bandwidth (GB/s) of MEASURED_PEAKS.json and where
    it came from."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def batch_measure(ws, rank, local, steps, warmup, inner_tol, eps, shape=None, max_inner=1000000,
                  storage="ebe"):
    """The 256-mesh workload (node counts log-uniform in [2,000, 200,000],
    per-mesh seeds, random right-hand sides), mixed precision to relres
    `eps`, all of a rank's meshes in one persistent launch per step; with N
    ranks the meshes are sharded (size-balanced) across ranks: fixed total
    work, no data-path collective.  Returns the measurements (rank 0's
    instances for the iteration statistics and the roofline)."""
    import torch
    from opentelemac_b200 import meshgen as mg, replicas
    from opentelemac_b200.batch import BatchSolver
    torch.cuda.set_device(local)
    sizes = mg.batch_sizes()
    mine = replicas.shard_instances([n * n for n in sizes], ws, rank)
    meshes, xs, ys, coefs, bvs = [], [], [], [], []
    for k in mine:
        x, y, ik, coef, bv = mg.batch_instance(k, sizes[k])
        meshes.append((x.size, ik))
        xs.append(x)
        ys.append(y)
        coefs.append(coef)
        bvs.append(bv)
    bs = BatchSolver(meshes, device=local)
    bs.assemble_wave(xs, ys, coefs)
    if storage == "seg":   # every instance's own STOSEG numbering, ASSEX3 on the device
        bs.set_segments([mg.segments(ik, npo)[:2] for npo, ik in meshes]).to_segments()
    b = bs.gather(bvs)
    x = torch.zeros_like(b)
    if shape:
        npt, tpb = shape[:2]
        if len(shape) > 2:
            bs.mesh.set_blocks_per_sm(shape[2])
    else:
        npt, tpb, _ = bs.autotune(b, inner_tol=inner_tol, outer_tol=eps)
    flush = torch.empty(1024 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{local}")
    clean = torch.ones(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{local}")
    times, kern = [], []
    for s in range(warmup + steps):
        flush.fill_(float(s))   # 1 GiB written, then 256 MB read: L2 flushed, lines clean
        clean.sum()
        x.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        r = bs.solve_mixed(x, b, inner_tol=inner_tol, outer_tol=eps, nodes_per_thread=npt,
                           threads_per_block=tpb, max_inner=max_inner)
        e1.record()
        e1.synchronize()
        if s >= warmup:
            times.append(e0.elapsed_time(e1))
            kern.append(r["kernel_ms"])
    step_ms = max_over_ranks(sum(times) / len(times), ws)
    ok = int(replicas.sum_over_ranks(int((r["status"] == 0).sum()))) if ws > 1 else int(
        (r["status"] == 0).sum())
    inner = r["inner"]
    # algorithmic bytes of this rank's launch: every instance's inner
    # iterations and binary64 refinements (the initial residual included)
    alg = 0
    for (npo, ik), ni, no in zip(meshes, r["inner"], r["outer"]):
        by = algorithmic_bytes(npo, ik.shape[0])
        alg += int(ni) * by["it32"] + (int(no) + 1) * by["upd"]
    kern_ms = sum(kern) / len(kern)
    hbm, src = hbm_peak()
    gbs = alg / (kern_ms * 1e-3) / 1e9
    out = {"value": 256 * 1000.0 / step_ms, "unit": "solves/s", "ms_per_step": step_ms,
           "kernel_ms": kern_ms, "converged": ok, "inner_tol": inner_tol,
           "max_inner": max_inner,
           "nodes_this_rank": int(bs.total_nodes), "nodes_per_thread": int(npt),
           "threads_per_block": int(tpb),
           "blocks_per_sm": int(bs.mesh.launch_info()[0]
                                // torch.cuda.get_device_properties(local).multi_processor_count),
           "autotune_ms_per_iteration": {f"npt{k[0]}_t{k[1]}_b{k[2]}": round(v, 4)
                                         for k, v in getattr(bs, "tune_table", {}).items()},
           "iterations_rank0": {"p50": float(np.percentile(inner, 50)),
                                "p99": float(np.percentile(inner, 99)),
                                "max": int(inner.max())},
           "roofline": {"bound": "hbm", "kernel": "k_batch", "achieved": gbs, "peak": hbm,
                        "unit": "GB/s", "frac": gbs / hbm,
                        "peak_source": f"{src} (MEASURED_PEAKS.json hbm_gbs)",
                        "bytes_per_launch": alg,
                        "note": "rank 0's instances; working set (13.0M nodes) far above L2"}}
    bs.close()
    del flush, clean, x, b
    return out


def run_batch(args, ws, rank, local):
    """--workload batch256: the batched line on its own."""
    shape = tuple(int(v) for v in args.batch_shape.split(",")) if args.batch_shape else None
    m = batch_measure(ws, rank, local, args.steps, args.warmup, args.inner_tol, args.eps, shape,
                      args.batch_max_inner, args.storage)
    if rank == 0:
        line = {"metric": "batched P1 CG solves/s (256 meshes, mixed, relres 1e-8)",
                "value": m["value"], "unit": "solves/s", "n_gpus": ws,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": m["ms_per_step"],
                "higher_is_better": True, "scaling": "strong" if ws > 1 else "weak",
                "vs_baseline": None, "dtype": "f32 inner / f64 refinement",
                "data": "synthetic",
                "config": {"workload": "256 meshes, 2,000-200,000 nodes (log-uniform), one "
                                       "persistent launch per rank",
                           "nodes_this_rank": m["nodes_this_rank"],
                           "nodes_per_thread": m["nodes_per_thread"],
                           "threads_per_block": m["threads_per_block"],
                           "blocks_per_sm": m["blocks_per_sm"],
                           "autotune_ms_per_iteration": m["autotune_ms_per_iteration"],
                           "storage": "segments (STO=3)" if args.storage == "seg"
                                      else "EBE (STO=1)",
                           "parallelism": f"shards x{ws}"},
                "converged": m["converged"], "kernel_ms": m["kernel_ms"],
                "max_inner": m["max_inner"],
                "roofline": m["roofline"], "iterations_rank0": m["iterations_rank0"]}
        print(json.dumps(line), flush=True)


def _grid_info(mesh, device):
    """Blocks and threads of the persistent solvers on this mesh (the
    dot-product tree) and the resident blocks per SM they were built for."""
    import torch
    G, T = mesh.launch_info()
    nsm = torch.cuda.get_device_properties(device).multi_processor_count
    return {"blocks": G, "threads": T, "blocks_per_sm": max(1, G // nsm)}


def config2_measure(P2, ws, flush_l2, hbm, steps=2, warmup=1):
    """The 2001 x 2001-node mesh with the log-uniform depth (4,004,001
    nodes, 8,000,000 triangles), relres 1e-10: binary64 GRACJG, the mixed
    solve with refinement threshold 1e-4 (as the workload specifies) and 0.1,
    each timed over `steps` solves after `warmup`, L2 flushed before each;
    a binary64 solve to relres 1e-13 is the accuracy reference both are
    measured against."""
    import torch
    from opentelemac_b200 import bief
    A, b, mesh = P2["A"], P2["b"], P2["mesh"]
    by = algorithmic_bytes(P2["npoin"], P2["nelem"], P2["nseg"])
    eps = 1e-10
    x = torch.zeros_like(b)

    def timed(fn):
        ms, kern, res = [], [], None
        for s in range(warmup + steps):
            flush_l2(s)
            x.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            res = fn()
            e1.record()
            e1.synchronize()
            if s >= warmup:
                ms.append(e0.elapsed_time(e1))
                kern.append(mesh.last_timing()[0])
        return (max_over_ranks(sum(ms) / len(ms), ws), sum(kern) / len(kern), res)

    cfg = bief.SlvCfg(slv=1, nitmax=1000000, precon=2, krylov=0, eps=eps, zero=0.0)
    f64_ms, f64_kern, f64_res = timed(lambda: bief.solve(x, A, b, cfg))
    x64 = x.clone()
    x.zero_()
    tight = bief.SlvCfg(slv=1, nitmax=1000000, precon=2, krylov=0, eps=1e-13, zero=0.0)
    _, nit_t, rel_t = bief.solve(x, A, b, tight)
    x13 = x.clone()
    nrm = lambda v: float(torch.linalg.norm(v))
    f64_bytes = f64_res[1] * by["it64"]
    out = {"workload": "2001x2001-node P1 mesh, log-uniform depth in [0.5, 500] m (3 "
                       "smoothing passes), relres 1e-10",
           "npoin": P2["npoin"], "nelem": P2["nelem"],
           "persistent_grid": _grid_info(mesh, b.device),
           "fp64": {"ms": f64_ms, "kernel_ms": f64_kern, "iterations": f64_res[1],
                    "relres": f64_res[2], "kernel": "k_cg64",
                    "gbs": f64_bytes / (f64_kern * 1e-3) / 1e9,
                    "frac": f64_bytes / (f64_kern * 1e-3) / 1e9 / hbm,
                    "bytes_per_launch": f64_bytes},
           "tight_fp64": {"relres": rel_t, "iterations": nit_t,
                          "fp64_vs_tight": nrm(x64 - x13) / nrm(x13)}}
    for key, itol in (("mixed_itol_1e-4", 1e-4), ("mixed_itol_0.1", 0.1)):
        ms, kern, res = timed(lambda: bief.solve_mixed(x, A, b, precon=2, inner_tol=itol,
                                                       outer_tol=eps))
        st, outer, inner, relres = res
        mb = inner * by["it32"] + (outer + 1) * by["upd"]
        out[key] = {"ms": ms, "kernel_ms": kern, "inner": inner, "refinements": outer,
                    "relres": relres, "speedup_vs_fp64": f64_ms / ms,
                    "vs_fp64": nrm(x - x64) / nrm(x64), "vs_tight_fp64": nrm(x - x13) / nrm(x13),
                    "kernel": "k_mixed", "gbs": mb / (kern * 1e-3) / 1e9,
                    "frac": mb / (kern * 1e-3) / 1e9 / hbm, "bytes_per_launch": mb}
    del x, x64, x13
    return out


def config3_measure(ws, steps=3, warmup=1):
    """The differentiation workload on the 501 x 501-node mesh (251,001
    nodes, 500,000 triangles): per-element depth h = the smooth field +
    N(0, 0.1^2), L = 0.5 ||x(h) - x_obs||^2 with x_obs solved from the
    unperturbed field, solves to relres 1e-13.  Timed with CUDA events:
    one forward + backward (assembly, forward CG, adjoint CG, per-element
    gradient), and the 50-step unrolled loop x_{n+1} = A(h)^-1 M x_n with a
    checkpoint every 10 steps, forward and backward (150 solves)."""
    import torch
    from opentelemac_b200 import autograd as ag, bief, meshgen as mg
    x, y, ik = mg.square_mesh(501)
    prob = ag.WaveProblem(x, y, ik, eps=1e-13)
    h0 = torch.tensor(mg.depth_smooth(x, y, ik), device="cuda")
    h = h0 + torch.tensor(np.random.default_rng(3).normal(0.0, 0.1, ik.shape[0]),
                          device="cuda")
    xt = torch.tensor(mg.random_solution(x.size), device="cuda")
    b = torch.zeros_like(xt)
    bief.matvec("X=AY    ", b, prob.assemble(mg.DT * mg.GRAV * h0), xt)
    x_obs = prob.solve(mg.DT * mg.GRAV * h0, b)

    def ev_time(fn):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        out = fn()
        e1.record()
        e1.synchronize()
        return e0.elapsed_time(e1), out

    def fwd_bwd():
        hv = h.clone().requires_grad_(True)
        xs = ag.wave_solve(mg.DT * mg.GRAV * hv, b, prob)
        L = 0.5 * ((xs - x_obs) ** 2).sum()
        L.backward()
        return hv.grad

    ts = []
    for s in range(warmup + steps):
        t, g = ev_time(fwd_bwd)
        if s >= warmup:
            ts.append(t)
    fb_ms = max_over_ranks(sum(ts) / len(ts), ws)

    def loop():
        hv = h.clone().requires_grad_(True)
        xs = ag.unrolled_loop(mg.DT * mg.GRAV * hv, xt, prob, nsteps=50, checkpoint_every=10)
        (0.5 * (xs * xs).sum()).backward()
        return hv.grad

    n0 = prob.solves
    loop_ms, _ = ev_time(loop)
    loop_solves = prob.solves - n0
    loop_ms = max_over_ranks(loop_ms, ws)
    prob.close()
    return {"workload": "501x501-node P1 mesh, per-element depth, L = 0.5 ||x(h) - x_obs||^2, "
                        "relres 1e-13",
            "npoin": int(x.size), "nelem": int(ik.shape[0]),
            "forward_backward_ms": fb_ms,
            "grad_norm": float(torch.linalg.norm(g)),
            "unrolled_loop": {"steps": 50, "checkpoint_every": 10, "ms": loop_ms,
                              "solves": loop_solves,
                              "ms_per_solve": loop_ms / max(loop_solves, 1)}}


def run_matvec(args, ws, rank, local):
    """MATVEC 'X=AY' alone: binary64 EBE (k_matvec / k_mvseg) and binary32
    (k_matvec32) on the --n x --n mesh, --steps timed launches each after
    --warmup, L2 flushed before every launch, library events around each
    launch.  One line: the binary64 product's GB/s (algorithmic bytes)."""
    import torch
    from opentelemac_b200 import bief
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    P = build_problem(args.n, local, "smooth", args.storage)
    by = algorithmic_bytes(P["npoin"], P["nelem"], P["nseg"])
    flush = torch.empty(1024 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    clean = torch.ones(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    y = P["xt"]
    out = torch.zeros_like(y)
    y32 = y.float()
    out32 = torch.empty_like(y32)
    bief.matvec32(out32, P["A"], y32)

    def lib_times(fn):
        ts = []
        for s in range(args.warmup + args.steps):
            flush.fill_(float(s))
            clean.sum()
            fn()
            torch.cuda.synchronize()
            if s >= args.warmup:
                ts.append(P["mesh"].last_timing()[1])
        return ts

    launches0 = P["mesh"].kernel_launches()
    barrier(ws)
    t64 = lib_times(lambda: bief.matvec("X=AY    ", out, P["A"], y))
    t32 = lib_times(lambda: bief.matvec32(out32, P["A"], y32))
    launches = P["mesh"].kernel_launches() - launches0
    m64 = max_over_ranks(statistics.median(t64), ws)
    m32 = max_over_ranks(statistics.median(t32), ws)
    hbm = 6650.0
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            hbm = float(json.load(fh).get("hbm_gbs", hbm))
    except OSError:
        pass
    g64 = ws * by["mv64"] / (m64 * 1e-3) / 1e9
    g32 = ws * by["mv32"] / (m32 * 1e-3) / 1e9
    if rank == 0:
        kern = "k_mvseg" if args.storage == "seg" else "k_matvec16"
        print(json.dumps({
            "metric": "EBE MATVEC 'X=AY' HBM GB/s (algorithmic bytes)", "value": g64,
            "unit": "GB/s", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": m64, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"MATVEC on the {args.n}x{args.n}-node P1 mesh",
                       "npoin": P["npoin"], "nelem": P["nelem"],
                       "storage": "segments (STO=3)" if args.storage == "seg" else "EBE (STO=1)",
                       "l2": "1 GiB written then 256 MB read before every timed launch"},
            "roofline": {"bound": "hbm", "kernel": kern, "achieved": g64 / ws, "peak": hbm,
                         "unit": "GB/s", "frac": g64 / ws / hbm, "bytes": by["mv64"]},
            "matvec32": {"kernel": "k_matvec32", "ms": m32, "gbs": g32, "frac": g32 / ws / hbm,
                         "bytes": by["mv32"]},
            "gpu_launches": launches}), flush=True)
    P["mesh"].close()


def run_mixedcap(args, ws, rank, local):
    """Mixed solves stopped after --max-inner inner iterations on the --n x
    --n mesh (--depth field), --warmup + --steps solves from x = 0: a bounded
    launch of k_mixed for profiling.  One line: ms per inner iteration."""
    import torch
    from opentelemac_b200 import bief
    torch.cuda.set_device(local)
    P = build_problem(args.n, local, args.depth, args.storage)
    x = torch.zeros_like(P["b"])
    ts, its = [], 0
    for s in range(args.warmup + args.steps):
        x.zero_()
        st, outer, its, rel = bief.solve_mixed(x, P["A"], P["b"], precon=2,
                                               inner_tol=args.inner_tol, outer_tol=args.eps,
                                               max_inner=args.max_inner)
        if s >= args.warmup:
            ts.append(P["mesh"].last_timing()[0])
    m = max_over_ranks(statistics.median(ts), ws)
    if rank == 0:
        print(json.dumps({
            "metric": "mixed inner iteration time (bounded solve)", "value": m / max(its, 1),
            "unit": "ms/iteration", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": m, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 inner / f64 refinement", "data": "synthetic",
            "config": {"workload": f"mixed solve capped at {args.max_inner} inner iterations on "
                                   f"the {args.n}x{args.n}-node P1 mesh", "depth": args.depth,
                       "inner_tol": args.inner_tol, "storage": args.storage},
            "inner_iterations": its, "status": st}), flush=True)
    P["mesh"].close()


def run_fp64_solve(args, ws, rank, local):
    """Binary64 GRACJG alone on the --n x --n mesh (--depth, --storage,
    --eps, --nitmax): --warmup + --steps solves from x = 0, L2 flushed before
    each, the library's events around the solver launch.  One line: ms per
    solve and the k_cg64 (or segment) kernel's algorithmic GB/s."""
    import torch
    from opentelemac_b200 import bief
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    P = build_problem(args.n, local, args.depth, args.storage)
    by = algorithmic_bytes(P["npoin"], P["nelem"], P["nseg"])
    flush = torch.empty(1024 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    clean = torch.ones(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    x = torch.zeros_like(P["b"])
    cfg = bief.SlvCfg(slv=1, nitmax=args.nitmax, precon=2, krylov=0, eps=args.eps, zero=0.0)
    ts, nit, rel = [], 0, 0.0
    for s in range(args.warmup + args.steps):
        flush.fill_(float(s))
        clean.sum()
        x.zero_()
        st, nit, rel = quiet(lambda: bief.solve(x, P["A"], P["b"], cfg))
        if s >= args.warmup:
            ts.append(P["mesh"].last_timing()[0])
    m = max_over_ranks(statistics.median(ts), ws)
    hbm, src = hbm_peak()
    gbs = nit * by["it64"] / (m * 1e-3) / 1e9
    if rank == 0:
        print(json.dumps({
            "metric": "binary64 GRACJG time-to-solution", "value": m, "unit": "ms",
            "n_gpus": ws, "steps": args.steps, "warmup": args.warmup, "ms_per_step": m,
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": f"binary64 GRACJG (relres {args.eps:g}, NITMAX "
                                   f"{args.nitmax}) on the {args.n}x{args.n}-node P1 mesh",
                       "depth": args.depth, "storage": args.storage},
            "iterations": nit, "relres": rel, "ms_per_iteration": m / max(nit, 1),
            "roofline": {"bound": "hbm", "kernel": "k_cg64", "achieved": gbs, "peak": hbm,
                         "unit": "GB/s", "frac": gbs / hbm,
                         "peak_source": f"{src} (MEASURED_PEAKS.json hbm_gbs)",
                         "bytes_per_iteration": by["it64"]}}), flush=True)
    P["mesh"].close()


def main():
    args = parse()
    ws, rank, local = dist_init()
    if args.impl == "b200" and args.workload == "fp64":
        run_fp64_solve(args, ws, rank, local)
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    if args.impl == "b200" and args.workload == "mixedcap":
        run_mixedcap(args, ws, rank, local)
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    if args.impl == "b200" and args.workload == "matvec":
        run_matvec(args, ws, rank, local)
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    if args.impl == "b200" and args.workload == "batch256":
        run_batch(args, ws, rank, local)
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    if args.impl == "reference":
        run_reference(args, ws, rank)
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    import torch
    from opentelemac_b200 import bief
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    P = build_problem(args.n, local, args.depth, args.storage)
    A, b, mesh = P["A"], P["b"], P["mesh"]
    npoin, nelem = P["npoin"], P["nelem"]
    by = algorithmic_bytes(npoin, nelem, P["nseg"])
    # Before every timed kernel 1 GiB is written (flushes the 126 MB L2 and
    # keeps the GPU busy while the host enqueues the timed launch), then 256 MB
    # are read, so that the L2 holds clean lines and the timed kernel does not
    # pay for writing back the flush's dirty ones.
    flush = torch.empty(1024 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    clean = torch.ones(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def flush_l2(s):
        flush.fill_(float(s))
        clean.sum()

    x = torch.zeros_like(b)
    cfg = bief.SlvCfg(slv=1, nitmax=1000000, precon=2, krylov=0, eps=args.eps, zero=0.0)

    def run_mixed():
        x.zero_()
        return bief.solve_mixed(x, A, b, precon=2, inner_tol=args.inner_tol, outer_tol=args.eps)

    def run_fp64():
        x.zero_()
        return bief.solve(x, A, b, cfg)

    def timed(fn, steps, warmup):
        """per-step device time (ms) with an L2 flush before each step, and
        the library's kernel time of the solver launch."""
        out, kern, res = [], [], None
        for s in range(warmup + steps):
            flush_l2(s)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            res = fn()
            e1.record()
            e1.synchronize()
            if s >= warmup:
                out.append(e0.elapsed_time(e1))
                kern.append(mesh.last_timing()[0])
        return out, kern, res

    # binary64 GRACJG (reported beside the headline)
    barrier(ws)
    f64_ms, f64_kern, f64_res = timed(run_fp64, max(2, args.steps // 2), args.warmup)
    f64_x_err = float(torch.linalg.norm(x - P["xt"]) / torch.linalg.norm(P["xt"]))
    x_f64 = x.clone()
    nit64 = f64_res[1]

    # how far the binary64 iterates move per CG step where the solve stops:
    # the iterate one step before the returned one (NITMAX = nit - 2, since
    # the converged exit skips the last X update) and one step after it
    # (NITMAX = nit).  A second solution at the same relres cannot be
    # expected closer to the binary64 one than this.
    def fp64_at(nitmax):
        x.zero_()
        c = bief.SlvCfg(slv=1, nitmax=nitmax, precon=2, krylov=0, eps=1e-30, zero=0.0)
        quiet(lambda: bief.solve(x, A, b, c))   # NITMAX reached: the message is not ours
        return float(torch.linalg.norm(x - x_f64) / torch.linalg.norm(x_f64))

    f64_step = {"before_stop": fp64_at(nit64 - 2), "after_stop": fp64_at(nit64)}

    # a binary64 solve converged far past the stopping test (relres 1e-13):
    # the accuracy reference the binary64 and the mixed solutions are both
    # measured against
    x.zero_()
    tight_cfg = bief.SlvCfg(slv=1, nitmax=1000000, precon=2, krylov=0, eps=1e-13, zero=0.0)
    _, nit_tight, rel_tight = bief.solve(x, A, b, tight_cfg)
    x_tight = x.clone()
    f64_vs_tight = float(torch.linalg.norm(x_f64 - x_tight) / torch.linalg.norm(x_tight))

    # binary64 GRACJG with MODASS = 3 (compensated dot products)
    def run_fp64_comp():
        x.zero_()
        return bief.solve(x, A, b, cfg, modass=3)

    c64_ms, c64_kern, c64_res = timed(run_fp64_comp, 2, 1)
    c64_vs_f64 = float(torch.linalg.norm(x - x_f64) / torch.linalg.norm(x_f64))

    # standalone EBE matvec bandwidth (binary64, full diagonal)
    y = P["xt"]
    out = torch.zeros_like(y)
    mv_ms, mv_lib = [], []
    for s in range(args.warmup + 20):
        flush_l2(s)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        bief.matvec("X=AY    ", out, A, y)
        e1.record()
        e1.synchronize()
        if s >= args.warmup:
            mv_ms.append(e0.elapsed_time(e1))
            mv_lib.append(mesh.last_timing()[1])   # events around the launch itself
    mv_t = statistics.median(mv_lib)
    mv_t_call = statistics.median(mv_ms)

    # the binary32 inner operator's product on the stored matrix (its copy
    # is built by the first call, outside the timed launches)
    y32 = y.float()
    out32 = torch.empty_like(y32)
    bief.matvec32(out32, A, y32)
    mv32_lib = []
    for s in range(args.warmup + 20):
        flush_l2(s)
        bief.matvec32(out32, A, y32)
        torch.cuda.synchronize()
        if s >= args.warmup:
            mv32_lib.append(mesh.last_timing()[1])
    mv32_t = statistics.median(mv32_lib)
    mv32_err = float(torch.linalg.norm(out32.double() - out) / torch.linalg.norm(out))

    # both MATVECs again on the 2001 x 2001-node mesh (4.0M nodes, 8.0M
    # triangles: the mixed-precision configuration's size)
    mv_large = None
    PL = None
    if args.n < 2001 and not (args.no_large_matvec and args.no_extras):
        # log-uniform depth: the configuration's own operator (the values do
        # not change the product's time); its solves follow the headline
        PL = build_problem(2001, local, "loguniform", args.storage)
    if PL is not None and not args.no_large_matvec:
        byl = algorithmic_bytes(PL["npoin"], PL["nelem"], PL["nseg"])

        def lib_median(fn, mesh_l):
            ts = []
            for s in range(args.warmup + 20):
                flush_l2(s)
                fn()
                torch.cuda.synchronize()
                if s >= args.warmup:
                    ts.append(mesh_l.last_timing()[1])
            return statistics.median(ts)

        yl = PL["xt"]
        ol = torch.zeros_like(yl)
        t64 = lib_median(lambda: bief.matvec("X=AY    ", ol, PL["A"], yl), PL["mesh"])
        y32l = yl.float()
        o32l = torch.empty_like(y32l)
        bief.matvec32(o32l, PL["A"], y32l)
        t32 = lib_median(lambda: bief.matvec32(o32l, PL["A"], y32l), PL["mesh"])
        mv_large = {"npoin": PL["npoin"], "nelem": PL["nelem"]}
        for key, t_ms, nb in (("matvec64", t64, byl["mv64"]), ("matvec32", t32, byl["mv32"])):
            g = nb / (t_ms * 1e-3) / 1e9
            mv_large[key] = {"ms": t_ms, "bytes": nb, "gbs": g}
        del yl, ol, y32l, o32l

    # headline: mixed precision, timed steps, clocks sampled meanwhile
    barrier(ws)
    launches0 = mesh.kernel_launches()
    with ClockSampler(local) as clk:
        mx_ms, mx_kern, mx_res = timed(run_mixed, args.steps, args.warmup)
    launches = (mesh.kernel_launches() - launches0) * args.steps // (args.steps + args.warmup)
    st, outer, inner, relres = mx_res
    mixed_x_err = float(torch.linalg.norm(x - P["xt"]) / torch.linalg.norm(P["xt"]))
    mixed_vs_f64 = float(torch.linalg.norm(x - x_f64) / torch.linalg.norm(x_f64))
    mixed_vs_tight = float(torch.linalg.norm(x - x_tight) / torch.linalg.norm(x_tight))
    barrier(ws)
    step_ms = max_over_ranks(sum(mx_ms) / len(mx_ms), ws)
    f64_step_ms = max_over_ranks(sum(f64_ms) / len(f64_ms), ws)
    kern_ms = sum(mx_kern) / len(mx_kern)
    f64_kern_ms = sum(f64_kern) / len(f64_kern)

    # end to end through the public API with pinned host buffers: matrix and
    # right-hand side uploaded, solution read back, every step
    dm_h, xm_h, _ = A.get()
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()
    dm_p, xm_p = pin(dm_h), pin(xm_h)
    b_p = pin(b.cpu().numpy())
    x_p = pin(np.zeros(npoin))
    e2e = []
    for s in range(args.warmup + args.steps):
        x_p[:] = 0.0
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        if args.storage == "seg":
            A.set_seg(dm_p, xm_p, "Q", "S")
        else:
            A.set(dm_p, xm_p, "Q", "S")
        bief.solve_mixed(x_p, A, b_p, precon=2, inner_tol=args.inner_tol, outer_tol=args.eps)
        t1 = time.perf_counter()
        if s >= args.warmup:
            e2e.append((t1 - t0) * 1e3)
    e2e_ms = max_over_ranks(sum(e2e) / len(e2e), ws)

    # the binary64 GRACJG the same way (SOLVE through the C ABI with host
    # buffers: matrix and right-hand side uploaded, solution read back)
    e2e64 = []
    for s in range(1 + max(2, args.steps // 4)):
        x_p[:] = 0.0
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        if args.storage == "seg":
            A.set_seg(dm_p, xm_p, "Q", "S")
        else:
            A.set(dm_p, xm_p, "Q", "S")
        bief.solve(x_p, A, b_p, cfg)
        t1 = time.perf_counter()
        if s >= 1:
            e2e64.append((t1 - t0) * 1e3)
    e2e64_ms = max_over_ranks(sum(e2e64) / len(e2e64), ws)
    e2e64_nsteps = len(e2e64)

    # beside the headline: the 2001 x 2001 log-uniform configuration and the
    # 256-mesh batch
    cfg2 = None
    hbm_b, _ = hbm_peak()
    if PL is not None and not args.no_extras:
        cfg2 = config2_measure(PL, ws, flush_l2, hbm_b)
    if PL is not None:
        PL["mesh"].close()
        del PL
    batch = None
    cfg3 = None
    if not args.no_extras:
        batch = batch_measure(ws, rank, local, 2, 1, 1e-4, args.eps)
        batch["steps"], batch["warmup"] = 2, 1
        cfg3 = config3_measure(ws)

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        cpu = cpu_baseline(args.n, args.eps, nit64, args.cpu_seconds, args.depth)

    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            peaks = json.load(fh)
    except Exception:
        pass
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    if mv_large:
        for key in ("matvec64", "matvec32"):
            mv_large[key]["frac"] = mv_large[key]["gbs"] / hbm
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    traffic = {}
    try:
        with open(os.path.join(ROOT, "profiles",
                               f"traffic_{args.n}_{args.storage}_{args.depth}.json")) as fh:
            traffic = json.load(fh)
    except Exception:
        pass
    mixed_bytes = inner * by["it32"] + (outer + 1) * by["upd"]
    achieved = mixed_bytes / (kern_ms * 1e-3) / 1e9
    mixed_traffic = traffic.get("k_mixed_bytes_per_launch")
    dram_gbs = mixed_traffic / (kern_ms * 1e-3) / 1e9 if mixed_traffic else None
    # the binary32 operator and vectors of the 1M-node solve (~96 MB) fit in
    # the 126 MB L2: whether the launch's working set stays in L2
    l2_resident = by["mv32"] < 126e6
    f64_bytes = nit64 * by["it64"]
    mv_gbs = by["mv64"] / (mv_t * 1e-3) / 1e9
    mv32_gbs = by["mv32"] / (mv32_t * 1e-3) / 1e9

    if rank == 0:
        line = {
            "metric": METRIC, "value": ws * 1000.0 / step_ms, "unit": UNIT, "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": step_ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 inner / f64 refinement", "data": "synthetic",
            "config": solve_config(args, npoin, nelem, P["nseg"], ws),
            "persistent_grid": _grid_info(P["mesh"], local),
            "time_to_solution_ms": {"mixed": step_ms, "fp64": f64_step_ms,
                                    "mixed_kernel": kern_ms, "fp64_kernel": f64_kern_ms},
            "speedup_mixed_vs_fp64": f64_step_ms / step_ms,
            "iterations": {"fp64": nit64, "mixed_inner": inner, "mixed_updates": outer},
            "cg_iterations_per_s": {"fp64": nit64 * 1000.0 / f64_kern_ms,
                                    "mixed_inner": inner * 1000.0 / kern_ms},
            "relres": {"mixed": relres, "fp64": f64_res[2]},
            "error": {"mixed_vs_fp64": mixed_vs_f64, "mixed_vs_xtrue": mixed_x_err,
                      "fp64_vs_xtrue": f64_x_err,
                      "fp64_one_step_at_stop": f64_step,
                      "vs_tight_fp64": {"mixed": mixed_vs_tight, "fp64": f64_vs_tight,
                                        "tight_relres": rel_tight,
                                        "tight_iterations": nit_tight}},
            "matvec": {"op": "X=AY binary64 TYPDIA=Q",
                       "kernel": "k_mvseg" if args.storage == "seg" else "k_matvec16", "ms": mv_t,
                       "ms_call": mv_t_call,
                       "timing": "ms: library events around the launch; ms_call: torch events "
                                 "around the Python call",
                       "gbs": mv_gbs, "frac": mv_gbs / hbm, "bytes": by["mv64"],
                       "traffic": traffic.get("k_matvec_bytes_per_launch")},
            "matvec32": {"op": "X=AY binary32, the mixed solve's inner operator applied to the "
                               "stored matrix (coefficients assembled per neighbour)",
                         "kernel": "k_matvec32", "ms": mv32_t, "gbs": mv32_gbs,
                         "frac": mv32_gbs / hbm, "bytes": by["mv32"],
                         "vs_fp64_matvec": mv32_err},
            "matvec_2001x2001": mv_large,
            "fp64_modass3": {"ms": sum(c64_ms) / len(c64_ms), "iterations": c64_res[1],
                             "vs_fp64": c64_vs_f64,
                             "note": "GRACJG with compensated dot products (MODASS=3)"},
            "fp64_cg": {"kernel": "k_cg64", "gbs": f64_bytes / (f64_kern_ms * 1e-3) / 1e9,
                        "frac": f64_bytes / (f64_kern_ms * 1e-3) / 1e9 / hbm,
                        "bytes_per_iteration": by["it64"], "bytes_per_launch": f64_bytes,
                        "traffic": traffic.get("k_cg64_bytes_per_launch")},
            "roofline": {"bound": "hbm", "kernel": "k_mixed", "achieved": achieved,
                         "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                         "peak_source": f"{peak_src} (MEASURED_PEAKS.json hbm_gbs)",
                         "bytes_per_launch": mixed_bytes,
                         "traffic": mixed_traffic,
                         "dram_gbs": dram_gbs,
                         "dram_frac": dram_gbs / hbm if dram_gbs else None,
                         "working_set": ("L2-resident: the binary32 operator and vectors "
                                         "(~96 MB) stay in the 126 MB L2, so frac is "
                                         "algorithmic bytes over time, not DRAM traffic "
                                         "(dram_frac); limited by L2 latency and the grid "
                                         "barriers" if l2_resident else
                                         "above L2: streamed from HBM")},
            "e2e": {"value": ws * 1000.0 / e2e_ms, "unit": UNIT,
                    "h2d_bytes_per_step": 8 * (npoin + int(xm_h.size)) + 16 * npoin,
                    "d2h_bytes_per_step": 8 * npoin, "ms_per_step": e2e_ms},
            "e2e_fp64": {"value": ws * 1000.0 / e2e64_ms, "unit": UNIT,
                         "h2d_bytes_per_step": 8 * (npoin + int(xm_h.size)) + 16 * npoin,
                         "d2h_bytes_per_step": 8 * npoin, "ms_per_step": e2e64_ms,
                         "steps": e2e64_nsteps,
                         "note": "binary64 GRACJG through bief_set_matrix + bief_solve with "
                                 "host buffers"},
            "config2": cfg2,
            "config3": cfg3,
            "batch256": batch,
            "gpu_launches": int(launches),
            "clocks": clk.summary(),
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    barrier(ws)
    mesh.close()
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
