"""Throughput benchmark: cell-updates/s of the explicit FV loop on one B200.

Workload (default): the 3D ramp channel (x in [0,3], y in [0,1], z in [0,1],
12 deg ramp from x = 0.5 up to y = 0.2) meshed as 200x100x50 hexes split into
6 tetrahedra each = 6,000,000 tets; Mach 3, p = 101325 Pa, T = 300 K;
HLLC flux, cell-limited MUSCL with the Venkatakrishnan limiter (K = 5),
Green-Gauss gradients, RK4 (the reference's standard coefficients),
LocalAccTime1 evaluated from stage-start values, CFL 0.5; FP32 state and
fluxes, FP64 geometry / RK state / residual norms; cells on a Hilbert curve.
One step = one iteration (4 RK stages) over all cells; by default the
timed region is the workload's whole 500-iteration run from the freestream
start (--steps overrides). Synthetic mesh and freestream start: no dataset
is involved.

  value : cell-updates/s with the state resident in HBM (K iterations in one
          psst_explicit_solve call, replayed as one CUDA graph captured
          before the timed region; CUDA events on the solver's stream)
  e2e   : same metric through the C ABI with host buffers: the initial state
          copied from pinned host memory, K per-iteration psst_explicit_solve
          calls each returning its residual columns to the host, the final
          state copied back -- all inside the timed region
  roofline: the dominant kernel's algorithmic bytes per launch over its mean
          launch time (psst_solver_profile), against the measured HBM peak
  cpu_baseline: the reference compiled from its own sources (oracle/_ref),
          one process per host core, on a reduced mesh of the same workload

--impl reference runs the reference's CPU implementation of the path on the
host cores instead and prints the same metric.
Multi-GPU: the path runs as independent replicas (one case per GPU, no
collective); value = all ranks' cell-updates / max rank time.
"""
import argparse
import glob
import json
import math
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    # the bandwidth benchmark: 200x100x50 hexes x 6 tets, FP32, MUSCL/Venkatakrishnan
    "wedge3d_6M_tets": dict(dim=3, mesh=(200, 100, 50), mach=3.0, angle=12.0, precision=32, limiter=5,
                            cpu_mesh=(40, 20, 4), cpu_procs=0, run_steps=500),
    # small case of the same workload for ncu captures
    "wedge3d_750k_tets": dict(dim=3, mesh=(100, 50, 25), mach=3.0, angle=12.0, precision=32, limiter=5,
                              cpu_mesh=(40, 20, 4), cpu_procs=0),
    # the reference's own 2D case (40x120 quads, 15 deg, Mach 2.5), FP64, MUSCL/Barth-Jespersen; the CPU
    # reference runs the same mesh on one core (it has no Barth-Jespersen: DM/VanLeer there)
    "ramp2d_120x40_fp64": dict(dim=2, mesh=(120, 40), mach=2.5, angle=15.0, precision=64, limiter=4,
                               cpu_mesh=(120, 40), cpu_procs=1),
    # the 2D case of the configs at its own size in the reference's own evaluation order: 120x40
    # quads, FP64, MUSCL/Barth-Jespersen, LocalAccTime1 in the reference's in-loop order (one
    # persistent launch per call); one step = the whole 2000-iteration run
    "ramp2d_120x40_seq_2000": dict(dim=2, mesh=(120, 40), mach=2.5, angle=15.0, precision=64, limiter=4,
                                   lc1_mode=0, step_iters=2000, cpu_mesh=(120, 40), cpu_procs=1, cpu_iters=100),
    # the reference's own published case, from its shipped files (tests/golden/shipped_wedge):
    # wedge80_240.msh (19,200 quads), HLL, first order, LocalAccTime1 in the reference's in-loop
    # order, RK1, CFL 2.08; one step = the whole 3000-iteration solve; FP64 (bit-exact with the
    # shipped wedge.sav); published: 152.856 s on the authors' PC
    "wedge80_240_shipped": dict(dim=2, shipped=True, precision=64, cpu_procs=1, cpu_iters=300),
}
# cell-updates/s of the published run: 19,200 cells x 3000 iterations in 152.856 s
PUBLISHED_SHIPPED = 19200 * 3000 / 152.856
SCHEME = dict(flux=3, order=2, grad=1, lc=1, rk_level=4, cfl=0.5)
CPU_LIMITER = 3  # the reference has no cell-based limiters: its DM/VanLeer path is timed


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled every 200 ms."""

    FIELDS = "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active," \
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown," \
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None
        self.path = tempfile.mktemp(suffix=".csv")

    def __enter__(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.dev), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            self.proc.wait()
            self.f.close()

    def summary(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        rows = []
        for line in open(self.path):
            p = [x.strip() for x in line.split(",")]
            if len(p) >= 9:
                rows.append(p)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def ramp_mesh(dim, size, angle):
    from supersonicflowsolver_b200 import meshgen

    if dim == 2:
        return meshgen.wedge2d(size[0], size[1], angle)
    return meshgen.wedge3d(size[0], size[1], size[2], angle, tets=True)


def shipped_fixture():
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    import make_shipped_wedge

    return make_shipped_wedge


def build_case(workload, directory):
    from supersonicflowsolver_b200 import meshgen
    from supersonicflowsolver_b200.psst import Grid

    w = WORKLOADS[workload]
    if w.get("shipped"):
        mesh_path, _, _ = shipped_fixture().unpack(directory)
        grid = Grid.read_fluent(mesh_path)
        sc, prim = grid.read_case(directory, "wedge")
        sc.precision = 64
        sc.lc1_mode = 0  # the reference's in-loop order
        sc.renumber = 1
        return grid, sc, prim
    mesh = ramp_mesh(w["dim"], w["mesh"], w["angle"])
    zones = [z.name for z in mesh.face_zones if z.bc_type != 2 and z.name not in ("in", "out", "side")]
    meshgen.write_case(directory, "bench", dim=w["dim"], zones=zones, mach=w["mach"], max_iter=1,
                       limiter=w["limiter"], **SCHEME)
    grid = Grid.from_mesh(mesh)
    del mesh
    sc, prim = grid.read_case(directory, "bench")
    sc.precision = w["precision"]
    sc.lc1_mode = w.get("lc1_mode", 1)
    sc.renumber = 1
    return grid, sc, prim


def traffic_model(grid, nnz, kind, precision=32):
    """Algorithmic (compulsory) DRAM bytes per launch of each kernel for the FP32
    3D MUSCL/Venkatakrishnan configuration: every array touched once, neighbour
    data counted once per cell (perfect on-chip reuse). s = 4 B state word,
    g = 8 B geometry word, i = 4 B index."""
    nint, ngh, nf = grid.ninterior, grid.nghost, grid.nface
    K = nnz / nint
    if kind == "face":
        # per face: face record read (64: c0,c1 (2i), S (g), n (3g), two FP32 offset vectors)
        # and the face output record written (32: flux*area 5s, time-step terms 3s);
        # per interior cell: state record (32) + limited-gradient record (64); ghosts: state (32)
        return nf * (64 + 32) + nint * (32 + 64) + ngh * 32
    if kind == "cell":
        # per cell: CSR ptr (i) + K entries (i) + K face areas (s) + own-order perm (8) + V (g) +
        # the stage-start FP64 state read (5x8) + new state record (32) + ghost ptr (i), and,
        # averaged over the S stages of an iteration, the stage-start copy written on the first
        # stage and w and dt written on the last (5x8 + 5x8 + 8) / S; per face: face output
        # record (32); per ghost: record in and out (2x32) + ids (2i)
        S = SCHEME["rk_level"]
        return nint * (4 + 4 * K + 4 * K + 8 + 8 + 40 + 88.0 / S + 32 + 4) + nf * 32 + ngh * 72
    if kind == "gradient":
        if precision == 32 and K == 4:
            # FP32, 4 faces per cell (the per-entry coefficient table): per cell the 4
            # neighbour ids (4i), the table (4 entries x (2 dim + 1) s), eps^2 (g), own state
            # record (32), limited-gradient record written (64); ghosts: state record (32)
            return nint * (16 + 16 * (2 * grid.dim + 1) + 8 + 32 + 64) + ngh * 32
        # per cell: CSR (i + K i) + perm + V + eps^2 + own state record (32) + limited-gradient
        # record written (64); per face: face record (64) + beta (g); ghosts: state record (32)
        return nint * (4 + 4 * K + 8 + 8 + 8 + 32 + 64) + nf * 72 + ngh * 32
    if kind == "ghost_update":
        return ngh * (12 + 20 + 20 + 24 + 24)
    return 0


def read_traffic(kernel, workload):
    """DRAM bytes (read + write) per launch of k_<kernel> on `workload` from the
    committed ncu summaries: a line 'dram_bytes_per_launch[<workload>]: N' in
    profiles/k_<kernel>_*.txt."""
    tag = "dram_bytes_per_launch[%s]:" % workload
    for path in sorted(glob.glob(os.path.join(ROOT, "profiles", "k_%s_*.txt" % kernel))):
        for line in open(path):
            if line.startswith(tag):
                return float(line.split(":")[1].split()[0])
    return None


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d["hbm_gbs"], "measured"
    return 6650.0, "fallback"


# ---------------------------------------------------------------- CPU side ---
def reference_binary():
    ref = os.path.join(ROOT, "oracle", "_ref", "psst_ref")
    if os.path.exists(ref):
        return ref, "reference"
    port = os.path.join(ROOT, "oracle", "_build", "psst_oracle")
    if not os.path.exists(port):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "port"], capture_output=True)
    return port, "port"


def cpu_run(n_iter, procs, workload="wedge3d_6M_tets"):
    """Runs the reference (or the oracle port where the reference was not built)
    on the reduced mesh, `procs` independent processes, n_iter iterations each.
    Returns per-process per-iteration loop times (s) from the residual file's
    time column (mesh reading and setup excluded, as the reference prints)."""
    from supersonicflowsolver_b200 import meshgen

    exe, kind = reference_binary()
    w = WORKLOADS[workload]
    base = tempfile.mkdtemp(prefix="psst_cpu_")
    runs = []
    if w.get("shipped"):  # the shipped files, with maxIter (line 4) and iterSaveStep (line 5) bounded
        name, ncells = "wedge", 19200
        for p in range(procs):
            d = os.path.join(base, "p%d" % p)
            os.makedirs(d)
            shipped_fixture().unpack(d)
            lines = open(os.path.join(d, "wedge.inp")).read().split("\n")
            lines[3] = "%d\t\t//maxIter" % n_iter
            lines[4] = "%d\t\t//iterSaveStep" % 10 ** 6
            open(os.path.join(d, "wedge.inp"), "w").write("\n".join(lines))
            open(os.path.join(d, "problem_manager"), "w").write("wedge80_240.msh\nwedge")
            runs.append(subprocess.Popen([exe], cwd=d, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL))
    else:
        name = "c"
        mesh = ramp_mesh(w["dim"], w["cpu_mesh"], w["angle"])
        ncells = mesh.ncells
        zones = [z.name for z in mesh.face_zones if z.bc_type != 2 and z.name not in ("in", "out", "side")]
        meshgen.write_fluent(mesh, os.path.join(base, "m.msh"))
        for p in range(procs):
            d = os.path.join(base, "p%d" % p)
            os.makedirs(d)
            os.link(os.path.join(base, "m.msh"), os.path.join(d, "m.msh"))
            meshgen.write_case(d, "c", dim=w["dim"], zones=zones, mach=w["mach"], max_iter=n_iter,
                               save_step=10 ** 6, limiter=CPU_LIMITER, **SCHEME)
            open(os.path.join(d, "problem_manager"), "w").write("m.msh\nc")
            runs.append(subprocess.Popen([exe], cwd=d, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL))
    for r in runs:
        r.wait()
    times = []
    for p in range(procs):
        f = os.path.join(base, "p%d" % p, name + "_residual.dat")
        rows = [l.split() for l in open(f) if l.strip()] if os.path.exists(f) else []
        if len(rows) == n_iter:
            times.append([float(r[1]) for r in rows])
    shutil.rmtree(base, ignore_errors=True)
    return times, kind, ncells, exe


def cpu_procs(workload):
    n = WORKLOADS[workload]["cpu_procs"]
    return n if n > 0 else max(1, os.cpu_count() or 1)


def cpu_sample_text(workload, ncells):
    w = WORKLOADS[workload]
    if w.get("shipped"):
        return "the shipped case itself (%d quads, HLL first order, RK1, LocalAccTime1), iterations bounded" % ncells
    mesh = "x".join(str(v) for v in w["cpu_mesh"])
    kind = "tets (%s hexes x6" % mesh if w["dim"] == 3 else "quads (%s" % mesh
    return "%d %s, same ramp/Mach/scheme, DM+VanLeer limiter)" % (ncells, kind)


def cpu_baseline(warm, steps, workload):
    times, kind, ncells, exe = cpu_run(warm + steps, cpu_procs(workload), workload)
    if not times:
        return None
    # the time column is cumulative ms-resolution wall time since the loop began
    span = [t[warm + steps - 1] - (t[warm - 1] if warm > 0 else 0.0) for t in times]
    rate = sum(ncells * steps / s for s in span if s > 0)
    return {"value": rate, "unit": "cell-updates/s", "cores": len(times), "kind": kind,
            "sample": "%s, %d timed + %d warm-up iterations per process, %d processes" %
                      (cpu_sample_text(workload, ncells), steps, warm, len(times)),
            "binary": os.path.relpath(exe, ROOT)}


def run_reference_arm(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    iters = WORKLOADS[args.workload].get("cpu_iters")
    warm, steps = (1, iters) if iters else (args.warmup, args.steps)
    times, kind, ncells, exe = cpu_run(warm + steps, cpu_procs(args.workload), args.workload)
    if not times:
        print(json.dumps({"impl": "reference", "unavailable": "the reference binary produced no residual file"}))
        return
    span = [t[-1] - t[warm - 1] for t in times]
    value = sum(ncells * steps / s for s in span if s > 0)
    ms = 1000.0 * max(span) / steps
    print(json.dumps({
        "metric": "cell-updates/s", "value": value, "unit": "cell-updates/s", "impl": "reference",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "%s (CPU sample: %s)" % (args.workload, cpu_sample_text(args.workload, ncells)),
                   "scheme": scheme_text(args.workload, cpu=True),
                   "parallelism": "%d independent processes" % len(times)},
        "cpu_baseline": {"value": value, "unit": "cell-updates/s", "cores": len(times), "kind": kind,
                         "sample": "%d cells per process, %d timed + %d warm-up iterations (ms_per_step: "
                                   "one iteration)" % (ncells, steps, warm)},
        "e2e": {"value": value, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def scheme_text(workload, cpu=False):
    w = WORKLOADS[workload]
    if w.get("shipped"):
        return "HLL, first order, LocalAccTime1 in the reference's in-loop order, RK1, CFL 2.08 (wedge.inp)"
    lim = "DM/VanLeer" if cpu else ("MUSCL/Venkatakrishnan(K=5)" if w["limiter"] == 5 else "MUSCL/Barth-Jespersen")
    lc = "LocalAccTime1" if cpu or w.get("lc1_mode") == 0 else "LocalAccTime1 (stage-start values)"
    if not cpu and w.get("lc1_mode") == 0:
        lc += " in the reference's in-loop order"
    return "HLLC + %s, Green-Gauss, RK4 std, %s, CFL 0.5, Mach %g, %g deg ramp" % (lim, lc, w["mach"], w["angle"])


# ---------------------------------------------------------------- GPU side ---
def max_over_ranks(values, ws, device):
    """Element-wise max over the ranks of the process group (the slowest
    replica's times); identity for one rank."""
    if ws <= 1:
        return list(values)
    import torch
    import torch.distributed as dist

    t = torch.tensor(values, dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t]


def replica_throughput(ws, cells, steps, ms_max, e2e_s_max):
    """Whole-job cell-updates/s of ws independent replicas of `cells` cells
    run for `steps` iterations, timed by the slowest rank (device ms, e2e s)."""
    return ws * cells * steps / (ms_max / 1000.0), ws * cells * steps / e2e_s_max


def field_errors(grid, sc, a, b):
    """Max and RMS relative difference of rho, p and Mach between two states
    (prim layout of psst_solver_get_state, rho from get("rho")) over interior
    cells; a is measured against b."""
    nv, dim = grid.nvol, grid.dim
    interior = grid.get("vol_bc") == 1
    out = {}
    for k in ("rho", "p", "mach"):
        x, y = a[k][interior], b[k][interior]
        rel = np.abs(x - y) / np.abs(y)
        out[k] = {"max_rel": float(rel.max()), "rms_rel": float(np.sqrt(np.mean(rel * rel)))}
    return out


def state_fields(solver, grid, sc):
    prim = solver.get_state()
    nv, dim = grid.nvol, grid.dim
    T = prim[nv:2 * nv]
    speed = np.sqrt(sum(prim[(2 + k) * nv:(3 + k) * nv] ** 2 for k in range(dim)))
    return {"rho": solver.get("rho"), "p": prim[:nv], "mach": speed / np.sqrt(sc.gamma * sc.rm * T)}


def reference_scheme(args, grid, sc, prim, stream_ptr, dev):
    """The FP32 path on the same mesh with the limiter the reference arm runs
    (DM reconstruction + VanLeer, the reference's own scheme; it has no cell
    limiters): device-resident throughput, its own tuned launch shapes, K
    iterations in one graph replay -- the figure to set beside the reference
    arm's per-cell rate."""
    import torch
    from supersonicflowsolver_b200.psst import Solver

    sc3 = type(sc).from_buffer_copy(sc)
    sc3.limiter = CPU_LIMITER
    s3 = Solver(grid, sc3, device=dev)
    s3.set_stream(stream_ptr)
    s3.set_state(prim)
    shapes = s3.autotune(2) if not args.no_autotune else s3.launch_shape()
    s3.use_graphs(True)
    s3.explicit_solve(args.warmup)
    s3.explicit_solve(args.steps)
    s3.explicit_solve(args.steps)
    torch.cuda.synchronize()
    s3.explicit_solve(args.steps)
    ms = s3.last_stats()[1]
    s3.close()
    return {"value": grid.ninterior * args.steps / (ms / 1000.0), "unit": "cell-updates/s",
            "ms_per_step": ms / args.steps, "threads_per_block": shapes,
            "scheme": scheme_text(args.workload).replace("MUSCL/Venkatakrishnan(K=5)", "DM/VanLeer")}


def fp64_and_precision(args, grid, sc, prim, fp32_solver, stream_ptr, dev, n_prec=500):
    """The same workload on the FP64 path (the reference's precision): its
    device-resident throughput over `steps` iterations, and the FP32
    production path's field error against it after n_prec iterations from the
    same start (rho, p, Mach; max and RMS relative, interior cells)."""
    import torch
    from supersonicflowsolver_b200.psst import Solver

    sc64 = type(sc).from_buffer_copy(sc)
    sc64.precision = 64
    s64 = Solver(grid, sc64, device=dev)
    s64.set_stream(stream_ptr)
    s64.set_state(prim)
    shapes = s64.autotune(2) if not args.no_autotune else s64.launch_shape()
    s64.use_graphs(True)
    s64.explicit_solve(args.warmup)
    s64.explicit_solve(args.steps)
    s64.explicit_solve(args.steps)
    torch.cuda.synchronize()
    s64.explicit_solve(args.steps)
    ms = s64.last_stats()[1]
    prof = s64.profile(2)
    rec = {"value": grid.ninterior * args.steps / (ms / 1000.0), "ms_per_step": ms / args.steps,
           "kernel_ms_per_iteration": {k: t / 2 for k, (t, n) in prof.items()}, "threads_per_block": shapes,
           "note": "same mesh and scheme on the FP64 path (FP64 state, fluxes and arithmetic; -fmad=false), its "
                   "own tuned launch shapes, K iterations in one call replayed as a CUDA graph"}
    # precision: both paths n_prec iterations from the freestream start
    s64.set_state(prim)
    fp32_solver.set_state(prim)
    s64.explicit_solve(n_prec)
    fp32_solver.explicit_solve(n_prec)
    err = field_errors(grid, sc, state_fields(fp32_solver, grid, sc), state_fields(s64, grid, sc64))
    s64.close()
    return rec, {"iterations": n_prec, "fp32_vs_fp64": err}


def gemm_throughput():
    """The learned part's tensor-core GEMM (psst_tc_gemm_bf16, tcgen05 BF16 ->
    FP32) on the warm-start network's training shapes: a hidden layer forward
    (16384 points x 256 outputs x 256 inputs, both operands contiguous along
    K) and its weight gradient (256 x 256 over 16384 points, both operands
    contiguous along M/N, split over K in 256-row slices), plus a square
    8192^3 product that the tensor cores bound. TFLOP/s against the measured
    BF16 peak and against each shape's own HBM bound (operands read once,
    FP32 result written once); device time per launch, launches back to
    back."""
    import torch
    from supersonicflowsolver_b200.mlp import tc_gemm_time

    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    d = json.load(open(p)) if os.path.exists(p) else {}
    peak, peak_kind = (d["bf16_tflops"], "measured") if "bf16_tflops" in d else (1590.0, "fallback")
    hbm, _ = peaks()
    g = torch.Generator(device="cuda").manual_seed(0)
    X = torch.randn((16384, 256), generator=g, device="cuda").to(torch.bfloat16)
    W = torch.randn((256, 256), generator=g, device="cuda").to(torch.bfloat16)
    Y = torch.randn((16384, 256), generator=g, device="cuda").to(torch.bfloat16)
    out = {"peak_tflops": peak, "peak_kind": peak_kind}
    S = torch.randn((8192, 8192), generator=g, device="cuda").to(torch.bfloat16)
    T = torch.randn((8192, 8192), generator=g, device="cuda").to(torch.bfloat16)
    for name, kw, M, N, K, dbytes, reps in (
            ("forward_16384x256x256", dict(A=X, B=W), 16384, 256, 256, 16384 * 256 * 4, 20),
            ("weight_grad_256x256x16384", dict(A=X, B=Y, a_strides=(1, 256), b_strides=(1, 256), M=256, N=256,
                                               K=16384, k_split=256), 256, 256, 16384, 64 * 256 * 256 * 4, 20),
            ("square_8192", dict(A=S, B=T), 8192, 8192, 8192, 8192 * 8192 * 4, 5)):
        tc_gemm_time(reps=2, **kw)
        ms = tc_gemm_time(reps=reps, **kw)
        flops = 2.0 * M * N * K
        byts = 2.0 * (M * K + N * K) + dbytes
        tf = flops / (ms * 1e-3) / 1e12
        bound = min(peak, flops / (byts / (hbm * 1e9)) / 1e12)
        out[name] = {"ms": ms, "tflops": tf, "frac_of_peak": tf / peak, "hbm_bound_tflops": bound,
                     "frac_of_shape_bound": tf / bound}
    del S, T
    # one whole training step of the warm-start network (forward, backward,
    # Adam, the loss read back), batch 16384: wall time per step
    from supersonicflowsolver_b200.mlp import MLP

    net = MLP(seed=0)
    xb = torch.rand((16384, 4), generator=g, device="cuda") * 2.0 - 1.0
    tb = torch.rand((16384, 4), generator=g, device="cuda")
    for _ in range(3):
        net.train_step(xb, tb, 1e-3)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(20):
        net.train_step(xb, tb, 1e-3)
    torch.cuda.synchronize()
    step_ms = (time.perf_counter() - t0) * 1000.0 / 20
    # 5 forward, 5 weight-gradient and 4 data-gradient GEMMs (none into the features)
    gemm_flops = 2.0 * 16384 * (3 * (256 * 128 + 4 * 256 * 256) - 256 * 128)
    out["mlp_train_step_16384"] = {"ms": step_ms, "gemm_tflops_effective": gemm_flops / (step_ms * 1e-3) / 1e12,
                                   "note": "wall time per step (it reads the loss back, so each step waits for "
                                           "its kernels); 14 tensor-core GEMMs plus features, output layer, "
                                           "reductions and Adam"}
    net.close()
    return out


def run_gpu(args):
    import torch

    ws, rank, local = dist_env()
    if ws > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    dev = local
    torch.cuda.set_device(dev)
    from supersonicflowsolver_b200.psst import Solver

    tmp = tempfile.mkdtemp(prefix="psst_bench_")
    grid, sc, prim = build_case(args.workload, tmp)
    solver = Solver(grid, sc, device=dev)
    stream = torch.cuda.Stream(device=dev)
    solver.set_stream(stream.cuda_stream)
    solver.set_state(prim)
    nint = grid.ninterior
    wl = WORKLOADS[args.workload]
    shipped = bool(wl.get("shipped"))
    # one step: one iteration, or a whole run (the published solve; the 2000-iteration case)
    per_step = int(sc.max_iter) if shipped else int(wl.get("step_iters", 1))
    whole = per_step > 1  # sequential LocalAccTime1: one persistent launch per call
    shapes = solver.autotune(3) if not (args.no_autotune or whole) else solver.launch_shape()
    # replay whole explicit_solve calls as CUDA graphs (no launch gaps between
    # the passes; on small meshes launch latency dominates); the published case
    # runs as one persistent launch per call (sequential LocalAccTime1)
    if args.graphs == "on":
        solver.use_graphs(True)

    def barrier():
        if ws > 1:
            import torch.distributed as dist

            dist.barrier()
        torch.cuda.synchronize()

    # warm-up
    solver.explicit_solve(args.warmup * per_step)
    if solver.graphs_on and not whole:  # capture the timed call's graphs (one per buffer parity) outside the timed region
        solver.explicit_solve(args.steps * per_step)
        solver.explicit_solve(args.steps * per_step)
        solver.explicit_solve(per_step)
        solver.explicit_solve(per_step)
    barrier()
    # device-resident timed region; inputs (~2.6 GB of mesh + state) exceed the 126 MB L2
    with ClockSampler(dev) as clk:
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        barrier()
        ev0.record(stream)
        linf, _ = solver.explicit_solve(args.steps * per_step)
        ev1.record(stream)
        barrier()
        ms = ev0.elapsed_time(ev1)
        launches, lib_ms = solver.last_stats()
        # end-to-end through the C ABI with host buffers
        host_prim = torch.from_numpy(prim).pin_memory()
        host_out = torch.empty_like(host_prim).pin_memory()
        barrier()
        t0 = time.perf_counter()
        if whole:  # each step: the whole run from its initial state, host to host
            for _ in range(args.steps):
                solver.set_state(host_prim.numpy())
                solver.explicit_solve(per_step)
                out = solver.get_state(out=host_out.numpy())
        else:
            solver.set_state(host_prim.numpy())
            for _ in range(args.steps):
                solver.explicit_solve(1)
            out = solver.get_state(out=host_out.numpy())
        torch.cuda.synchronize()
        e2e_s = time.perf_counter() - t0
    clocks = clk.summary()
    ms_max, e2e_max = max_over_ranks([ms, e2e_s], ws, "cuda")
    value, e2e_value = replica_throughput(ws, nint * per_step, args.steps, ms_max, e2e_max)
    # per-kernel timing for the roofline (CUDA events around each launch)
    prof = solver.profile(2 * per_step if whole else 2)
    nnz = 2 * grid.nface - grid.nghost  # CSR entries: interior faces twice, boundary faces once
    kernel, (kms, kcnt) = max(prof.items(), key=lambda kv: kv[1][0])
    peak, peak_kind = peaks()
    finite = bool(np.all(np.isfinite(linf))) and bool(np.all(np.isfinite(out)))
    if whole:
        info = solver.schedule_info()
        nopi = sc.rk_level + (1 if sc.order == 2 else 0)
        nsteps = info["period"] * (2 * per_step * nopi - 1) + info["levels"] + 1  # of the profiled call
        roof = {"bound": "latency", "kernel": "wavefront", "achieved": None, "peak": peak, "peak_kind": peak_kind,
                "unit": "GB/s", "frac": None, "traffic": None,
                "note": "one persistent launch per call; a %d-iteration call is %d grid-barrier steps "
                        "(period %d, %d levels, %d CTAs), %.2f us per step: bound by the barrier and the "
                        "dependent loads of a step, not by HBM" %
                        (2 * per_step, nsteps, info["period"], info["levels"], info["blocks"],
                         1000.0 * kms / kcnt / nsteps)}
    else:
        algo = traffic_model(grid, nnz, kernel, wl["precision"])
        achieved = algo / (kms / kcnt / 1000.0) / 1e9
        roof = {"bound": "hbm", "kernel": kernel, "achieved": achieved, "peak": peak, "peak_kind": peak_kind,
                "unit": "GB/s", "frac": achieved / peak, "algorithmic_bytes_per_launch": algo,
                "launch_ms": kms / kcnt, "traffic": read_traffic(kernel, args.workload)}
        # every kernel of the iteration against the same peak (the same event timings)
        per, tot = {}, 0.0
        for k, (t, n) in prof.items():
            b = traffic_model(grid, nnz, k, wl["precision"])
            if n == 0 or t <= 0.0 or b == 0:
                continue
            tot += b * n / (2 * per_step)
            per[k] = {"launch_ms": t / n, "algorithmic_bytes_per_launch": b,
                      "achieved": b / (t / n / 1000.0) / 1e9, "frac": b / (t / n / 1000.0) / 1e9 / peak}
        roof["kernels"] = per
        it_s = ms_max / (args.steps * per_step) / 1000.0  # the timed iteration
        roof["iteration"] = {"algorithmic_bytes": tot, "ms": it_s * 1000.0, "frac": tot / it_s / 1e9 / peak}
    extra = {}
    if args.workload == "wedge3d_6M_tets" and not args.no_fp64 and ws == 1:
        extra["fp64"], extra["precision"] = fp64_and_precision(args, grid, sc, prim, solver, stream.cuda_stream, dev)
    if args.workload == "wedge3d_6M_tets" and ws == 1:
        extra["reference_scheme"] = reference_scheme(args, grid, sc, prim, stream.cuda_stream, dev)
        extra["tensor_gemm"] = gemm_throughput()
    if rank == 0:
        nv = grid.dim + 2
        state_bytes = (2 + grid.dim) * grid.nvol * 8
        line = {
            "metric": "cell-updates/s", "value": value, "unit": "cell-updates/s", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
            "higher_is_better": True, "scaling": "weak",
            "vs_baseline": value / PUBLISHED_SHIPPED if shipped else None,
            "dtype": "f32" if wl["precision"] == 32 else "f64",
            "data": "the reference's shipped mesh and setup" if shipped else "synthetic",
            "config": {"workload": args.workload, "cells": nint, "faces": grid.nface,
                       "scheme": scheme_text(args.workload),
                       "precision": ("FP32 state/flux; FP64 geometry, RK state, residual norms"
                                     if wl["precision"] == 32 else "FP64 throughout (the parity path)"),
                       "parallelism": "replicas" if ws > 1 else "single GPU",
                       "threads_per_block": shapes,
                       "cuda_graphs": args.graphs == "on" and not whole,
                       "l2_flush": ("not needed: >2.5 GB of mesh + state per step, L2 is 126 MB" if wl["dim"] == 3
                                    else "none: this small case stays in L2 (not the bandwidth benchmark)")},
            "e2e": {"value": e2e_value, "unit": "cell-updates/s",
                    "h2d_bytes_per_step": state_bytes if whole else state_bytes / args.steps,
                    "d2h_bytes_per_step": (state_bytes + per_step * 2 * nv * 8 + 16) if whole else
                                          (state_bytes / args.steps) + 2 * nv * 8 + 16,
                    "note": ("per step: set_state from pinned host memory, one psst_explicit_solve of the %d "
                             "iterations returning every residual column, get_state into pinned host memory; "
                             "all timed" % per_step) if whole else
                            "set_state from pinned host memory + K psst_explicit_solve(1) calls each returning "
                            "residual columns + get_state into pinned host memory, all timed"},
            "gpu_launches": int(launches),
            "clocks": clocks,
            "roofline": roof,
            "kernel_ms_per_iteration": {k: v[0] / (2 * per_step if whole else 2) for k, v in prof.items()},
            "library_device_ms": lib_ms,
            "finite": finite,
        }
        if whole:
            line["config"]["step"] = "the whole run: %d iterations of %d cells" % (per_step, nint)
        if shipped:
            line["config"]["published"] = {"wall_s": 152.856, "cell_updates_per_s": PUBLISHED_SHIPPED,
                                           "hardware": "authors' PC, one thread (README)"}
        line.update(extra)
        if not args.no_cpu_baseline:
            iters = wl.get("cpu_iters")
            cb = cpu_baseline(1, iters if iters else (10 if wl["dim"] == 3 else 200), args.workload)
            line["cpu_baseline"] = cb
        print(json.dumps(line))
    solver.close()
    shutil.rmtree(tmp, ignore_errors=True)
    if ws > 1:
        import torch.distributed as dist

        dist.barrier()
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None,
                    help="timed steps (default: the workload's run length, e.g. the 6M-tet ramp's 500 iterations)")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="wedge3d_6M_tets", choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--graphs", choices=["on", "off"], default="on",
                    help="replay each explicit_solve call as a CUDA graph")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default launch shapes")
    ap.add_argument("--no-fp64", action="store_true",
                    help="skip the FP64 line and the FP32-vs-FP64 field error of the 6M-tet workload")
    ap.add_argument("--gemm-only", action="store_true",
                    help="print only the tensor-core GEMM figures (the tensor_gemm object) and exit")
    args = ap.parse_args()
    if args.steps is None:
        args.steps = WORKLOADS[args.workload].get("run_steps", 20)
    if args.warmup < 3:
        ap.error("--warmup must be at least 3")
    if args.gemm_only:
        print(json.dumps({"tensor_gemm": gemm_throughput()}))
        return
    if args.impl == "reference":
        run_reference_arm(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
