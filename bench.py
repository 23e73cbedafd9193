"""Benchmark: FP64-accurate solves/s of the 2-D P1 Poisson problem on a
2049x2049-node triangulated unit square (n = 4,190,209 unknowns, nnz =
29,315,089), f uniform in [-1, 1] per node from seed 1234, u = 0 on the
boundary.

One step = Equation::build() (element assembly into the CSR matrix and RHS
from the source term resident in HBM) + the solve to an FP64 true relative
residual ||b - A x|| / ||b|| <= 1e-10 + insertBC.  The chosen solver is the
learned + mixed-precision one: FP64 refinement around a preconditioned CG in FP32
whose preconditioner M = G^T G is predicted by the library's network from the
assembled matrix inside every step (the network is trained once before the
timed region, on small problems, by the library's own kernels); `--prec
jacobi` selects the Jacobi inner iteration.  The plain FP64 CG + D-ILU solve
(OFELI's own method) is timed once beside it.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
                    [--workload poisson2d|kuhn3d|batch2d|transient2d|meshfile2d]

N > 1 runs N independent replicas (the problem does not shard; no
collective in the data path), launched one rank per GPU by torchrun.
"""
import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

METRIC = "FP64-accurate solves/sec (2-D P1 Poisson 2049x2049, true rel. residual <= 1e-10)"
METRIC_3D = "FP64-accurate solves/sec (3-D P1 variable-k diffusion 129^3, true rel. residual <= 1e-10)"
METRIC_TRANSIENT = ("backward-Euler time steps/sec (DC2DT3 convection-diffusion 1025x1025, "
                    "GMRES(30) to 1e-10 per step, warm start)")
METRIC_BATCH = ("FP64-accurate solves/sec (1024 uneven 2-D P1 problems, 1e3..6.4e4 nodes, "
                "true rel. residual <= 1e-10)")
METRIC_MESHFILE = ("mesh nodes/sec from an OFELI .m file to the assembled P1 system on the device "
                   "(Mesh::get + SpMatrix(mesh) + build(), 1.05M-node annulus)")
UNIT = "solves/s"
SEED = 1234
TOL = 1e-10
# OFELI's own CG + ILU (= diagonal ILU) on this problem converges in this
# many iterations (run to convergence with the reference built from its
# sources, tol 1e-10); used to extrapolate the bounded CPU samples.
REF_ITERS_2049_ILU = 2030
# the same for the 3-D problem (Kuhn cube 129^3, lognormal k, seed 1234):
# 257 CG + ILU iterations; OFELI's own times at -O2 on one core of the
# container that ran it (graph, assembly, solve)
REF_ITERS_129_ILU = 257
REF_TIMES_129_ILU = {"graph_s": 43.9, "assembly_s": 9.13, "solve_s": 56.2}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--nx", type=int, default=2048, help="cells per side (nodes = nx+1)")
    ap.add_argument("--workload", default="poisson2d",
                    choices=["poisson2d", "kuhn3d", "batch2d", "transient2d", "meshfile2d"],
                    help="poisson2d: the headline 2-D problem; kuhn3d: the 3-D "
                         "variable-coefficient problem (129^3 Kuhn cube, lognormal k); batch2d: "
                         "1024 uneven jittered 2-D problems in one persistent launch; "
                         "transient2d: DC2DT3 backward-Euler steps at 1025^2 (a step = one time "
                         "step); meshfile2d: an OFELI .m mesh file read and turned into the "
                         "assembled P1 system on the device (a step = one file)")
    ap.add_argument("--nprob", type=int, default=1024,
                    help="batch2d: number of problems (the workload is 1024; smaller counts are "
                         "for profiling captures)")
    ap.add_argument("--shard", action="store_true",
                    help="batch2d with N > 1: split the problem list over the ranks by estimated "
                         "cost (strong scaling) instead of one replica of it per rank")
    ap.add_argument("--batch-bits", type=int, default=32, choices=[32, 64],
                    help="batch2d: inner CG precision (32: FP32 CG inside FP64 refinement)")
    ap.add_argument("--tprec", default="MIXED", choices=["ILU", "DIAG", "MIXED", "LEARNED"],
                    help="transient2d: solver of the timed steps -- ILU / DIAG: FP64 GMRES(30) "
                         "(OFELI's GMRes) with that preconditioner; MIXED / LEARNED: the "
                         "mixed-precision flexible GMRES(30) (FP32 products, FP64 Gram-Schmidt "
                         "and refinement, converged on the FP64 true residual) with the diagonal "
                         "or the learned preconditioner (the plain ILU form is timed beside it)")
    ap.add_argument("--t-inner-tol", type=float, default=1e-5,
                    help="transient2d MIXED / LEARNED: residual reduction of one FGMRES cycle")
    ap.add_argument("--m3d", type=int, default=128, help="kuhn3d cells per side")
    ap.add_argument("--mf-n", type=int, default=1024,
                    help="meshfile2d: circles and nodes per circle of the annulus (the workload "
                         "is 1024; smaller sizes are for profiling captures)")
    ap.add_argument("--inner-bits", type=int, default=0, choices=[0, 32, 16],
                    help="matrix values of the inner iteration: 32 FP32, 16 BF16, 0 BF16 when "
                         "every value is exact in BF16 (lossless) else FP32")
    ap.add_argument("--prec", default="learned", choices=["jacobi", "learned"],
                    help="preconditioner of the FP32 inner iteration (learned: the network is "
                         "trained first on small problems of the workload's dimension, outside "
                         "the timed region, and runs inside every step)")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain FP64 CG+D-ILU solve")
    ap.add_argument("--no-3d", action="store_true",
                    help="poisson2d: skip the 3-D problem the default run also measures")
    ap.add_argument("--cpu-iters", type=int, default=10, help="CG iterations per CPU sample")
    return ap.parse_args()


# ------------------------------------------------------------------ clocks --
class ClockSampler:
    """nvidia-smi sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    try:
        with open(os.path.join(HERE, "MEASURED_PEAKS.json")) as fh:
            j = json.load(fh)
        return float(j["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def ncu_traffic(kernel):
    """DRAM bytes per launch from the committed ncu summary, or None."""
    try:
        with open(os.path.join(HERE, "profiles", "traffic.json")) as fh:
            return json.load(fh).get(kernel)
    except (OSError, ValueError):
        return None


# ------------------------------------------------------ CPU baseline (port) --
def cpu_baseline_port(nx, iters):
    """The oracle port (C restatement, 1 thread) on a bounded sample of the
    same workload: mesh, graph, assembly, D-ILU setup and `iters` CG
    iterations; the solve is extrapolated to the iteration count OFELI
    needs at this size."""
    from oracle import oracle as O
    from ofeli_b200 import fields
    xy, elem, code = O.mesh2d(nx, nx)
    f = fields.uniform_pm1(SEED, code.size)
    dof, n = O.number_equations(code)
    rp, ci = O.node_graph(elem, 3, dof, n)
    t0 = time.perf_counter()
    a, b = O.assemble(2, xy, elem, dof, code, n, rp, ci, f=f, bc=np.zeros(code.size))
    t1 = time.perf_counter()
    x, it = O.cg(rp, ci, a, b, O.ILU, iters, 1e-300)
    t2 = time.perf_counter()
    full_iters = REF_ITERS_2049_ILU if (nx == 2048 and REF_ITERS_2049_ILU) else None
    per_it = (t2 - t1) / iters
    if full_iters is None:
        full_iters = int(round(1097 * (nx / 1024.0)))  # CG+ILU iterations grow ~ linearly in nx
    t_solve = (t1 - t0) + per_it * full_iters
    return {"value": 1.0 / t_solve, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": "oracle port, 1 thread: assembly + D-ILU setup + %d CG iterations at %dx%d "
                      "nodes, solve extrapolated to %d iterations (%.3f s assembly, %.4f s/iter)"
                      % (iters, nx + 1, nx + 1, full_iters, t1 - t0, per_it),
            "host_cores": os.cpu_count()}


def cpu_baseline_port3d(M, iters, full_iters):
    """The oracle port, 1 thread, on the 3-D problem: assembly + D-ILU setup
    + `iters` CG iterations, extrapolated to the CG + ILU iteration count of
    the full solve (the GPU plain path's count, which equals OFELI's wherever
    both were run)."""
    from oracle import oracle as O
    from ofeli_b200 import fields
    xyz, elem, code = O.mesh3d(M)
    cent = xyz.reshape(-1, 3)[elem.reshape(-1, 4)].mean(axis=1)
    k = fields.lognormal_k(SEED, cent, 1.5, 0.1, grid=256)
    f = fields.uniform_pm1(SEED, code.size)
    dof, n = O.number_equations(code)
    rp, ci = O.node_graph(elem, 4, dof, n)
    t0 = time.perf_counter()
    a, b = O.assemble(3, xyz, elem, dof, code, n, rp, ci, k=k, f=f, bc=np.zeros(code.size))
    t1 = time.perf_counter()
    O.cg(rp, ci, a, b, O.ILU, iters, 1e-300)
    t2 = time.perf_counter()
    per_it = (t2 - t1) / iters
    t_solve = (t1 - t0) + per_it * abs(full_iters)
    return {"value": 1.0 / t_solve, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": "oracle port, 1 thread: assembly + D-ILU setup + %d CG iterations on the "
                      "%d^3 Kuhn cube, solve extrapolated to %d iterations (%.3f s assembly, "
                      "%.4f s/iter)" % (iters, M + 1, abs(full_iters), t1 - t0, per_it),
            "host_cores": os.cpu_count()}


# --------------------------------------------------------- reference arm ----
def run_reference(args):
    from oracle import oracle as O
    from ofeli_b200 import fields
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    if args.workload == "meshfile2d":
        return run_reference_meshfile(args)
    nx = args.nx
    flavour = "ofast" if O.have_reference("ofast") else "o2"
    if not O.have_reference(flavour):
        print(json.dumps({"impl": "reference", "unavailable":
                          "oracle/_ref was not built (needs the reference sources)"}))
        return 0
    f = fields.uniform_pm1(SEED, (nx + 1) ** 2)
    nsteps = args.warmup + args.steps
    t0 = time.perf_counter()
    info, _ = O.run_reference(["bench2d", nx, "ILU", args.cpu_iters, nsteps], {"f": f},
                              flavour=flavour)
    wall = time.perf_counter() - t0
    ta = [float(v) for v in str(info["t_assembly_steps"]).split(",")][args.warmup:]
    tp = [float(v) for v in str(info["t_prec_steps"]).split(",")][args.warmup:]
    ti = [float(v) for v in str(info["t_iters_steps"]).split(",")][args.warmup:]
    full_iters = REF_ITERS_2049_ILU if (nx == 2048 and REF_ITERS_2049_ILU) else \
        int(round(1097 * (nx / 1024.0)))
    per_step = [a + p + i / args.cpu_iters * full_iters for a, p, i in zip(ta, tp, ti)]
    t_step = statistics.mean(per_step)
    value = 1.0 / t_step
    sample = ("OFELI (reference sources, -%s), 1 thread: per step Equation::build() + "
              "Prec(A, ILU_PREC) + %d CG iterations at %dx%d nodes, solve extrapolated to %d "
              "iterations; graph (SpMatrix(mesh)) %.1f s once, outside the steps"
              % ("Ofast" if flavour == "ofast" else "O2", args.cpu_iters, nx + 1, nx + 1,
                 full_iters, float(info["t_graph"])))
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": t_step * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "2-D P1 Poisson %dx%d nodes, CG + ILU (OFELI's diagonal ILU), "
                                   "tol 1e-10" % (nx + 1, nx + 1), "nodes": (nx + 1) ** 2,
                       "unknowns": int(info["n"]), "seed": SEED},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "kind": "reference",
                             "sample": sample, "host_cores": os.cpu_count()},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "wall_s": wall}
    pin = reference_full_run(nx)
    if pin:
        line["reference_full_run"] = pin
    print(json.dumps(line))
    return 0


def reference_full_run(nx):
    """OFELI's own CG + ILU on this problem run to convergence (the committed
    pin, measured where the reference was built: -O2, one core), beside the
    per-step model: the model's extrapolated solve against that measured
    one."""
    if nx != 2048:
        return None
    try:
        z = np.load(os.path.join(HERE, "tests", "golden", "p2d_2049_pins.npz"))
        info = json.loads(str(z["info"]))
    except (OSError, KeyError, ValueError):
        return None
    return {"source": "tests/golden/p2d_2049_pins.npz", "build": "-O2, 1 thread",
            "iterations": info["iters"], "graph_s": info["t_graph_cpu_o2_s"],
            "assembly_s": info["t_assembly_cpu_o2_s"], "solve_s": info["t_solve_cpu_o2_s"],
            "solve_s_per_iteration": info["t_solve_cpu_o2_s"] / info["iters"],
            "note": "measured to convergence once; the timed steps above are bounded samples "
                    "(build + Prec + a few iterations, -Ofast) extrapolated to this "
                    "iteration count"}


# --------------------------------------------------------------- our arm ----
def measure(args, wl, R, work_stream, dev, world, rank, with_cpu=True):
    """One workload (poisson2d or kuhn3d) through the chosen solver: warm-up,
    the timed device-resident steps, the kernel profile, the end-to-end
    steps, the plain FP64 CG + D-ILU solve and the error against it.
    Returns the JSON line (rank 0) or None."""
    import torch
    from ofeli_b200 import capi, fields
    from ofeli_b200 import ofeli as F
    local = dev.index
    nx = args.nx
    k_dev = None
    if wl == "kuhn3d":
        M = args.m3d
        mesh = F.Mesh.kuhn(M)
        coords, elem, _, _ = mesh.arrays()
        cent = coords.reshape(-1, 3)[elem.reshape(-1, 4)].mean(axis=1)
        k_host = fields.lognormal_k(SEED, cent, 1.5, 0.1, grid=256)
        del coords, elem, cent
        k_dev = torch.from_numpy(k_host).to(dev)
        workload = ("3-D P1 diffusion -div(k grad u) = f, Kuhn cube %d^3 nodes (%d tetrahedra), "
                    "k = exp(g), g Gaussian (sigma 1.5, corr. length 0.1), contrast %.1e"
                    % (M + 1, 6 * M ** 3, k_host.max() / k_host.min()))
    else:
        mesh = F.Mesh(0.0, 1.0, 0.0, 1.0, nx, nx, 1, 1, 1, 1)
        workload = "2-D P1 Poisson, %dx%d nodes" % (nx + 1, nx + 1)
    A = F.SpMatrix(mesh)
    n, nn = A.n, mesh.nn
    f_host = fields.uniform_pm1(SEED, nn)
    f_dev = torch.from_numpy(f_host).to(dev)
    b_dev = torch.zeros(n, dtype=torch.float64, device=dev)
    x_dev = torch.zeros(n, dtype=torch.float64, device=dev)
    u_dev = torch.zeros(nn, dtype=torch.float64, device=dev)
    P = F._ptr
    stream = work_stream
    PL, train_info, fell_back = None, None, []
    if args.prec == "learned":
        from ofeli_b200 import learned as LN
        net, train_info = LN.train_default(dim=3 if wl == "kuhn3d" else 2)
        capi.call("ofg_assemble_p1", mesh._h, A._h, P(k_dev), P(f_dev), None, P(b_dev))
        PL = F.Prec(A, F.LEARNED_PREC, net=net)

    def solve():
        if PL is not None:
            PL.setMatrix()  # the network runs on the newly assembled values
            o, i, r, fb = F.fcg_learned(PL, b_dev, x_dev, inner_bits=args.inner_bits, toler=TOL)
            fell_back.append(fb)
            return o, i, r
        return F.solve_mixed(A, b_dev, x_dev, prec=F.DIAG_PREC, inner_bits=args.inner_bits,
                             toler=TOL)

    def step_device():
        capi.call("ofg_assemble_p1", mesh._h, A._h, P(k_dev), P(f_dev), None, P(b_dev))
        x_dev.zero_()
        o, i, r = solve()
        capi.call("ofg_insert_bc", mesh._h, P(x_dev), None, P(u_dev))
        return o, i, r

    k_pin = k_dev.cpu().pin_memory() if k_dev is not None else None
    f_pin = torch.from_numpy(f_host).pin_memory()
    u_pin = torch.zeros(nn, dtype=torch.float64).pin_memory()

    def step_e2e():
        # public API with host buffers: f goes up, u comes back, every step
        capi.call("ofg_assemble_p1", mesh._h, A._h, P(k_pin), P(f_pin), None, P(b_dev))
        x_dev.zero_()
        o, i, r = solve()
        capi.call("ofg_insert_bc", mesh._h, P(x_dev), None, P(u_pin))
        return o, i, r

    barrier = R.barrier

    max_over_ranks = R.max

    for _ in range(args.warmup):
        step_device()
    torch.cuda.synchronize()

    # ------------------------------------------------ timed: device-resident
    launches0 = capi.launch_count()
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.4)
    barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    stats = []
    for _ in range(args.steps):
        stats.append(step_device())
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    ms = e0.elapsed_time(e1)
    clk = clocks.stop()
    launches = capi.launch_count() - launches0
    ms = max_over_ranks(ms)
    # the dominant kernel's launches timed with CUDA events on the library
    # stream (every 4th launch), over one more step of the same workload;
    # kept out of the timed steps so the events do not perturb them
    capi.profile_enable(4)
    step_device()
    torch.cuda.synchronize()
    prof = {k: capi.profile_read(k) for k in ("spmv32", "spmv16", "spmv64", "assembly",
                                              "network_gemm", "learned_apply")}
    capi.profile_enable(0)
    learned = None
    if PL is not None:
        # the network's forward pass alone (one per assembled matrix)
        for _ in range(2):
            PL.setMatrix()
        torch.cuda.synchronize()
        n0 = torch.cuda.Event(enable_timing=True)
        n1 = torch.cuda.Event(enable_timing=True)
        n0.record(stream)
        for _ in range(5):
            PL.setMatrix()
        n1.record(stream)
        torch.cuda.synchronize()
        net_ms = n0.elapsed_time(n1) / 5
        capi.profile_enable(1)
        PL.setMatrix()
        torch.cuda.synchronize()
        g_cnt, g_ms, g_bytes = capi.profile_read("network_gemm")
        capi.profile_enable(0)
        g_us = g_ms / max(g_cnt, 1) * 1e3
        g_flops = 2.0 * n * 128 * 64  # one layer product, [n x 128] x [128 x 64]
        a_cnt, a_ms, a_bytes = prof["learned_apply"]
        learned = dict(train_info)
        learned.update({
            "network_forward_ms": net_ms,
            "layer_gemm": {"kernel": "gemm_tc_tma (TMA-fed A tiles, two stages; tcgen05.mma kind::f16, BF16 -> FP32 in TMEM)",
                           "launches": g_cnt, "avg_us": g_us,
                           "GB/s": (g_bytes / max(g_cnt, 1)) / (g_us * 1e-6) / 1e9 if g_cnt else None,
                           "TFLOP/s": g_flops / (g_us * 1e-6) / 1e12 if g_cnt else None},
            "factor_apply": {"kernels": "lg_lower + lg_upper (FP32 SELL-32 products with G, G^T)",
                             "launches": a_cnt,
                             "avg_us": a_ms / max(a_cnt, 1) * 1e3,
                             "GB/s": (a_bytes / max(a_cnt, 1)) / (a_ms / max(a_cnt, 1) * 1e-3) / 1e9
                             if a_cnt else None},
            "fell_back_steps": int(sum(1 for f in fell_back if f)),
        })
    worst_res = max(s[2] for s in stats)
    if worst_res > TOL:
        raise SystemExit("solve missed the FP64 target: %.3e" % worst_res)

    # ------------------------------------------------ timed: end to end
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    g0 = torch.cuda.Event(enable_timing=True)
    g1 = torch.cuda.Event(enable_timing=True)
    g0.record(stream)
    e2e_stats = [step_e2e() for _ in range(args.steps)]
    g1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max(g0.elapsed_time(g1), (time.perf_counter() - t0) * 1e3)
    e2e_ms = max_over_ranks(e2e_ms)
    if max(s[2] for s in e2e_stats) > TOL:
        raise SystemExit("end-to-end solve missed the FP64 target")
    u_ref = u_dev.cpu().numpy()
    if not np.allclose(u_pin.numpy(), u_ref, rtol=0, atol=1e-12 * np.abs(u_ref).max()):
        raise SystemExit("end-to-end result differs from the device-resident one")
    x_chosen = x_dev.cpu().numpy()

    # ------------------------------------------------ plain FP64 CG + D-ILU
    plain, err_vs_fp64 = None, None
    if not args.no_plain and rank == 0:
        capi.call("ofg_assemble_p1", mesh._h, A._h, P(k_dev), P(f_dev), None, P(b_dev))
        Pc = F.Prec(A, F.ILU_PREC)
        x_dev.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        it = F.CG(A, Pc, b_dev, x_dev, 100000, TOL)
        torch.cuda.synchronize()
        t_plain = time.perf_counter() - t0
        plain = {"solver": "CG + ILU (OFELI's diagonal ILU), FP64, natural order",
                 "iterations": it, "solve_s": t_plain,
                 "true_rel_residual": F.residual(A, b_dev, x_dev)}
        x_plain = x_dev.cpu().numpy()
        err_vs_fp64 = {"value": float(np.linalg.norm(x_chosen - x_plain) /
                                      np.linalg.norm(x_plain)),
                       "what": "||x - x_fp64|| / ||x_fp64||, x_fp64 = the plain FP64 CG + ILU "
                               "solution (true rel. residual <= 1e-10)"}
        del Pc
    # SpMV FP64 bandwidth (the plain path's kernel), live CUDA events
    xs = torch.rand(n, dtype=torch.float64, device=dev)
    ys = torch.empty_like(xs)
    for _ in range(3):
        capi.call("ofg_spmv_device", A._h, 1, P(xs), P(ys))
    torch.cuda.synchronize()
    h0 = torch.cuda.Event(enable_timing=True)
    h1 = torch.cuda.Event(enable_timing=True)
    reps = 50
    h0.record(stream)
    for _ in range(reps):
        capi.call("ofg_spmv_device", A._h, 1, P(xs), P(ys))
    h1.record(stream)
    torch.cuda.synchronize()
    spmv64_us = h0.elapsed_time(h1) / reps * 1e3
    spmv64_bytes = 12.0 * A.nnz + 20.0 * n + 4.0

    if rank != 0:
        return None

    peak, peak_kind = measured_peaks()
    # the value format the solves streamed (inner_bits 0 decides per matrix)
    bits = 16 if prof["spmv16"][0] > prof["spmv32"][0] else 32
    fam = "spmv32" if bits == 32 else "spmv16"
    cnt, tot_ms, tot_bytes = prof[fam]
    avg_us = tot_ms / max(cnt, 1) * 1e3
    achieved = (tot_bytes / max(cnt, 1)) / (avg_us * 1e-6) / 1e9 if cnt else None
    # slices with uniform column offsets stream one offset per slice position
    # (the bytes per launch fall below value + 16-bit offset per entry)
    uniform = cnt and tot_bytes / cnt < ((4.0 if bits == 32 else 2.0) + 2.0) * A.nnz + 12.0 * n
    traffic = ncu_traffic(("mx_spmv_f32" if bits == 32 else "mx_spmv_bf16") +
                          ("_uniform" if uniform else ""))
    if wl != "poisson2d":
        traffic = None  # the committed capture is of the 2-D matrix
    cpu = None
    if world == 1 and wl == "poisson2d":
        cpu = cpu_baseline_port(nx, args.cpu_iters)
    elif world == 1 and plain and with_cpu:
        # extrapolated to the iteration count OFELI itself needs on this
        # problem (run to convergence with the reference, committed pin)
        cpu = cpu_baseline_port3d(args.m3d, args.cpu_iters,
                                  REF_ITERS_129_ILU if args.m3d == 128 else plain["iterations"])
    outer = sum(s[0] for s in stats) / len(stats)
    inner = sum(s[1] for s in stats) / len(stats)
    value = world * args.steps / (ms / 1e3)
    line = {
        "metric": METRIC if wl == "poisson2d" else METRIC_3D, "value": value,
        "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "f64 (refinement, residual, dots) / f32 (inner CG: SpMV, Jacobi, vectors)"
        if bits == 32 else "f64 (refinement, residual, dots) / f32 (inner CG: SpMV, vectors) "
        "with bf16 matrix values" + (" (lossless: every value of A is exact in bf16)"
                                     if args.inner_bits == 0 else ""),
        "data": "synthetic",
        "config": {"workload": "%s (%d unknowns, %d nonzeros), assembly + solve to FP64 "
                               "true rel. residual <= 1e-10" % (workload, n, A.nnz),
                   "solver": "FP64 refinement around FP32 Jacobi-PCG (direction kept)"
                   if PL is None else "FP64 refinement around FP32 CG with the learned "
                   "preconditioner M = G^T G (network run per assembled matrix, inside the step)",
                   "seed": SEED, "inputs_larger_than_l2": True,
                   "refinements_per_solve": outer, "inner_iterations_per_solve": inner},
        "gpu_launches": launches,
        "e2e": {"value": world * args.steps / (e2e_ms / 1e3), "unit": UNIT,
                "h2d_bytes_per_step": 8 * nn, "d2h_bytes_per_step": 8 * nn},
        "roofline": {"kernel": ("mx_spmv<float> (SELL-32 SpMV inside the FP32 CG"
                                if bits == 32 else "mx_spmv<bf16> (SELL-32 SpMV inside the FP32 "
                                "CG, bf16 values") +
                     (", uniform-slice column offsets)" if uniform else ")"),
                     "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": (achieved / peak) if achieved else None, "traffic": traffic,
                     "peak_source": peak_kind, "launches_timed": cnt,
                     "avg_launch_us": avg_us,
                     "bytes_per_launch": tot_bytes / max(cnt, 1)},
        "spmv_fp64": {"us": spmv64_us, "GB/s": spmv64_bytes / (spmv64_us * 1e-6) / 1e9,
                      "frac_of_peak": spmv64_bytes / (spmv64_us * 1e-6) / 1e9 / peak},
        "err_vs_fp64": err_vs_fp64,
        "plain": plain,
        "learned": learned,
        "cpu_baseline": cpu,
        "clocks": clk,
    }
    if plain:
        line["plain"]["solves_per_s"] = 1.0 / plain["solve_s"]
    return line


def run_ours(args):
    import torch
    from ofeli_b200 import capi, fields
    from ofeli_b200 import ofeli as F

    from ofeli_b200 import ranks
    world, rank, local = ranks.env()
    if not torch.cuda.is_available():
        raise SystemExit("bench.py needs a CUDA device")
    torch.cuda.set_device(local)
    R = ranks.Ranks("nccl", torch.device("cuda", local))
    L = capi.lib()
    # one stream for torch and the library: ordering without extra syncs
    work_stream = torch.cuda.Stream(device=torch.device("cuda", local))
    torch.cuda.set_stream(work_stream)
    capi.call("ofg_set_stream", ctypes.c_void_p(work_stream.cuda_stream))
    dev = torch.device("cuda", local)
    line = measure(args, args.workload, R, work_stream, dev, world, rank)
    if args.workload == "poisson2d" and not args.no_3d:
        # the 3-D variable-coefficient problem, in the same run: the chosen
        # form against the plain GPU CG + ILU, and its error against FP64
        import gc
        gc.collect()
        torch.cuda.empty_cache()
        l3 = measure(args, "kuhn3d", R, work_stream, dev, world, rank, with_cpu=False)
        if line is not None:
            pl = l3["plain"] or {}
            line["kuhn3d"] = {
                "workload": l3["config"]["workload"], "metric": l3["metric"],
                "value": l3["value"], "unit": l3["unit"], "ms_per_step": l3["ms_per_step"],
                "e2e": l3["e2e"], "solver": l3["config"]["solver"],
                "inner_iterations_per_solve": l3["config"]["inner_iterations_per_solve"],
                "refinements_per_solve": l3["config"]["refinements_per_solve"],
                "plain_ilu_cg": pl, "ofeli_ilu_cg_iterations": REF_ITERS_129_ILU,
                "ofeli_o2_measured_s": REF_TIMES_129_ILU,
                "ratio_vs_plain_gpu": (pl["solve_s"] * 1e3 / l3["ms_per_step"]) if pl else None,
                "err_vs_fp64": l3["err_vs_fp64"], "roofline": l3["roofline"],
                "gpu_launches": l3["gpu_launches"], "learned": l3["learned"],
                "clocks": l3["clocks"]}
    if line is not None:
        print(json.dumps(line))
    R.close()
    return 0


# ------------------------------------------------- batched workload -------
def batch_bytes(info, iters, nen=3, dim=2, bits=64):
    """Algorithmic bytes of one batched step: every problem's assembly
    (connectivity, coordinates, k, f, A and b written) plus, per CG + DIAG
    iteration, the minimum fused traffic -- FP64: 12 nnz + 108 n; FP32 inner
    iteration (FP32 value + 16-bit offset per entry): 6 nnz + 54 n, plus the
    FP32 value copy (12 nnz) once -- plus one true-residual SpMV in FP64
    (12 nnz + 24 n)."""
    nodes, elems, rows, nnz = (info[:, q].astype(np.float64) for q in range(4))
    asm = 4 * nen * elems + 8 * dim * nodes + 8 * elems + 8 * nodes + 8 * nnz + 8 * rows
    it = np.abs(iters).astype(np.float64)
    per_it = 12 * nnz + 108 * rows if bits == 64 else 6 * nnz + 54 * rows
    extra = 0 if bits == 64 else 12 * nnz
    return float((asm + extra + it * per_it + 12 * nnz + 24 * rows).sum())


def _batch_problem_inputs(nx, s):
    from oracle import oracle as O
    from ofeli_b200 import fields
    xy, elem, code = O.mesh2d(nx, nx)
    xy = fields.jitter_2d(s, xy, code, nx, nx, radius=0.3)
    cent = xy.reshape(-1, 2)[elem.reshape(-1, 3)].mean(axis=1)
    k = fields.lognormal_k(s, cent, 1.0, 0.1, grid=128)
    f = fields.uniform_pm1(s, code.size)
    dof, n = O.number_equations(code)
    rp, ci = O.node_graph(elem, 3, dof, n)
    return xy, elem, code, k, f, dof, n, rp, ci


def _batch_cpu_worker(jobs, barrier, out):
    """One single-threaded process of the parallel CPU baseline: builds the
    inputs of its problems (untimed), waits for the others, then assembles
    and solves them (CG + DIAG to 1e-10) and reports its start and end
    times and its work (nonzeros x iterations)."""
    from oracle import oracle as O
    data = [_batch_problem_inputs(nx, s) for nx, s in jobs]
    barrier.wait()
    t0 = time.time()
    work = 0.0
    for xy, elem, code, k, f, dof, n, rp, ci in data:
        a, b = O.assemble(2, xy, elem, dof, code, n, rp, ci, k=k, f=f)
        x, it = O.cg(rp, ci, a, b, O.DIAG, 100000, TOL)
        work += float(rp[-1]) * max(1, abs(it))
    out.put((t0, time.time(), work))


def cpu_parallel_batch(sizes, w_all, per_core=4):
    """N = host cores single-threaded oracle-port processes at once, each
    on its own problems of an evenly spaced sample of the batch (`per_core`
    per process on average, largest first to the least loaded process by
    the estimated cost nx^3, so that no process idles long); the batch
    extrapolated by the parallel wall time per (nonzeros x iterations) of
    the sample."""
    import multiprocessing as mp
    cores = os.cpu_count() or 1
    order = np.argsort(sizes)
    m = min(len(sizes), cores * per_core)
    pick = order[np.linspace(0, len(order) - 1, m).astype(int)]
    jobs = [[] for _ in range(cores)]
    load = [0.0] * cores
    for p in sorted(pick, key=lambda q: -int(sizes[q])):
        c = int(np.argmin(load))
        jobs[c].append((int(sizes[p]), SEED * 7919 + int(p)))
        load[c] += float(sizes[p]) ** 3
    ctx = mp.get_context("spawn")
    barrier = ctx.Barrier(cores)
    out = ctx.Queue()
    procs = [ctx.Process(target=_batch_cpu_worker, args=(j, barrier, out)) for j in jobs]
    for pr in procs:
        pr.start()
    res = [out.get(timeout=600) for _ in procs]
    for pr in procs:
        pr.join(timeout=60)
    wall = max(r[1] for r in res) - min(r[0] for r in res)
    w_sample = sum(r[2] for r in res)
    t_all = wall * w_all / w_sample
    return {"value": len(sizes) / t_all, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": "%d single-threaded oracle-port processes at once (one per host core), %d "
                      "problems of the batch (evenly spaced in size) assembled and solved with CG "
                      "+ DIAG to 1e-10 in %.2f s wall; the batch extrapolated by wall time per "
                      "(nonzeros x iterations) to %.1f s" % (cores, m, wall, t_all)}


def cpu_baseline_batch(sizes, iters, info, sample=16):
    """The oracle port (1 thread) on a bounded sample of the batch: every
    (count/sample)-th problem in size order, assembled and solved (CG + DIAG
    to 1e-10) in full; the whole batch extrapolated by the sample's time per
    (nonzeros x iterations)."""
    from oracle import oracle as O
    from ofeli_b200 import fields
    order = np.argsort(sizes)
    pick = order[np.linspace(0, len(order) - 1, sample).astype(int)]
    t_sample, w_sample = 0.0, 0.0
    for p in pick:
        nx = int(sizes[p])
        s = SEED * 7919 + int(p)
        xy, elem, code, k, f, dof, n, rp, ci = _batch_problem_inputs(nx, s)
        t0 = time.perf_counter()
        a, b = O.assemble(2, xy, elem, dof, code, n, rp, ci, k=k, f=f)
        x, it = O.cg(rp, ci, a, b, O.DIAG, 100000, TOL)
        t_sample += time.perf_counter() - t0
        w_sample += float(rp[-1]) * max(1, abs(it))
    w_all = float((info[:, 3].astype(np.float64) * np.maximum(1, np.abs(iters))).sum())
    t_all = t_sample * w_all / w_sample
    cores = os.cpu_count() or 1
    return {"value": len(sizes) / t_all, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": "oracle port, 1 thread: %d of the %d problems (evenly spaced in size) "
                      "assembled and solved with CG + DIAG to 1e-10 in %.2f s; the batch "
                      "extrapolated by time per (nonzeros x iterations) to %.1f s"
                      % (sample, len(sizes), t_sample, t_all),
            "host_cores": cores,
            "all_cores": cpu_parallel_batch(sizes, w_all)}


def run_batch(args):
    import torch
    from ofeli_b200 import capi, problems
    from ofeli_b200 import ofeli as F

    from ofeli_b200 import ranks
    world, rank, local = ranks.env()
    if not torch.cuda.is_available():
        raise SystemExit("bench.py needs a CUDA device")
    torch.cuda.set_device(local)
    R = ranks.Ranks("nccl", torch.device("cuda", local))
    work_stream = torch.cuda.Stream(device=torch.device("cuda", local))
    torch.cuda.set_stream(work_stream)
    capi.call("ofg_set_stream", ctypes.c_void_p(work_stream.cuda_stream))
    dev = torch.device("cuda", local)
    shard = args.shard and world > 1
    mine = None
    if shard:
        mine = problems.partition_by_cost(problems.batch_costs(SEED, args.nprob), world)[rank]
    meshes, k_host, f_host = problems.uneven_batch(SEED, count=args.nprob, indices=mine)
    sizes = problems.uneven_sizes(SEED, count=args.nprob)
    B = F.Batch(meshes)
    info = B.problem_info()
    k_dev = torch.from_numpy(k_host).to(dev)
    f_dev = torch.from_numpy(f_host).to(dev)
    B.set_inputs(k_dev, f_dev)
    B.set_precision(args.batch_bits)
    t0 = time.perf_counter()
    chosen, tune_ms = B.tune(100000, TOL)
    tune_s = time.perf_counter() - t0
    shape = F.Batch.config_shape(chosen)

    barrier = R.barrier

    max_over_ranks = R.max

    for _ in range(args.warmup):
        B.solve(100000, TOL)
    torch.cuda.synchronize()
    launches0 = capi.launch_count()
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.4)
    barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(work_stream)
    for _ in range(args.steps):
        B.solve(100000, TOL)
    e1.record(work_stream)
    torch.cuda.synchronize()
    barrier()
    ms = max_over_ranks(e0.elapsed_time(e1))
    clk = clocks.stop()
    launches = capi.launch_count() - launches0
    u_dev, iters, res = B.results()
    if res.max() > TOL or (iters < 0).any():
        raise SystemExit("batched solve missed the FP64 target: %.3e" % res.max())

    # end to end: k and f from pinned host memory, u back to pinned host
    k_pin = torch.from_numpy(k_host).pin_memory()
    f_pin = torch.from_numpy(f_host).pin_memory()
    u_pin = torch.zeros(B.nodes, dtype=torch.float64).pin_memory()
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    g0 = torch.cuda.Event(enable_timing=True)
    g1 = torch.cuda.Event(enable_timing=True)
    g0.record(work_stream)
    for _ in range(args.steps):
        B.set_inputs(k_pin, f_pin)
        B.solve(100000, TOL)
        capi.call("ofg_batch_get_results", B._h, F._ptr(u_pin), None, None)
    g1.record(work_stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(max(g0.elapsed_time(g1), (time.perf_counter() - t0) * 1e3))
    if not np.array_equal(u_pin.numpy(), u_dev):
        raise SystemExit("end-to-end result differs from the device-resident one")

    # the other inner precision, same launch shape
    other = None
    if rank == 0:
        ob = 64 if args.batch_bits == 32 else 32
        B.set_precision(ob)
        B.solve(100000, TOL)
        torch.cuda.synchronize()
        o0 = torch.cuda.Event(enable_timing=True)
        o1 = torch.cuda.Event(enable_timing=True)
        o0.record(work_stream)
        for _ in range(2):
            B.solve(100000, TOL)
        o1.record(work_stream)
        torch.cuda.synchronize()
        _, it_o, res_o = B.results()
        other = {"inner_bits": ob, "ms_per_step": o0.elapsed_time(o1) / 2,
                 "solves_per_s": 2 * B.nprob / (o0.elapsed_time(o1) / 1e3),
                 "iterations_mean": float(np.abs(it_o).mean()), "worst_true_rel_residual":
                 float(res_o.max())}
        B.set_precision(args.batch_bits)

    # the plain form: one problem after another through the single-problem
    # API (assembly + FP64 CG + DIAG per problem)
    plain = None
    if not args.no_plain and rank == 0:
        mats = [F.SpMatrix(m) for m in meshes]
        eoff = np.concatenate([[0], np.cumsum(info[:, 1])])
        noff = np.concatenate([[0], np.cumsum(info[:, 0])])
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        its = 0
        for p, (m, A) in enumerate(zip(meshes, mats)):
            b = torch.zeros(A.n, dtype=torch.float64, device=dev)
            capi.call("ofg_assemble_p1", m._h, A._h, F._ptr(k_dev[eoff[p]:eoff[p + 1]]),
                      F._ptr(f_dev[noff[p]:noff[p + 1]]), None, F._ptr(b))
            x = torch.zeros(A.n, dtype=torch.float64, device=dev)
            its += abs(F.CG(A, F.DIAG_PREC, b, x, 100000, TOL))
        torch.cuda.synchronize()
        t_plain = time.perf_counter() - t0
        plain = {"solver": "one problem at a time: ofg_assemble_p1 + CG + DIAG (FP64) per problem",
                 "solve_s": t_plain, "solves_per_s": len(meshes) / t_plain,
                 "iterations_total": int(its)}
        del mats

    if rank != 0:
        R.close()
        return 0
    peak, peak_kind = measured_peaks()
    nbytes = batch_bytes(info, iters, bits=args.batch_bits)
    achieved = nbytes / (ms / args.steps * 1e-3) / 1e9
    cpu = cpu_baseline_batch(sizes, iters, info) if world == 1 else None
    # problems solved per step by the whole job: the list once when sharded,
    # a replica of it per rank otherwise
    jobs = args.nprob if shard else world * B.nprob
    line = {
        "metric": METRIC_BATCH, "value": jobs * args.steps / (ms / 1e3),
        "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "strong" if shard else "weak",
        "vs_baseline": None,
        "dtype": "f64" if args.batch_bits == 64 else "f64 (assembly, refinement, true residual, "
                 "dots) / f32 (inner CG)", "data": "synthetic",
        "config": {"workload": "%d independent 2-D P1 diffusion problems, nodes log-uniform in "
                               "[1e3, 6.4e4] (%d nodes, %d unknowns, %d nonzeros in all), "
                               "jittered meshes, own lognormal k (sigma 1) and f each; assembly "
                               "+ CG + DIAG to FP64 true rel. residual <= 1e-10 + insertBC, all "
                               "in one persistent launch (CUDA graph)"
                               % (B.nprob, B.nodes, B.rows, B.nnz),
                   "seed": SEED, "inputs_larger_than_l2": True,
                   "launch_shape": {"threads_per_block": shape[0], "lanes_per_row": shape[1],
                                    "blocks_per_cluster": shape[2]},
                   "autotuner_ms": [round(float(t), 2) for t in tune_ms], "tune_s": tune_s,
                   "iterations": {"min": int(iters.min()), "mean": float(iters.mean()),
                                  "max": int(iters.max())}},
        "gpu_launches": launches,
        "e2e": {"value": jobs * args.steps / (e2e_ms / 1e3), "unit": UNIT,
                "h2d_bytes_per_step": 8 * (B.elements + B.nodes),
                "d2h_bytes_per_step": 8 * B.nodes},
        "roofline": {"kernel": "batch_kernel (assembly + CG + DIAG, every problem)",
                     "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": None, "peak_source": peak_kind,
                     "bytes_per_launch": nbytes, "avg_launch_us": ms / args.steps * 1e3},
        "plain": plain,
        "other_precision": other,
        "cpu_baseline": cpu,
        "clocks": clk,
    }
    print(json.dumps(line))
    R.close()
    return 0


# ------------------------------------------------- transient workload -----
T_NX, T_DT, T_EPS, T_M, T_TOL = 1024, 1e-3, 1e-3, 30, 1e-10


def transient_fields(xy, code):
    """u0 = Gaussian bump of width 0.05 at (0.3, 0.5), 0 on the boundary;
    v = (-(y - 0.5), x - 0.5) at the nodes."""
    P = xy.reshape(-1, 2)
    u0 = np.exp(-((P[:, 0] - 0.3) ** 2 + (P[:, 1] - 0.5) ** 2) / (2 * 0.05 ** 2))
    u0[code > 0] = 0.0
    v = np.stack([-(P[:, 1] - 0.5), P[:, 0] - 0.5], axis=1).reshape(-1)
    return u0, v


def cpu_baseline_transient(nsteps=2):
    """OFELI itself (reference sources, -Ofast) when it was built here, else
    the oracle port: `nsteps` backward-Euler steps at 1025^2 with GMRES(30) +
    ILU, graph construction once outside the steps."""
    from oracle import oracle as O
    xy, elem, code = O.mesh2d(T_NX, T_NX)
    u0, v = transient_fields(xy, code)
    flavour = "ofast" if O.have_reference("ofast") else ("o2" if O.have_reference("o2") else None)
    if flavour:
        info, _ = O.run_reference(["cd2d", T_NX, T_NX, nsteps, T_DT, T_EPS, "GMRES30", "ILU", T_TOL,
                                   2000], {"u0": u0, "v": v}, flavour=flavour)
        t_step = (float(info["t_assembly"]) + float(info["t_prec"]) + float(info["t_solve"])) / nsteps
        return {"value": 1.0 / t_step, "unit": "steps/s", "cores": 1, "kind": "reference",
                "sample": "OFELI (reference sources, -%s), 1 thread: %d DC2DT3 backward-Euler steps "
                          "(build() + Prec + GMRES(30), warm start, %d GMRES iterations in all); "
                          "graph %.1f s once, outside the steps"
                          % ("Ofast" if flavour == "ofast" else "O2", nsteps,
                             int(info["iters_total"]), float(info["t_graph"])),
                "host_cores": os.cpu_count()}
    dof, n = O.number_equations(code)
    rp, ci = O.node_graph(elem, 3, dof, n)
    u = u0.copy()
    x = np.zeros(n)
    t0 = time.perf_counter()
    its = 0
    for _ in range(nsteps):
        a, b = O.assemble_cd2d(xy, elem, dof, code, n, rp, ci, T_EPS, v, T_DT, u)
        x, it = O.gmres(rp, ci, a, b, O.ILU, T_M, 2000, T_TOL, x0=x)
        its += abs(it)
        u = O.insert_bc(code, x)
    t_step = (time.perf_counter() - t0) / nsteps
    return {"value": 1.0 / t_step, "unit": "steps/s", "cores": 1, "kind": "port",
            "sample": "oracle port, 1 thread: %d backward-Euler steps at 1025^2 (assembly + "
                      "D-ILU + GMRES(30), %d iterations)" % (nsteps, its),
            "host_cores": os.cpu_count()}


def run_transient(args):
    import torch
    from ofeli_b200 import capi
    from ofeli_b200 import ofeli as F

    from ofeli_b200 import ranks
    world, rank, local = ranks.env()
    if not torch.cuda.is_available():
        raise SystemExit("bench.py needs a CUDA device")
    torch.cuda.set_device(local)
    R = ranks.Ranks("nccl", torch.device("cuda", local))
    work_stream = torch.cuda.Stream(device=torch.device("cuda", local))
    torch.cuda.set_stream(work_stream)
    capi.call("ofg_set_stream", ctypes.c_void_p(work_stream.cuda_stream))
    dev = torch.device("cuda", local)
    P_ = F._ptr
    mesh = F.Mesh(0.0, 1.0, 0.0, 1.0, T_NX, T_NX, 1, 1, 1, 1)
    xy, _, code, _ = mesh.arrays()
    u0, v = transient_fields(xy, code)
    A = F.SpMatrix(mesh)
    n, nn = A.n, mesh.nn
    mixed = args.tprec in ("MIXED", "LEARNED")
    prec = {"ILU": F.ILU_PREC, "DIAG": F.DIAG_PREC, "MIXED": F.DIAG_PREC,
            "LEARNED": F.LEARNED_PREC}[args.tprec]
    net, train_info = None, None
    if args.tprec == "LEARNED":
        # trained before the timed region on smaller convection-diffusion
        # matrices with the workload's proportions (the library's kernels)
        from ofeli_b200 import learned as LN
        net, train_info = LN.train_transient()
    u_dev = torch.from_numpy(u0).to(dev)
    v_dev = torch.from_numpy(v).to(dev)
    b_dev = torch.zeros(n, dtype=torch.float64, device=dev)
    x_dev = torch.zeros(n, dtype=torch.float64, device=dev)
    Pc = None
    its = []
    cycles = []
    true_res = []

    def step(u_in, u_out):
        nonlocal Pc
        capi.call("ofg_assemble_cd2d", mesh._h, A._h, T_EPS, P_(v_dev), T_DT, P_(u_in), None,
                  P_(b_dev))
        if Pc is None:
            Pc = F.Prec(A, prec, net=net)
            if prec == F.LEARNED_PREC:
                # the matrix is the same at every step: the factor is computed
                # once, on the first step's matrix, and kept
                Pc.freeze()
        if mixed:
            # FP32 matrix values: the convection-diffusion values are not
            # exact in BF16 (the automatic format would check that every step)
            o, it, res, fb = F.fgmres_mixed(Pc, b_dev, x_dev, m=T_M, toler=T_TOL,
                                            inner_tol=args.t_inner_tol, inner_bits=32)
            if res > T_TOL or fb:
                raise SystemExit("a mixed FGMRES step missed the target: res %.3g fell_back %s"
                                 % (res, fb))
            cycles.append(o)
            true_res.append(res)
        else:
            it = F.GMRes(A, Pc, b_dev, x_dev, T_M, 2000, T_TOL)  # refactorises: values changed
        capi.call("ofg_insert_bc", mesh._h, P_(x_dev), None, P_(u_out))
        its.append(it)
        return it

    barrier = R.barrier

    for _ in range(args.warmup):
        step(u_dev, u_dev)
    torch.cuda.synchronize()
    del its[:]
    launches0 = capi.launch_count()
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.4)
    barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(work_stream)
    for _ in range(args.steps):
        step(u_dev, u_dev)
    e1.record(work_stream)
    torch.cuda.synchronize()
    barrier()
    ms = R.max(e0.elapsed_time(e1))
    clk = clocks.stop()
    launches = capi.launch_count() - launches0
    if any(i <= 0 for i in its):
        raise SystemExit("a GMRES solve did not converge: %s" % its)
    res = F.residual(A, b_dev, x_dev)
    timed_its = list(its)
    timed_cycles = list(cycles)
    # kernel families timed with CUDA events over two more steps (every 2nd
    # launch), kept out of the timed steps
    capi.profile_enable(2)
    for _ in range(2):
        step(u_dev, u_dev)
    torch.cuda.synchronize()
    families = ("sweep", "spmv64", "spmv32", "spmv16", "learned_apply", "gram_schmidt",
                "assembly")
    prof = {k: capi.profile_read(k) for k in families}
    capi.profile_enable(0)

    # end to end: the state u lives on the host (pinned) and goes up and
    # comes back every step
    u_pin = torch.from_numpy(u_dev.cpu().numpy()).pin_memory()
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    g0 = torch.cuda.Event(enable_timing=True)
    g1 = torch.cuda.Event(enable_timing=True)
    g0.record(work_stream)
    for _ in range(args.steps):
        step(u_pin, u_pin)
    g1.record(work_stream)
    torch.cuda.synchronize()
    e2e_ms = R.max(max(g0.elapsed_time(g1), (time.perf_counter() - t0) * 1e3))
    # the error of the timed form against the FP64 steps of OFELI's method:
    # 11 steps of each from the same initial state
    def trajectory(nsteps):
        u_dev.copy_(torch.from_numpy(u0).to(dev))
        x_dev.zero_()
        for _ in range(nsteps):
            step(u_dev, u_dev)
        torch.cuda.synchronize()
        return u_dev.cpu().numpy()

    u_timed = trajectory(11) if rank == 0 and not args.no_plain else None
    # the plain form (OFELI's GMRES(30) + ILU) over 10 steps from the same
    # initial state, and FP64 GMRES(30) + DIAG likewise
    plain, fp64_diag, err, learned_form = None, None, None, None

    def time_fp64(p, mixed_form=False):
        nonlocal prec, Pc, mixed
        prec, Pc, mixed = p, None, mixed_form
        u_dev.copy_(torch.from_numpy(u0).to(dev))
        x_dev.zero_()
        del its[:]
        step(u_dev, u_dev)  # factorisation plan and first step, untimed
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(10):
            step(u_dev, u_dev)
        torch.cuda.synchronize()
        t_pl = (time.perf_counter() - t0) / 10
        return {"ms_per_step": t_pl * 1e3, "steps_per_s": 1.0 / t_pl,
                "gmres_iterations_per_step": statistics.mean(its[1:]),
                "true_rel_residual": F.residual(A, b_dev, x_dev)}, u_dev.cpu().numpy()

    if rank == 0 and not args.no_plain:
        if args.tprec != "ILU":
            plain, u_ilu = time_fp64(F.ILU_PREC)
            plain["solver"] = "GMRES(30) + ILU (OFELI's diagonal ILU), FP64, warm start"
            err = float(np.linalg.norm(u_timed - u_ilu) / np.linalg.norm(u_ilu))
        if args.tprec != "DIAG":
            fp64_diag, _ = time_fp64(F.DIAG_PREC)
            fp64_diag["solver"] = "GMRES(30) + DIAG, FP64, warm start (OFELI's GMRes order)"
        if args.tprec != "LEARNED":
            # the learned preconditioner in the same mixed FGMRES (trained
            # here, outside any timed region; factor computed on the first
            # step's matrix and kept)
            from ofeli_b200 import learned as LN
            net, tinfo = LN.train_transient()
            learned_form, u_l = time_fp64(F.LEARNED_PREC, mixed_form=True)
            learned_form["solver"] = ("mixed-precision flexible GMRES(30) + learned M = G^T G, "
                                      "converged on the FP64 true residual")
            learned_form["training"] = tinfo
            learned_form["err_vs_fp64_ilu"] = (float(np.linalg.norm(u_l - u_ilu) /
                                                     np.linalg.norm(u_ilu))
                                               if plain else None)
    if rank != 0:
        R.close()
        return 0
    cpu = cpu_baseline_transient() if world == 1 else None
    peak, peak_kind = measured_peaks()
    fam = max((k for k in families if k != "assembly"), key=lambda k: prof[k][1])
    cnt, tot_ms, tot_bytes = prof[fam]
    avg_us = tot_ms / max(cnt, 1) * 1e3
    achieved = (tot_bytes / max(cnt, 1)) / (avg_us * 1e-6) / 1e9 if cnt else None
    shares = {k: round(prof[k][1], 3) for k in prof if prof[k][0]}
    kernel_names = {"sweep": "solve_sweep (D-ILU triangular sweeps)",
                    "spmv64": "spmv_sell_kernel (FP64 SELL-32 SpMV)",
                    "spmv32": "fg_product (FP32 SELL-32 product with A)",
                    "spmv16": "fg_product (BF16-value SELL-32 product with A)",
                    "learned_apply": "fg_product (products with G and G^T, BF16 values)",
                    "gram_schmidt": "fg_dots / fg_orth1 / fg_orth2 (FP64 classical "
                                    "Gram-Schmidt, twice)"}
    solver = {"ILU": "FP64 GMRES(30) + ILU (OFELI's GMRes, left preconditioned, MGS)",
              "DIAG": "FP64 GMRES(30) + DIAG (OFELI's GMRes, left preconditioned, MGS)",
              "MIXED": "mixed-precision flexible GMRES(30) + DIAG: FP32 products, FP64 CGS2 "
                       "and refinement, converged on the FP64 true residual",
              "LEARNED": "mixed-precision flexible GMRES(30) + learned M = G^T G (factor "
                         "computed on the first step's matrix and kept): FP32 products, BF16 "
                         "factor values, FP64 CGS2 and refinement, converged on the FP64 true "
                         "residual"}[args.tprec]
    line = {
        "metric": METRIC_TRANSIENT, "value": world * args.steps / (ms / 1e3), "unit": "steps/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "DC2DT3 on 1025x1025 nodes (%d unknowns, %d nonzeros): capacity + "
                               "diffusion eps 1e-3 + convection v = (-(y-0.5), x-0.5), u0 Gaussian "
                               "bump (0.3, 0.5) width 0.05, u = 0 on the boundary, backward Euler "
                               "dt 1e-3; per step build() + Prec + GMRES(30) warm-started to "
                               "OFELI's preconditioned residual 1e-10 + insertBC" % (n, A.nnz),
                   "preconditioner": args.tprec, "solver": solver,
                   "gmres_iterations_per_step": statistics.mean(timed_its),
                   "refinement_cycles_per_step": (statistics.mean(timed_cycles)
                                                  if timed_cycles else None),
                   "inner_tol": args.t_inner_tol if mixed else None,
                   "last_true_rel_residual": res, "inputs_larger_than_l2": True},
        "err_vs_fp64": {"value": err, "what": "||u - u_ref|| / ||u_ref|| after 11 steps from u0, "
                                              "u_ref = FP64 GMRES(30) + ILU (OFELI's method)"}
        if err is not None else None,
        "learned": train_info,
        "gpu_launches": launches,
        "e2e": {"value": world * args.steps / (e2e_ms / 1e3), "unit": "steps/s",
                "h2d_bytes_per_step": 8 * nn, "d2h_bytes_per_step": 8 * nn},
        "roofline": {"kernel": kernel_names[fam],
                     "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak if achieved else None, "traffic": None,
                     "peak_source": peak_kind, "launches_timed": cnt, "avg_launch_us": avg_us,
                     "bytes_per_launch": tot_bytes / max(cnt, 1),
                     "family_ms_sampled": shares},
        "plain": plain,
        "fp64_gmres_diag": fp64_diag,
        "learned_fgmres": learned_form,
        "cpu_baseline": cpu,
        "clocks": clk,
    }
    print(json.dumps(line))
    R.close()
    return 0


# ------------------------------------------------- mesh-file workload -----
MF_N = 1024          # annulus of MF_N + 1 circles of MF_N nodes, 2 MF_N^2 triangles
MF_SAMPLE = 512      # the same annulus at 512 for the reference's bounded CPU sample


def meshfile_write(nr, seed=SEED):
    """The annulus (random node numbering, random cell diagonals, jittered
    interior) written as an OFELI .m file by the library's own Mesh::put.
    Returns (path, node code, seconds spent in put)."""
    import tempfile
    from ofeli_b200 import ofeli as F
    from ofeli_b200 import problems
    xy, elem, code, sides, smark = problems.ring_mesh(nr, nr, seed=seed)
    mf = F.MeshFile.create(2, xy, code, elem, np.ones(elem.shape[0], np.int32), F.TRIANGLE,
                           sides=sides, side_code=smark)
    path = os.path.join(tempfile.mkdtemp(prefix="ofeli_meshfile_"), "annulus_%d.m" % nr)
    t0 = time.perf_counter()
    mf.put(path)
    return path, code, time.perf_counter() - t0


def meshfile_reference_sample(nsamples=1):
    """OFELI itself (reference sources, -Ofast, 1 thread) on the 512 annulus:
    Mesh(file, true) + SpMatrix(mesh) + build(), per sample."""
    from ofeli_b200 import fields
    from oracle import oracle as O
    flavour = "ofast" if O.have_reference("ofast") else ("o2" if O.have_reference("o2") else None)
    if not flavour:
        return None
    path, code, _ = meshfile_write(MF_SAMPLE)
    nn = code.size
    f = fields.uniform_pm1(SEED, nn)
    bc = np.where(code == 2, 1.0, 0.0)
    times = []
    for _ in range(nsamples):
        info, _ = O.run_reference(["mlap", path, "CG", "DIAG", 1e-10, 1], {"f": f, "bc": bc},
                                  flavour=flavour)
        times.append(float(info["t_mesh"]) + float(info["t_graph"]) + float(info["t_assembly"]))
    os.remove(path)
    return {"nodes": nn, "times": times, "flavour": flavour,
            "size_mb": None, "last": info}


def run_reference_meshfile(args):
    nsteps = args.warmup + args.steps
    t0 = time.perf_counter()
    r = meshfile_reference_sample(nsteps)
    if r is None:
        print(json.dumps({"impl": "reference", "unavailable":
                          "oracle/_ref was not built (needs the reference sources)"}))
        return 0
    t_step = statistics.mean(r["times"][args.warmup:])
    value = r["nodes"] / t_step
    info = r["last"]
    sample = ("OFELI (reference sources, -%s), 1 thread: Mesh(file, true) %.2f s + SpMatrix(mesh) "
              "%.2f s + build() %.2f s on the %d-node annulus file (the workload's mesh at "
              "%d x %d)" % ("Ofast" if r["flavour"] == "ofast" else "O2", float(info["t_mesh"]),
                            float(info["t_graph"]), float(info["t_assembly"]), r["nodes"],
                            MF_SAMPLE + 1, MF_SAMPLE))
    line = {"impl": "reference", "metric": METRIC_MESHFILE, "value": value, "unit": "nodes/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": t_step * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "OFELI .m file of a %d-node annulus, read + graph + P1 "
                                   "Laplace assembly" % r["nodes"]},
            "cpu_baseline": {"value": value, "unit": "nodes/s", "cores": 1, "kind": "reference",
                             "sample": sample, "host_cores": os.cpu_count()},
            "e2e": {"value": value, "unit": "nodes/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "wall_s": time.perf_counter() - t0}
    print(json.dumps(line))
    return 0


def run_meshfile(args):
    import torch
    from ofeli_b200 import capi, fields
    from ofeli_b200 import ofeli as F

    from ofeli_b200 import ranks
    world, rank, local = ranks.env()
    if not torch.cuda.is_available():
        raise SystemExit("bench.py needs a CUDA device")
    torch.cuda.set_device(local)
    R = ranks.Ranks("nccl", torch.device("cuda", local))
    work_stream = torch.cuda.Stream(device=torch.device("cuda", local))
    torch.cuda.set_stream(work_stream)
    capi.call("ofg_set_stream", ctypes.c_void_p(work_stream.cuda_stream))
    dev = torch.device("cuda", local)
    P_ = F._ptr
    path, code, t_put = meshfile_write(args.mf_n, seed=SEED + rank)
    size = os.path.getsize(path)
    mf0 = F.MeshFile(path)
    a0 = mf0.arrays()
    nn, ne = mf0.nn, mf0.ne
    f = fields.uniform_pm1(SEED, nn)
    bc = np.where(a0["node_code"][:, 0] == 2, 1.0, 0.0)
    m0 = mf0.to_mesh()
    n = m0.neq
    del m0, mf0
    # device-resident inputs of the device leg (the file's values, already parsed)
    d_xy = torch.from_numpy(np.ascontiguousarray(a0["coords"].ravel())).to(dev)
    d_el = torch.from_numpy(np.ascontiguousarray(a0["elem"].ravel())).to(dev)
    d_code = torch.from_numpy(np.ascontiguousarray(a0["node_code"][:, 0])).to(dev)
    d_f = torch.from_numpy(f).to(dev)
    d_bc = torch.from_numpy(bc).to(dev)
    d_b = torch.zeros(n, dtype=torch.float64, device=dev)
    f_pin = torch.from_numpy(f).pin_memory()
    bc_pin = torch.from_numpy(bc).pin_memory()
    b_pin = torch.zeros(n, dtype=torch.float64).pin_memory()
    nnz = [0]

    def step_device():
        h = ctypes.c_void_p()
        capi.call("ofg_mesh_create", 2, nn, P_(d_xy), ne, P_(d_el), P_(d_code), ctypes.byref(h))
        m = F.Mesh(_handle=h)
        A = F.SpMatrix(m)
        capi.call("ofg_assemble_p1", m._h, A._h, None, P_(d_f), P_(d_bc), P_(d_b))
        nnz[0] = A.nnz
        del A, m

    def step_e2e():
        m = F.Mesh.from_file(path)
        A = F.SpMatrix(m)
        capi.call("ofg_assemble_p1", m._h, A._h, None, P_(f_pin), P_(bc_pin), P_(b_pin))
        del A, m

    barrier = R.barrier

    def timed(fn, k):
        barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        t0 = time.perf_counter()
        e0.record(work_stream)
        for _ in range(k):
            fn()
        e1.record(work_stream)
        torch.cuda.synchronize()
        ms = max(e0.elapsed_time(e1), (time.perf_counter() - t0) * 1e3)
        barrier()
        return R.max(ms)

    for _ in range(args.warmup):
        step_device()
        step_e2e()
    torch.cuda.synchronize()
    launches0 = capi.launch_count()
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.4)
    ms = timed(step_device, args.steps)
    launches = capi.launch_count() - launches0
    e2e_ms = timed(step_e2e, args.steps)
    clk = clocks.stop()
    # the assembled system against the one assembled from the file read in
    # the e2e leg (same values: both gather in element order)
    same = bool(torch.equal(d_b.cpu(), b_pin))
    # phases of one e2e step, each closed by a synchronisation (untimed pass)
    ph = {}
    t0 = time.perf_counter()
    mf = F.MeshFile(path)
    ph["host_reader_s"] = time.perf_counter() - t0
    del mf
    t0 = time.perf_counter()
    m = F.Mesh.from_file(path)
    ph["device_reader_s"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    A = F.SpMatrix(m)
    torch.cuda.synchronize()
    ph["pattern_s"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    capi.call("ofg_assemble_p1", m._h, A._h, None, P_(d_f), P_(d_bc), P_(d_b))
    ph["assembly_s"] = time.perf_counter() - t0
    # the assembly kernel timed with CUDA events over 20 launches
    capi.profile_enable(1)
    for _ in range(20):
        capi.call("ofg_assemble_p1", m._h, A._h, None, P_(d_f), P_(d_bc), P_(d_b))
    torch.cuda.synchronize()
    cnt, tot_ms, tot_bytes = capi.profile_read("assembly")
    capi.profile_enable(0)
    del A, m
    os.remove(path)
    if rank != 0:
        R.close()
        return 0
    cpu = None
    if world == 1:
        r = meshfile_reference_sample(1)
        if r:
            info = r["last"]
            cpu = {"value": r["nodes"] / r["times"][0], "unit": "nodes/s", "cores": 1,
                   "kind": "reference",
                   "sample": "OFELI (reference sources, -%s), 1 thread: Mesh(file, true) %.2f s + "
                             "SpMatrix(mesh) %.2f s + build() %.2f s on the same annulus at "
                             "%d nodes" % ("Ofast" if r["flavour"] == "ofast" else "O2",
                                           float(info["t_mesh"]), float(info["t_graph"]),
                                           float(info["t_assembly"]), r["nodes"]),
                   "host_cores": os.cpu_count()}
    peak, peak_kind = measured_peaks()
    avg_us = tot_ms / max(cnt, 1) * 1e3
    achieved = (tot_bytes / max(cnt, 1)) / (avg_us * 1e-6) / 1e9 if cnt else None
    line = {
        "metric": METRIC_MESHFILE, "value": world * args.steps * nn / (ms / 1e3),
        "unit": "nodes/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "OFELI .m file (%.0f MB) of an annulus with %d nodes, %d triangles, "
                               "random node numbering; a step = Mesh::get + device mesh + "
                               "SpMatrix(mesh) pattern + Laplace2DT3 build() with f ~ U[-1,1] "
                               "and u = 1 on the outer circle (%d unknowns, %d nonzeros)"
                               % (size / 1e6, nn, ne, n, nnz[0]),
                   "value_leg": "mesh arrays already parsed and resident in HBM: device mesh + "
                                "pattern + assembly",
                   "e2e_leg": "the file (page cache) through Mesh.from_file "
                              "(ofg_mesh_read: staged to the device, tokenised and converted "
                              "there), SpMatrix(mesh) and ofg_assemble_p1 with host f, bc and b",
                   "host_threads": os.cpu_count(), "put_s": t_put,
                   "phases_one_step": ph, "device_and_file_rhs_equal": same,
                   "inputs_larger_than_l2": True},
        "gpu_launches": launches,
        "e2e": {"value": world * args.steps * nn / (e2e_ms / 1e3), "unit": "nodes/s",
                "h2d_bytes_per_step": size + 8 * 2 * nn, "d2h_bytes_per_step": 8 * n},
        "roofline": {"kernel": "assemble_rows<LaplaceT3> (row-gather P1 assembly)",
                     "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak if achieved else None, "traffic": None,
                     "peak_source": peak_kind, "launches_timed": cnt, "avg_launch_us": avg_us,
                     "bytes_per_launch": tot_bytes / max(cnt, 1)},
        "cpu_baseline": cpu,
        "clocks": clk,
    }
    print(json.dumps(line))
    R.close()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "batch2d":
        return run_batch(args)
    if args.workload == "transient2d":
        return run_transient(args)
    if args.workload == "meshfile2d":
        return run_meshfile(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
