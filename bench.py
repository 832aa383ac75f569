"""Benchmark: FV outer-iteration time and block-SpMV GB/s on one B200, FP64 and mixed precision.

Workload (the plain FP64 steady curved tube): a 90-degree arc tube of radius 2 mm on a bend of
radius 20 mm, a hexahedral O-grid core with five wedge wall layers graded toward the wall
(400,686 nodes, 501,600 elements, about 27 blocks per row), Carreau-Yasuda blood
(rho 1060, mu0 0.056, mu_inf 0.00345, lambda 3.313, a 2, n 0.3568), a parabolic 1 ml/s inlet,
a zero-pressure outlet, High Resolution advection. Synthetic: the mesh is generated, seeded.

A step is one outer iteration (assembly, boundary pass, AMG-FGMRES to 0.1, update, mass
flows, one read-back). ``value`` is outer iterations per second over the whole job (N
independent replicas for N > 1: the path does not shard across GPUs). The matrix (1.4 GB)
is larger than L2, so no flush is needed between steps.

``python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]``

Four further workloads print their own lines (``--workload bifurcation``: the ~2M-node
transient Y-bifurcation, mixed vs FP64 per BDF2 step; ``--workload ensemble``: 12 vessels
solved together vs one after another; ``--workload adjoint``: the adjoint gradient of the
~500k-node steady Y-bifurcation, checked against central differences; ``--workload smoothers``:
the AMG smoothers compared on the headline tube; ``--workload partitioned``: the partitioned
solve of 2 and 4 partitions sharing the GPU against the single-GPU solve on the headline tube);
the default is the headline above. ``--smoother chebyshev`` runs the headline with the Chebyshev smoother.
"""

from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "FV outer-iteration time & block-SpMV GB/s, mixed vs FP64 at 1e-8 rel. residual"
UNIT = "outer-iterations/s"
WORKLOAD = "curved Carreau-Yasuda tube, 400,686 nodes (hex core + 5 wedge wall layers), steady"
# DRAM bytes per algorithmic byte of one Gauss-Seidel pass on the finest level (the dominant
# kernel), from an ncu capture of a smaller tube whose matrix is larger than L2; None until
# captured. The traffic of the full pass is this ratio times its algorithmic bytes.
GS_TRAFFIC_PER_ALGORITHMIC_BYTE = None
GS_TRAFFIC_SOURCE = None


FULL_AXIAL = 285          # axial cells of the full 90-degree tube


def make_case(n_axial=FULL_AXIAL, same_cells=False):
    """The tube with ``n_axial`` cells over its 90-degree bend, or with ``same_cells`` a shorter
    arc of the full tube's cells (the bend angle scaled with ``n_axial``)."""
    from zvcfd_b200.fluid import CarreauYasuda, Fluid
    from zvcfd_b200.mesh import curved_tube

    R = 2e-3
    angle = np.pi / 2 * (n_axial / FULL_AXIAL if same_cells else 1.0)
    m = curved_tube(R, 20e-3, angle, n_core=20, n_ring=12, n_axial=n_axial, layers=5,
                    growth=0.8)
    z = {zz.name: k for k, zz in m.zones.items()}

    def shape(x):
        return np.clip(1.0 - (x[:, 0] ** 2 + x[:, 1] ** 2) / R ** 2, 0.0, None)

    bcs = {z["inlet"]: {"kind": "velocity", "flow_rate": 1e-6, "profile": shape},
           z["outlet"]: {"kind": "pressure", "value": 0.0}, z["wall"]: {"kind": "wall"}}
    return m, Fluid(1060.0, 0.00345, viscosity=CarreauYasuda()), bcs


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class Clocks:
    """nvidia-smi samples of the SM clock and throttle reasons during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-i", str(self.index)], stdout=subprocess.PIPE,
                stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [ln for ln in out.splitlines() if ln.strip()]

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in getattr(self, "lines", []):
            f = [v.strip() for v in ln.split(",")]
            try:
                sm.append(float(f[0]))
                mx.append(float(f[1]))
            except (ValueError, IndexError):
                continue
            for nm, v in zip(names, f[3:7]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(mx)),
                "samples": len(sm), "reasons": sorted(reasons)}


def spmv_roofline(solver, reps=20):
    """Time the FP64 and FP32 block-CSR SpMV on the assembled matrix with CUDA events."""
    import torch

    from zvcfd_b200._lib import call, ptr, stream_ptr

    A, _, _, _ = solver._assemble_fused()
    n, nnzb = A.n, A.nnzb
    lanes = 16
    x = torch.randn(n * 4, dtype=torch.float64, device="cuda")
    y = torch.empty_like(x)
    d32 = A.data.reshape(-1).float()
    x32, y32 = x.float(), torch.empty(n * 4, dtype=torch.float32, device="cuda")
    out = {}
    for name, fn, nbytes in (
            ("fp64", lambda: call("zvfv_bsr_spmv", n, ptr(A.indptr), ptr(A.indices), ptr(A.data),
                                  ptr(x), ptr(y), lanes, stream_ptr()),
             132 * nnzb + 72 * n + 8),
            ("fp32", lambda: call("zvfv_bsr_spmv_f32", n, ptr(A.indptr), ptr(A.indices),
                                  ptr(d32), ptr(x32), ptr(y32), lanes, stream_ptr()),
             68 * nnzb + 8 * (n + 1) + 32 * n)):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        t = e0.elapsed_time(e1) / 1e3 / reps
        out[name] = {"seconds": t, "bytes": nbytes, "gbs": nbytes / t / 1e9}
    return out, n, nnzb


def host_info() -> dict:
    """The host cores the CPU legs run on: count, model, thread settings."""
    model = ""
    try:
        for ln in open("/proc/cpuinfo"):
            if ln.startswith("model name"):
                model = ln.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    blas = None
    try:
        from threadpoolctl import threadpool_info

        blas = sum(int(d.get("num_threads", 0)) for d in threadpool_info()
                   if d.get("user_api") == "blas")
    except Exception:
        pass
    return {"nproc": os.cpu_count(), "model": model, "blas_threads": blas,
            "OMP_NUM_THREADS": os.environ.get("OMP_NUM_THREADS")}


class CpuCase:
    """The reference's CPU path for this workload, restated by the oracle: NumPy element assembly
    of the lagged Rhie-Chow system (``zvcfd/fv/reference.py:654-806``) and each linearisation
    solved by the reference's ACM inside FGMRES to ``linear_rtol`` 0.1 (``zvcfd/fv/linear.py:
    328-518``, its defaults: 2 block-Jacobi sweeps, omega 0.7, coarsest 400 rows, two pairwise
    passes, aggregates kept for 10 set-ups, restart 30), as SuperLU does not finish at this
    size. NumPy's element-wise and SciPy's sparse kernels run on one thread."""

    def __init__(self, n_axial=FULL_AXIAL):
        from oracle.fv import OracleSolver
        from oracle.linear import ACM, pairwise_arrays

        m, fl, bcs = make_case(n_axial, same_cells=True)
        self.n_nodes = m.n_nodes
        self.s = OracleSolver(m, fl, bcs)
        self.acm = ACM(coarse=400, matcher=pairwise_arrays, rebuild_every=10)
        self.linear_iterations = []

    def _linear(self, data, b, x0):
        from oracle.linear import fgmres

        A = self.s.system_matrix(data).tocsr()
        self.acm.setup(self.s.indptr, self.s.indices, data)
        x, its, _, _ = fgmres(lambda v: A @ v, b, x0, self.acm.vcycle, rtol=0.1, restart=30,
                              maxiter=200)
        self.linear_iterations.append(int(its))
        return x

    def step(self) -> float:
        t = time.perf_counter()
        self.s.solve(max_iterations=1, tol=0.0, linear=self._linear, resume=True)
        return time.perf_counter() - t


def cpu_spmv_gbs(indptr, indices, data, reps=3):
    import scipy.sparse as sp

    n = len(indptr) - 1
    M = sp.bsr_matrix((data.reshape(-1, 4, 4), indices, indptr), shape=(4 * n, 4 * n))
    x = np.random.default_rng(0).normal(size=4 * n)
    M @ x
    t = time.perf_counter()
    for _ in range(reps):
        M @ x
    t = (time.perf_counter() - t) / reps
    return (132 * len(indices) + 72 * n + 8) / t / 1e9


# the reference arm times at most this many full-size outer iterations (about 2 minutes each on
# one host core), after one untimed iteration that also builds the first aggregation
REFERENCE_MAX_STEPS = 2


def reference_arm(args, rank, world):
    """The reference's CPU path (the oracle's restatement, :class:`CpuCase`) on the full
    400,686-node tube on the host cores, rank 0 only: measured outer iterations, no scaling."""
    if rank != 0:
        return
    t0 = time.perf_counter()
    c = CpuCase(args.axial)
    setup = time.perf_counter() - t0
    warm = 1
    for _ in range(warm):
        c.step()
    steps = max(1, min(args.steps, REFERENCE_MAX_STEPS))
    times = [c.step() for _ in range(steps)]
    per = float(np.mean(times))
    value = 1.0 / per
    host = host_info()
    sample = (f"{steps} measured outer iterations of the full workload ({c.n_nodes:,} nodes) "
              f"after {warm} untimed (of {args.steps} and {args.warmup} requested: each takes "
              f"about two minutes on one core); NumPy assembly + ACM-FGMRES to 0.1; linear "
              f"iterations {c.linear_iterations}; solver set-up {setup:.1f} s untimed")
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": steps, "warmup": warm, "steps_requested": args.steps,
            "warmup_requested": args.warmup, "ms_per_step": per * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "impl": "reference",
            "config": {"workload": WORKLOAD, "nodes": c.n_nodes, "precision": "fp64",
                       "linear": "ACM-FGMRES (the reference's CPU AMG) to 0.1",
                       "l2": "inputs larger than L2"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "kind": "port",
                             "sample": sample, "host": host, "seconds": times},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def cpu_baseline_sample(n_axial=6, steps=2):
    """The bounded CPU sample of the default run (about 10-30 s): the reference arm's path on
    a short arc of the same tube (``n_axial`` of its cells, the same cell shapes), per outer
    iteration scaled linearly to the full node count (assembly and the ACM cycle are linear in
    the nodes; the iteration counts of the longer tube are not, so this is an estimate, the
    reference arm the measurement)."""
    c = CpuCase(n_axial)
    c.step()
    return float(np.mean([c.step() for _ in range(steps)])), c.n_nodes, c.linear_iterations


def bifurcation_workload(args):
    """The mixed-precision transient workload: a seeded-tet Y-bifurcation of about 2M nodes
    (parent radius 2 mm, daughters 1.6 and 1.4 mm at +-35 degrees, lengths 30/25/25 mm),
    Newtonian blood, inlet Q(t) = 1 + 0.5 sin(2 pi t / 0.8) ml/s, RCR outlets Rp 1e8, C 1e-9,
    Rd 1e9, BDF2 with dt 1e-3 and the reference's 5 coefficient loops per step. The FP32-
    hierarchy solver and the FP64 solver march the same steps from the same steady state; the
    field error of the mixed run against the FP64 run is reported at every step."""
    import torch

    from zvcfd_b200.fluid import Fluid
    from zvcfd_b200.lumped import RCR
    from zvcfd_b200.mesh import y_bifurcation
    from zvcfd_b200.solver import B200Solver

    h = 0.25e-3 * (56118.0 / args.nodes) ** (1.0 / 3.0)
    t0 = time.perf_counter()
    m = y_bifurcation(h, jitter_amount=0.05, seed=0)
    gen = time.perf_counter() - t0
    z = {zz.name: k for k, zz in m.zones.items()}

    def Q(t):
        return 1e-6 * (1.0 + 0.5 * np.sin(2 * np.pi * t / 0.8))

    def shape(x):
        return np.clip(1.0 - (x[:, 0] ** 2 + x[:, 1] ** 2) / 2e-3 ** 2, 0.0, None)

    def bcs():
        return {z["inlet"]: {"kind": "velocity", "flow_rate": Q, "profile": shape},
                z["outlet1"]: {"kind": "pressure", "lumped": RCR(rp=1e8, c=1e-9, rd=1e9)},
                z["outlet2"]: {"kind": "pressure", "lumped": RCR(rp=1e8, c=1e-9, rd=1e9)},
                z["wall"]: {"kind": "wall"}}

    fl = Fluid(1060.0, 3.5e-3)
    runs = {}
    for lin in ("b200", "b200-mixed"):
        s = B200Solver(m, fl, bcs(), linear=lin, linear_rtol=0.1)
        st = s.solve(max_iterations=400, tol=1e-8)
        steps = []
        for k in range(args.steps):
            torch.cuda.synchronize()
            t = time.perf_counter()
            rep = s.solve_transient(1e-3, 1, scheme="bdf2", loops=args.loops, tol=1e-8)
            torch.cuda.synchronize()
            last = rep["history"][-1]
            steps.append({"seconds": time.perf_counter() - t, "loops": rep["iterations"],
                          "converged": rep["converged"],
                          "loop_change": max(last["du"], last["dp"]),
                          "loop_rms": max(last[f"rms_{c}"] for c in "uvwp"),
                          "linear_iterations": sum(r["linear_iterations"] for r in rep["history"]),
                          "fields": s.fields(), "flows": s.patch_flows()})
        runs[lin] = {"steady_iterations": st["iterations"], "steps": steps}
        s.close()
    f64, mix = runs["b200"]["steps"], runs["b200-mixed"]["steps"]
    err = []
    for a, b in zip(f64, mix):
        err.append({k: float(np.linalg.norm(b["fields"][k] - a["fields"][k]) /
                             np.linalg.norm(a["fields"][k])) for k in ("U", "P")})
    t64 = float(np.mean([x["seconds"] for x in f64[1:] or f64]))
    tmx = float(np.mean([x["seconds"] for x in mix[1:] or mix]))
    line = {"metric": f"Y-bifurcation BDF2 time step ({args.loops} coefficient loops at most), "
                      "mixed vs FP64",
            "value": 1.0 / tmx, "unit": "time-steps/s", "n_gpus": 1, "steps": args.steps,
            "higher_is_better": True, "dtype": "f64 (FGMRES) / f32 (hierarchy)",
            "data": "synthetic",
            "config": {"workload": f"Y-bifurcation, {m.n_nodes:,} nodes, "
                                   f"{len(m.elements['tet']):,} seeded tets, lattice {h*1e3:.4f} mm",
                       "dt": 1e-3, "loops": args.loops, "mesh_seconds": gen},
            "fp64": {"seconds_per_step": t64, "steady_iterations": runs["b200"]["steady_iterations"],
                     "linear_iterations": [x["linear_iterations"] for x in f64]},
            "mixed": {"seconds_per_step": tmx, "speedup_vs_fp64": t64 / tmx,
                      "linear_iterations": [x["linear_iterations"] for x in mix],
                      "field_error_vs_fp64_per_step": err,
                      "max_field_error_vs_fp64": {k: max(e[k] for e in err) for k in ("U", "P")}},
            "loops_per_step": {"fp64": [x["loops"] for x in f64], "mixed": [x["loops"] for x in mix]},
            "last_loop_change_per_step": {"fp64": [x["loop_change"] for x in f64],
                                          "mixed": [x["loop_change"] for x in mix]},
            "last_loop_rms_residual_per_step": {"fp64": [x["loop_rms"] for x in f64],
                                                "mixed": [x["loop_rms"] for x in mix]},
            "steps_converged_to_1e-8": {"fp64": sum(x["converged"] for x in f64),
                                        "mixed": sum(x["converged"] for x in mix)},
            "outlet_flows_ml_s": [{str(k): v * 1e6 for k, v in x["flows"].items()} for x in mix]}
    print(json.dumps(line), flush=True)


def ensemble_workload(args):
    """The batched-ensemble workload: 12 seeded vessels of log-uniform sizes in 50k-1.2M nodes
    (straight, curved, bifurcating in turn), random inlet flows and RCR outlets, steady to
    1e-8; the instances solved one after another in plain FP64 against all of them solved
    together with the FP32 hierarchy and the lanes autotuner."""
    import torch

    from zvcfd_b200.ensemble import B200Ensemble, solve_sequentially, synthetic_ensemble
    from zvcfd_b200.fluid import Fluid

    def log(msg):
        print(msg, file=sys.stderr, flush=True)

    t0 = time.perf_counter()
    cases = synthetic_ensemble(count=args.instances, high=args.max_nodes, seed=0)
    gen = time.perf_counter() - t0
    log(f"{len(cases)} meshes generated in {gen:.1f} s")
    fl = Fluid(1060.0, 3.5e-3)
    torch.cuda.synchronize()
    seq = solve_sequentially(cases, fl, tol=1e-8, max_iterations=400, linear="b200", log=log)
    torch.cuda.synchronize()
    t = time.perf_counter()
    ens = B200Ensemble(cases, fl, krylov=args.krylov, linear="b200-mixed",
                       linear_options={"autotune": True})
    log(f"ensemble set up in {time.perf_counter() - t:.1f} s")
    rep = ens.solve(tol=1e-8, max_iterations=400, log=log)
    torch.cuda.synchronize()
    t_ens = time.perf_counter() - t
    err = []
    for i, r in enumerate(seq["instances"]):
        f = ens.fields(i)
        err.append(max(float(np.linalg.norm(f[k] - r["fields"][k]) / np.linalg.norm(r["fields"][k]))
                       for k in ("U", "P")))
    ens.close()
    sizes = [m.n_nodes for m, _ in cases]
    line = {"metric": "batched ensemble solves/s vs sequential FP64", "value": len(cases) / t_ens,
            "unit": "solves/s", "n_gpus": 1, "higher_is_better": True, "data": "synthetic",
            "dtype": "f64 (FGMRES) / f32 (hierarchy)",
            "config": {"workload": f"{len(cases)} vessels, {sum(sizes):,} nodes in all",
                       "nodes": sizes, "tol": 1e-8, "krylov": args.krylov,
                       "mesh_seconds": gen},
            "sequential_fp64": {"value": len(cases) / seq["seconds"], "seconds": seq["seconds"],
                                "outer_iterations": [r["iterations"] for r in seq["instances"]],
                                "converged": all(r["converged"] for r in seq["instances"])},
            "batched_mixed": {"seconds": t_ens, "outer_iterations": rep["iterations"],
                              "converged": rep["converged"],
                              "first_converged": [int(x) for x in rep["first_converged"]],
                              "field_error_vs_sequential": err},
            "speedup": seq["seconds"] / t_ens}
    print(json.dumps(line), flush=True)


def smoothers_workload(args):
    """The AMG smoothers compared on the headline tube: per configuration (precision,
    smoother, degree or sweeps), the mean outer-iteration time and Krylov steps of iterations
    4-11, one V-cycle and one finest-level smoothing pass (CUDA events), the spectral estimate
    of the Chebyshev smoother, and the steady solve to 1e-8 from scratch. One JSON line per
    configuration."""
    import ctypes

    import torch

    from zvcfd_b200._lib import call, stream_ptr
    from zvcfd_b200.solver import B200Solver

    m, fl, bcs = make_case(args.axial)
    cheb = {"smoother": "chebyshev", "presweeps": 2, "postsweeps": 2}
    runs = [("b200", {"smoother": "gs"}), ("b200", cheb),
            ("b200", {"smoother": "chebyshev", "presweeps": 3, "postsweeps": 3}),
            ("b200", {"smoother": "dilu"}), ("b200", {"smoother": "ilu0"}),
            ("b200-mixed", {"smoother": "gs"}), ("b200-mixed", cheb),
            ("b200-mixed", {"smoother": "dilu"})]
    for lin, opts in runs:
        s = B200Solver(m, fl, bcs, linear=lin, linear_rtol=0.1, linear_options=opts)
        for _ in range(3):
            s.iterate()
        torch.cuda.synchronize()
        t = time.perf_counter()
        its = [s.iterate()["linear_iterations"] for _ in range(8)]
        torch.cuda.synchronize()
        per = (time.perf_counter() - t) / 8
        A, b, _, x0 = s._assemble_fused()
        s.linear.setup(A)
        r = b.reshape(-1) - A.matvec(x0)
        tv = event_time(lambda: s.linear.vcycle(r), reps=10)
        tp = event_time(lambda: call("zvfv_solver_smooth", s.linear._h, 0, 1, stream_ptr()),
                        reps=10)
        lmax = None
        if opts["smoother"] == "chebyshev":
            v = ctypes.c_double()
            call("zvfv_solver_get_option", s.linear._h, b"cheb_lmax", ctypes.byref(v))
            lmax = v.value
        s.close()
        s2 = B200Solver(m, fl, bcs, linear=lin, linear_rtol=0.1, linear_options=opts)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        rep = s2.solve(max_iterations=80, tol=1e-8)
        torch.cuda.synchronize()
        s2.close()
        print(json.dumps({"workload": WORKLOAD, "linear": lin, **opts,
                          "ms_per_outer_iteration": per * 1e3, "krylov_steps": its,
                          "vcycle_ms": tv * 1e3, "finest_pass_ms": tp * 1e3,
                          "cheb_lmax": lmax, "to_1e-8_s": time.perf_counter() - t0,
                          "outer_iterations": rep["iterations"],
                          "converged": rep["converged"]}), flush=True)


def partitioned_workload(args):
    """The partitioned solve (partitions sharing this GPU, the reference's own test setting)
    against the single-GPU solve on the headline tube: per partition count (0 is the single-GPU
    solver, with the partitioned solver's aggregate rebuild every 10 set-ups), the set-up time,
    the partition report, the mean outer-iteration time and Krylov steps of iterations 4-11
    (host clock around synchronised iterations), and the steady solve to 1e-8 from scratch with
    its relative L2 field difference from the single-GPU solve. One JSON line per count."""
    import torch

    from zvcfd_b200.multi import B200MultiSolver
    from zvcfd_b200.solver import B200Solver

    m, fl, bcs = make_case(args.axial)
    single = None
    for parts in [0] + [int(p) for p in args.parts.split(",") if p]:
        def build():
            if parts == 0:
                return B200Solver(m, fl, bcs, linear="b200", linear_rtol=0.1,
                                  linear_options={"rebuild_every": 10})
            return B200MultiSolver(m, fl, bcs, parts=parts, linear="b200", linear_rtol=0.1)

        t0 = time.perf_counter()
        s = build()
        torch.cuda.synchronize()
        setup = time.perf_counter() - t0
        report = getattr(s, "report", None)
        for _ in range(3):
            s.iterate()
        torch.cuda.synchronize()
        t = time.perf_counter()
        its = [s.iterate()["linear_iterations"] for _ in range(8)]
        torch.cuda.synchronize()
        per = (time.perf_counter() - t) / 8
        s.close()
        s2 = build()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        rep = s2.solve(max_iterations=150, tol=1e-8)
        torch.cuda.synchronize()
        to_tol = time.perf_counter() - t0
        f = s2.fields()
        s2.close()
        if single is None:
            single = f
        err = {k: float(np.linalg.norm(f[k] - single[k]) / np.linalg.norm(single[k]))
               for k in ("U", "P")}
        print(json.dumps({"workload": WORKLOAD, "parts": parts, "setup_s": setup,
                          "report": report, "ms_per_outer_iteration": per * 1e3,
                          "krylov_steps": its, "to_1e-8_s": to_tol,
                          "outer_iterations": rep["iterations"], "converged": rep["converged"],
                          "field_rel_l2_vs_single": err}), flush=True)


def adjoint_workload(args):
    """The adjoint workload: the Y-bifurcation coarsened to about 500k nodes, steady,
    Carreau-Yasuda blood, a 1 ml/s inlet and RCR outlets (Rp 1e8, C 1e-9, Rd 1e9), a fixed
    advection blend. Objectives: the two outlet flow fractions and the mean wall shear stress on
    each daughter's wall beyond the junction; parameters: the inlet flow, each outlet's
    (Rp, C, Rd) and mu0. Timed: the forward solve to round-off and the adjoint gradient (one
    FGMRES solve per objective on the transposed Jacobian, preconditioned by the forward
    hierarchy's transposed V-cycle). Checked: central differences (step 1e-6 relative) of
    converged solves restarted from the solved state, for every parameter."""
    import torch

    from zvcfd_b200.fluid import CarreauYasuda, Fluid
    from zvcfd_b200.lumped import RCR
    from zvcfd_b200.mesh import y_bifurcation
    from zvcfd_b200.sensitivity import SteadyResidual
    from zvcfd_b200.solver import B200Solver

    def log(msg):
        print(msg, file=sys.stderr, flush=True)

    names = ["Q_in", "Rp1", "C1", "Rd1", "Rp2", "C2", "Rd2", "mu0"]
    theta0 = np.array([1e-6, 1e8, 1e-9, 1e9, 1e8, 1e-9, 1e9, 0.056])
    h = 0.25e-3 * (56118.0 / args.adjoint_nodes) ** (1.0 / 3.0)
    t0 = time.perf_counter()
    m = y_bifurcation(h, jitter_amount=0.05, seed=0)
    gen = time.perf_counter() - t0
    z = {zz.name: k for k, zz in m.zones.items()}
    f = m.zones[z["wall"]].faces
    wn = np.unique(f[f >= 0])
    xw = m.nodes[wn]
    beyond = xw[:, 2] > 2.5e-3
    walls = {"daughter1": torch.as_tensor(wn[beyond & (xw[:, 0] > 0)], device="cuda"),
             "daughter2": torch.as_tensor(wn[beyond & (xw[:, 0] < 0)], device="cuda")}

    def shape(x):
        return np.clip(1.0 - (x[:, 0] ** 2 + x[:, 1] ** 2) / 2e-3 ** 2, 0.0, None)

    def solve(theta, start=None):
        q, rp1, c1, rd1, rp2, c2, rd2, mu0 = (float(v) for v in theta)
        bcs = {z["inlet"]: {"kind": "velocity", "flow_rate": q, "profile": shape},
               z["outlet1"]: {"kind": "pressure", "lumped": RCR(rp=rp1, c=c1, rd=rd1)},
               z["outlet2"]: {"kind": "pressure", "lumped": RCR(rp=rp2, c=c2, rd=rd2)},
               z["wall"]: {"kind": "wall"}}
        fl = Fluid(1060.0, 0.00345, viscosity=CarreauYasuda(mu_0=mu0))
        s = B200Solver(m, fl, bcs, advection=1.0, linear_rtol=0.1)
        if start is not None:
            s.initialise(U=start[0], P=start[1])
        torch.cuda.synchronize()
        t = time.perf_counter()
        count = [0]

        def every(msg):                      # one line in a hundred of the solve's log
            count[0] += 1
            if count[0] % 100 == 0:
                log(msg)

        rep = s.solve(max_iterations=args.adjoint_iterations, tol=args.adjoint_tol, log=every)
        torch.cuda.synchronize()
        return s, rep, time.perf_counter() - t

    log(f"mesh: {m.n_nodes:,} nodes in {gen:.1f} s")
    s, rep, t_fwd = solve(theta0)
    log(f"forward: {rep['iterations']} outer iterations, {t_fwd:.1f} s, converged {rep['converged']}")
    res = SteadyResidual(s, z["inlet"], [z["outlet1"], z["outlet2"]], walls)
    torch.cuda.synchronize()
    t = time.perf_counter()
    grad, J, info = res.sensitivities(rtol=args.adjoint_rtol, restart=args.adjoint_restart)
    torch.cuda.synchronize()
    t_adj = time.perf_counter() - t
    grad, J = grad.cpu().numpy(), J.cpu().numpy()
    log(f"adjoint: {t_adj:.1f} s, {info}")
    start = (s.U.cpu().numpy(), s.P.cpu().numpy())
    peak_gb = torch.cuda.max_memory_allocated() / 1e9
    s.close()
    del res
    fd = np.full_like(grad, np.nan)
    fd_solves = []
    checked = [names.index(x) for x in args.adjoint_fd.split(",")] if args.adjoint_fd \
        else list(range(len(theta0)))
    for p in checked:
        step = 1e-6 * theta0[p]
        vals = []
        for sgn in (1.0, -1.0):
            th = theta0.copy()
            th[p] += sgn * step
            sp, rp, tp = solve(th, start)
            r2 = SteadyResidual(sp, z["inlet"], [z["outlet1"], z["outlet2"]], walls)
            x2, m2 = r2.state()
            vals.append(r2.objectives(x2, m2, r2.theta0()).cpu().numpy())
            fd_solves.append({"iterations": rp["iterations"], "converged": rp["converged"],
                              "seconds": tp})
            sp.close()
            del r2
        fd[:, p] = (vals[0] - vals[1]) / (2 * step)
        log(f"fd {names[p]} done")
    objectives = ["Q1/Q_in", "Q2/Q_in", "WSS daughter1", "WSS daughter2"]
    err = []
    for k in range(grad.shape[0]):
        ref = np.abs(fd[k, checked] * theta0[checked]).max()
        err.append(float(np.abs((grad[k, checked] - fd[k, checked]) * theta0[checked]).max()
                         / ref))
    line = {"metric": "steady adjoint gradient (4 objectives x 8 parameters) vs central differences",
            "value": 1.0 / t_adj, "unit": "gradients/s", "n_gpus": 1, "higher_is_better": True,
            "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"Y-bifurcation, {m.n_nodes:,} nodes, "
                                   f"{len(m.elements['tet']):,} seeded tets, Carreau-Yasuda, steady",
                       "lattice_mm": h * 1e3, "forward_tol": args.adjoint_tol,
                       "adjoint_rtol": args.adjoint_rtol, "restart": args.adjoint_restart,
                       "fd_step": "1e-6 relative", "mesh_seconds": gen},
            "forward": {"seconds": t_fwd, "outer_iterations": rep["iterations"],
                        "converged": rep["converged"]},
            "adjoint": {"seconds": t_adj, "seconds_per_objective": t_adj / len(objectives),
                        "adjoint_vs_forward": t_adj / t_fwd,
                        "krylov": [{"objective": o, **i} for o, i in zip(objectives, info)],
                        "peak_device_gb": peak_gb},
            "objectives": dict(zip(objectives, J.tolist())),
            "gradient": {o: dict(zip(names, g.tolist())) for o, g in zip(objectives, grad)},
            "central_differences": {o: {names[p]: float(g[p]) for p in checked}
                                    for o, g in zip(objectives, fd)},
            "fd_parameters": [names[p] for p in checked],
            "max_error_vs_fd_relative_to_largest_sensitivity": dict(zip(objectives, err)),
            "capacitance_gradients_zero": bool(np.all(grad[:, [2, 5]] == 0.0)),
            "fd_solves": fd_solves}
    print(json.dumps(line), flush=True)


def max_over_ranks(value, dist, device):
    """The largest of every rank's ``value`` (the job's time is its slowest replica's)."""
    import torch

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def run_steps(solver, steps):
    import torch

    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    recs = [solver.iterate() for _ in range(steps)]
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / 1e3, recs


def event_time(fn, reps=5):
    """Mean seconds of ``fn`` on the current stream (CUDA events), after one untimed call."""
    import torch

    fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / 1e3 / reps


# ---------------------------------------------------------------- algorithmic bytes

def spmv_bytes(n, nnz, value_bytes=8, vec_bytes=8):
    """Block-CSR product: blocks, column indices, row pointers, x read once, y written."""
    return (16 * value_bytes + 4) * nnz + 8 * (n + 1) + 2 * 4 * vec_bytes * n


def gs_pass_bytes(n, nnz, value_bytes=8, vec_bytes=8):
    """One Gauss-Seidel pass over all colours of a level: the level's blocks, indices and row
    pointers once, each row's 4x4 inverse, b read, x read and written."""
    return (16 * value_bytes + 4) * nnz + 8 * (n + 1) + 16 * value_bytes * n + 3 * 4 * vec_bytes * n


def cheb_step_bytes(n, nnz, value_bytes=8, vec_bytes=8):
    """One Chebyshev step on a level: the level's blocks, indices and row pointers once, each
    row's 4x4 inverse, b and x_in read, the update read and written, x_out written."""
    return (16 * value_bytes + 4) * nnz + 8 * (n + 1) + 16 * value_bytes * n + 5 * 4 * vec_bytes * n


def vcycle_bytes(stats, value_bytes=8, gs_levels=2, gs_passes=6, jacobi_sweeps=4,
                 coarse_sweeps=8, smoother="gs", cheb_steps=4):
    """Algorithmic bytes of one V-cycle over the hierarchy ``stats`` (rows and blocks per
    level): Gauss-Seidel passes on the finest ``gs_levels`` (pre 1 + post 2 symmetric sweeps),
    damped Jacobi sweeps below, the residual product, restriction and prolongation of each
    level, and the permutations in and out of a Gauss-Seidel level's colour order; with the
    Chebyshev smoother ``cheb_steps`` steps (pre + post degree) on every level instead."""
    vb = value_bytes
    total = 0
    rows, blocks = stats["levels"], stats["blocks"]
    for i, (n, nnz) in enumerate(zip(rows, blocks)):
        last = i + 1 == len(rows)
        vec = 4 * vb * n
        if last and n <= 24:
            total += 16 * n * n * vb + 2 * vec            # dense inverse times the vector
            continue
        if smoother == "chebyshev":
            total += (coarse_sweeps if last else cheb_steps) * cheb_step_bytes(n, nnz, vb, vb)
        elif i < gs_levels:
            total += gs_passes * gs_pass_bytes(n, nnz, vb, vb) + 4 * vec
        else:
            sweeps = coarse_sweeps if last else jacobi_sweeps
            total += sweeps * (spmv_bytes(n, nnz, vb, vb) + 16 * vb * n + 2 * vec)
        if not last:
            total += spmv_bytes(n, nnz, vb, vb) + 3 * vec + 4 * n   # residual, restrict, prolong
    return total


def element_bytes(asm) -> dict:
    """Algorithmic bytes of the element stage (the ideal of one pass over the data): the matrix
    written once (128 B per block), b (32 B per node), the node values read once (188 B per node:
    X 24, U 24, grad U 72, grad p 24, beta 24, d 8, s 8, own 4), and per element its
    connectivity, mass flows and block positions. The colour-ordered scatter reads and writes
    each element's n^2 blocks instead (``scatter``)."""
    N, nnzb = asm.N, asm.nnzb
    per_elem = sum(K.E * (4 * K.n + 8 * K.nip + 4 * K.n * K.n) for K in asm.kinds)
    assemble = 128 * nnzb + 32 * N + 188 * N + per_elem
    scatter = sum(K.E * K.n * K.n * 256 for K in asm.kinds)
    # mass flows: X, U, grad p, P, d, s per node; mdot written; outflow, adv, vdiag
    massflow = N * (24 + 24 + 24 + 8 + 8 + 8 + 24) + sum(K.E * (4 * K.n + 8 * K.nip)
                                                         for K in asm.kinds)
    return {"assemble": assemble, "assemble_scatter": scatter, "massflow": massflow}


def stage_times(solver, peak, value_bytes=8, smoother="gs"):
    """CUDA-event times and HBM fractions of the outer iteration's stages on the solver's
    current state, and the smoother's pass on the finest level (the dominant kernel) alone:
    one Gauss-Seidel pass over all colours, or one Chebyshev step; ``value_bytes`` is the
    hierarchy's value size (8 FP64, 4 for the FP32 hierarchy)."""
    import torch

    from zvcfd_b200._lib import call, ptr, stream_ptr

    asm = solver.asm
    gradU, gradP, beta, diag = solver._stage1()
    dnode, snode = solver.Vd / diag, solver.Vd / diag
    own = solver._own_inflow()
    vd = torch.zeros(solver.N, dtype=torch.float64, device="cuda")
    mcopy = {k: v.clone() for k, v in solver.mdot.items()}
    eb = element_bytes(asm)
    out = {}
    t = event_time(lambda: asm.assemble(solver.U, solver.mdot, gradU, beta, gradP, dnode, snode,
                                        own=own))
    out["assemble"] = {"ms": t * 1e3, "algorithmic_bytes": eb["assemble"],
                       "frac": eb["assemble"] / t / 1e9 / peak,
                       "scatter_bytes": eb["assemble_scatter"],
                       "scatter_frac": eb["assemble_scatter"] / t / 1e9 / peak}
    t = event_time(lambda: asm.massflow(solver.U, solver.P, gradP, dnode, snode, out=mcopy,
                                        vdiag=vd))
    out["massflow_vdiag"] = {"ms": t * 1e3, "algorithmic_bytes": eb["massflow"],
                             "frac": eb["massflow"] / t / 1e9 / peak}
    t = event_time(lambda: solver._assemble_fused())
    out["assembly_stage"] = {"ms": t * 1e3, "what": "gradients, diagonal, limiter (frozen after "
                                                    "10 iterations), assembly, boundary pass"}
    A, b, _, x0 = solver._assemble_fused()
    lin = solver.linear
    lin.setup(A)
    st = lin.stats()
    r = b.reshape(-1) - A.matvec(x0)
    t = event_time(lambda: lin.vcycle(r), reps=10)
    vb = vcycle_bytes(st, value_bytes, smoother=smoother,
                      cheb_steps=lin.presweeps + lin.postsweeps, coarse_sweeps=lin.coarse_sweeps)
    out["vcycle"] = {"ms": t * 1e3, "algorithmic_bytes": vb, "frac": vb / t / 1e9 / peak,
                     "levels": st["levels"], "blocks": st["blocks"]}
    n0, nnz0 = st["levels"][0], st["blocks"][0]
    t = event_time(lambda: call("zvfv_solver_smooth", lin._h, 0, 1, stream_ptr()), reps=10)
    if smoother == "chebyshev":
        cb = cheb_step_bytes(n0, nnz0, value_bytes, value_bytes)
        kern = "double, double>" if value_bytes == 8 else "float, float>"
        out["gs_pass"] = {"ms": t * 1e3, "algorithmic_bytes": cb, "frac": cb / t / 1e9 / peak,
                          "kernel": f"k_cheby<{_lanes(n0, nnz0)}, false, false, " + kern,
                          "launches": 1, "what": "one Chebyshev step on the finest level"}
        return out, st
    gb = gs_pass_bytes(n0, nnz0, value_bytes, value_bytes)
    kern = "double, double>" if value_bytes == 8 else "float, float>"
    out["gs_pass"] = {"ms": t * 1e3, "algorithmic_bytes": gb, "frac": gb / t / 1e9 / peak,
                      "kernel": "k_gs_colour_pdl<16, " + ("4, " if value_bytes == 8 else "8, ")
                                + kern,
                      "launches": int(_gs_colours(lin))}
    return out, st


def _lanes(n, nnz):
    """Lanes per row of the hierarchy's row kernels (without the autotuner)."""
    per = nnz / max(n, 1)
    return 32 if per > 40 else (16 if per > 12 else 8)


def _gs_colours(lin):
    """Launches of one Gauss-Seidel pass on the finest level (its colours)."""
    from zvcfd_b200._lib import call, lib, stream_ptr

    before = lib.zvfv_launch_count()
    call("zvfv_solver_smooth", lin._h, 0, 1, stream_ptr())
    return lib.zvfv_launch_count() - before


def iteration_bytes(solver, stats, linear_iterations, value_bytes=8, smoother="gs"):
    """Algorithmic bytes of one outer iteration (mean over the timed window): the element
    stage, two gradient passes, the boundary pass (matrix read and written once), per Krylov
    step one V-cycle, one operator product and the Arnoldi passes (CGS2 over the basis, mean
    index k), the update, and the hierarchy's coefficient refresh (Galerkin sums)."""
    N, nnzb = solver.N, solver.nnzb
    eb = element_bytes(solver.asm)
    its = float(np.mean(linear_iterations)) if linear_iterations else 0.0
    n4 = 4 * N * 8
    lin = solver.linear
    vc = vcycle_bytes(stats, value_bytes, smoother=smoother,
                      cheb_steps=lin.presweeps + lin.postsweeps, coarse_sweeps=lin.coarse_sweeps)
    krylov = vc + spmv_bytes(N, nnzb) + (4 * (its / 2 + 1) + 8) * n4
    grad = 2 * (nnzb * (24 + 4) + 8 * N + 4 * 8 * N + 12 * 8 * N)
    finalise = 2 * 128 * nnzb + 8 * nnzb + 4 * n4
    refresh = sum(2 * 16 * 8 * nb for nb in stats["blocks"])
    return eb["assemble"] + eb["massflow"] + grad + finalise + its * krylov + 2 * n4 + refresh


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--axial", type=int, default=285, help="axial cells (285: the full tube)")
    ap.add_argument("--cpu-axial", type=int, default=6,
                    help="axial cells of the CPU sample (an arc of the full tube's cells)")
    ap.add_argument("--no-converge", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-stages", action="store_true")
    ap.add_argument("--workload", default="tube",
                    choices=["tube", "bifurcation", "ensemble", "adjoint", "smoothers",
                             "partitioned"],
                    help="tube: the headline (default); bifurcation: the 2M-node transient; "
                         "ensemble: the 12-vessel batch; adjoint: the 500k-node steady "
                         "gradient; smoothers: the AMG smoothers compared on the headline tube; "
                         "partitioned: partitions sharing the GPU vs the single-GPU solve")
    ap.add_argument("--parts", default="2,4", help="partitioned workload: partition counts")
    ap.add_argument("--nodes", type=int, default=2_000_000, help="bifurcation workload size")
    ap.add_argument("--loops", type=int, default=5,
                    help="bifurcation: coefficient loops per time step at most (the reference's 5)")
    ap.add_argument("--instances", type=int, default=12, help="ensemble workload size")
    ap.add_argument("--max-nodes", type=int, default=1_200_000,
                    help="largest ensemble instance")
    ap.add_argument("--krylov", default="segmented", choices=["segmented", "union"],
                    help="ensemble: one Krylov recurrence per instance, or one over the union")
    ap.add_argument("--adjoint-nodes", type=int, default=500_000, help="adjoint workload size")
    ap.add_argument("--adjoint-tol", type=float, default=1e-10,
                    help="adjoint workload: the forward solves' residual target")
    ap.add_argument("--adjoint-iterations", type=int, default=1000,
                    help="adjoint workload: the forward solves' outer-iteration limit")
    ap.add_argument("--adjoint-rtol", type=float, default=1e-10,
                    help="adjoint workload: the adjoint FGMRES tolerance")
    ap.add_argument("--adjoint-fd", default="",
                    help="adjoint workload: the parameters checked by central differences, "
                         "comma-separated (default all): Q_in,Rp1,C1,Rd1,Rp2,C2,Rd2,mu0")
    ap.add_argument("--adjoint-restart", type=int, default=40,
                    help="adjoint workload: the adjoint FGMRES restart length")
    ap.add_argument("--smoother", default=None,
                    choices=["chebyshev", "gs", "dilu", "ilu0", "jacobi"],
                    help="tube: the AMG smoother of both solvers (default: the library's)")
    ap.add_argument("--nvtx", action="store_true",
                    help="mark the timed steps with an NVTX range 'timed' (for ncu --nvtx-include)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        return reference_arm(args, rank, world)
    if args.workload != "tube":
        import torch

        torch.cuda.set_device(local)
        if rank == 0:
            {"bifurcation": bifurcation_workload, "ensemble": ensemble_workload,
             "adjoint": adjoint_workload, "smoothers": smoothers_workload,
             "partitioned": partitioned_workload}[args.workload](args)
        return

    import torch

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    from zvcfd_b200._lib import lib
    from zvcfd_b200.solver import B200Solver

    m, fl, bcs = make_case(args.axial)
    # two identical solvers: `value` is timed on one, `e2e` on the other over the same outer
    # iterations (warm-up + 1 .. warm-up + steps) - the device work is deterministic
    lopts = {} if args.smoother is None else {"smoother": args.smoother}
    solver = B200Solver(m, fl, bcs, linear="b200", linear_rtol=0.1, linear_options=lopts)
    twin = B200Solver(m, fl, bcs, linear="b200", linear_rtol=0.1, linear_options=lopts)
    for _ in range(args.warmup):
        solver.iterate()
        twin.iterate()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    l0 = lib.zvfv_launch_count()
    if args.nvtx:
        torch.cuda.nvtx.range_push("timed")
    with Clocks(local) as clk:
        elapsed, recs = run_steps(solver, args.steps)
    if args.nvtx:
        torch.cuda.nvtx.range_pop()
    launches = lib.zvfv_launch_count() - l0
    if dist:
        elapsed = max_over_ranks(elapsed, dist, "cuda")
        dist.barrier()
    per = elapsed / args.steps
    value = world * args.steps / elapsed
    # end to end through the public API on the twin: every step copies the state in from
    # pinned host memory, runs one outer iteration (B200Solver.iterate, whose record - the
    # residuals, changes and flows - is read back) and copies the new state out
    N = m.n_nodes
    Uh = torch.empty((N, 3), dtype=torch.float64, pin_memory=True)
    Ph = torch.empty(N, dtype=torch.float64, pin_memory=True)
    Uh.copy_(twin.U)
    Ph.copy_(twin.P)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    twin_recs = []
    for _ in range(args.steps):
        twin.U.copy_(Uh, non_blocking=True)
        twin.P.copy_(Ph, non_blocking=True)
        twin_recs.append(twin.iterate())
        Uh.copy_(twin.U, non_blocking=True)
        Ph.copy_(twin.P, non_blocking=True)
        torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    if dist:
        e2e_s = max_over_ranks(e2e_s, dist, "cuda")
    e2e = world * args.steps / e2e_s
    same = [r["linear_iterations"] for r in recs] == [r["linear_iterations"] for r in twin_recs]
    twin.close()
    # mixed precision on the same case and window
    mixed = B200Solver(m, fl, bcs, linear="b200-mixed", linear_rtol=0.1, linear_options=lopts)
    for _ in range(args.warmup):
        mixed.iterate()
    melapsed, mrecs = run_steps(mixed, args.steps)
    extra = {"fp64_linear_iterations": [r["linear_iterations"] for r in recs],
             "e2e_window_matches_value_window": same,
             "mixed": {"ms_per_step": melapsed / args.steps * 1e3,
                       "outer_iterations_per_s": args.steps / melapsed,
                       "speedup_vs_fp64": elapsed / melapsed,
                       "linear_iterations": [r["linear_iterations"] for r in mrecs]}}
    peak, peak_kind = peaks()
    peak_source = (f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
                   else "fallback 6.65 TB/s")
    # SpMV on the assembled matrix, stages, the dominant kernel alone
    sp, n, nnzb = spmv_roofline(solver)
    extra["spmv"] = {"fp64_gbs": sp["fp64"]["gbs"], "fp32_gbs": sp["fp32"]["gbs"],
                     "fp64_us": sp["fp64"]["seconds"] * 1e6, "fp32_us": sp["fp32"]["seconds"] * 1e6,
                     "fp64_frac": sp["fp64"]["gbs"] / peak, "nnzb": nnzb, "rows": n}
    roof = None
    if not args.no_stages:
        stages, hstats = stage_times(solver, peak, smoother=solver.linear.smoother)
        mstages, _ = stage_times(mixed, peak, 4, smoother=mixed.linear.smoother)
        ib = iteration_bytes(solver, hstats, extra["fp64_linear_iterations"],
                             smoother=solver.linear.smoother)
        extra["stages"] = {"fp64": stages,
                           "mixed": {k: mstages[k] for k in ("vcycle", "gs_pass")}}
        extra["outer_iteration_roofline"] = {
            "algorithmic_bytes": ib, "achieved_gbs": ib / per / 1e9, "peak": peak,
            "frac": ib / per / 1e9 / peak, "unit": "GB/s",
            "note": "sum of the algorithmic bytes of every stage of one outer iteration "
                    "(mean Krylov steps of the window) over ms_per_step"}
        g = stages["gs_pass"]
        what = g.get("what", "one pass over all colours of the finest level")
        roof = {"kernel": f"{g['kernel']} ({what})",
                "bound": "hbm", "achieved": g["algorithmic_bytes"] / (g["ms"] * 1e-3) / 1e9,
                "peak": peak, "unit": "GB/s", "frac": g["frac"], "peak_source": peak_source,
                "algorithmic_bytes": g["algorithmic_bytes"],
                "traffic": None if GS_TRAFFIC_PER_ALGORITHMIC_BYTE is None or
                solver.linear.smoother != "gs"
                else GS_TRAFFIC_PER_ALGORITHMIC_BYTE * g["algorithmic_bytes"],
                "traffic_source": GS_TRAFFIC_SOURCE if solver.linear.smoother == "gs" else None}
    if not args.no_converge and rank == 0:
        conv = {}
        for tag, lin in (("fp64", "b200"), ("mixed", "b200-mixed")):
            s = B200Solver(m, fl, bcs, linear=lin, linear_rtol=0.1, linear_options=lopts)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            rep = s.solve(max_iterations=400, tol=1e-8)
            torch.cuda.synchronize()
            conv[tag] = {"outer_iterations": rep["iterations"], "converged": rep["converged"],
                         "seconds": time.perf_counter() - t0,
                         "final_rms": max(rep["history"][-1][f"rms_{c}"] for c in "uvwp"),
                         "fields": s.fields()}
            s.close()
        f64, fmx = conv["fp64"].pop("fields"), conv["mixed"].pop("fields")
        conv["mixed"]["field_error_vs_fp64"] = {
            "U": float(np.linalg.norm(fmx["U"] - f64["U"]) / np.linalg.norm(f64["U"])),
            "P": float(np.linalg.norm(fmx["P"] - f64["P"]) / np.linalg.norm(f64["P"]))}
        conv["mixed"]["speedup_vs_fp64"] = conv["fp64"]["seconds"] / conv["mixed"]["seconds"]
        extra["to_1e-8"] = conv
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        t_cpu, n_cpu, its = cpu_baseline_sample(args.cpu_axial)
        per_cpu = t_cpu * N / n_cpu
        A, _, _, _ = solver._assemble_fused()
        gbs = cpu_spmv_gbs(A.indptr.cpu().numpy(), A.indices.cpu().numpy(),
                           A.data.cpu().numpy())
        cpu = {"value": 1.0 / per_cpu, "unit": UNIT, "cores": 1, "kind": "port",
               "sample": f"the reference arm's path (oracle NumPy assembly + ACM-FGMRES to 0.1) "
                         f"on a {args.cpu_axial}-cell arc of the same tube (the same cells) "
                         f"({n_cpu} nodes, linear iterations {its}), per outer iteration scaled "
                         f"by node count to {N:,} nodes: an estimate (bench.py --impl reference "
                         f"measures the full size); SciPy BSR SpMV on the full matrix "
                         f"{gbs:.2f} GB/s",
               "spmv_gbs": gbs, "host": host_info()}
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": per * 1e3,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic",
                "config": {"workload": WORKLOAD, "nodes": N, "blocks": nnzb,
                           "precision": "fp64 (mixed below)", "linear_rtol": 0.1,
                           "smoother": solver.linear.smoother,
                           "parallelism": f"replicas x{world}", "l2": "inputs larger than L2"},
                "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": 32 * N,
                        "d2h_bytes_per_step": 32 * N + 8 * 29},
                "gpu_launches": int(launches), "roofline": roof, "cpu_baseline": cpu,
                "clocks": clk.summary(), **extra}
        print(json.dumps(line), flush=True)
    solver.close()
    mixed.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
