"""Benchmark: one Backward-Euler step of 3D transient heat on a 128^3 Q1-hex mesh, solved to a
1e-8 relative residual checked in FP64 -- mixed FP32/FP64 CG+Jacobi (the headline) beside plain
FP64 CG+Jacobi on the same steps, plus the dominant kernel's roofline and the reference CPU path.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--size S] [--impl ours|reference]

A step is everything BackwardEulerRunner::step does in the reference: Udot, K + M/dt assembly,
load, (1/dt) M U_prev, Dirichlet lift, the CG solve warm-started from U, the stage residual norm
and the advance.  Inputs are synthetic (the configuration's seeded sine-mode initial condition).
With N > 1 every rank runs an independent replica (the solve has no exchange step to shard).
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)


def load_package():
    import importlib.util
    name = "residuum_solver_b200"
    if name in sys.modules:
        return sys.modules[name]
    pkg = os.path.join(ROOT, "residuum-solver_b200")
    spec = importlib.util.spec_from_file_location(name, os.path.join(pkg, "__init__.py"), submodule_search_locations=[pkg])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


# ---------------------------------------------------------------------------------------------
# synthetic input: std::mt19937_64 (its output sequence is fixed by the C++ standard), uniform
# double u = (x >> 11) * 2^-53, integer in [a, b] = a + floor(u (b - a + 1))
# ---------------------------------------------------------------------------------------------
class MT19937_64:
    def __init__(self, seed):
        self.mt = [0] * 312
        self.mt[0] = seed & 0xFFFFFFFFFFFFFFFF
        for i in range(1, 312):
            self.mt[i] = (6364136223846793005 * (self.mt[i - 1] ^ (self.mt[i - 1] >> 62)) + i) & 0xFFFFFFFFFFFFFFFF
        self.idx = 312

    def next(self):
        if self.idx >= 312:
            mt = self.mt
            for i in range(312):
                x = (mt[i] & 0xFFFFFFFF80000000) | (mt[(i + 1) % 312] & 0x7FFFFFFF)
                xa = x >> 1
                if x & 1:
                    xa ^= 0xB5026F5AA96619E9
                mt[i] = mt[(i + 156) % 312] ^ xa
            self.idx = 0
        y = self.mt[self.idx]
        self.idx += 1
        y ^= (y >> 29) & 0x5555555555555555
        y ^= (y << 17) & 0x71D67FFFEDA60000
        y ^= (y << 37) & 0xFFF7EEE000000000
        y ^= y >> 43
        return y & 0xFFFFFFFFFFFFFFFF

    def uniform(self):
        return (self.next() >> 11) * (1.0 / 9007199254740992.0)

    def integer(self, a, b):
        return a + int(self.uniform() * (b - a + 1))


_MT_U, _MT_L, _MT_A = np.uint64(0xFFFFFFFF80000000), np.uint64(0x7FFFFFFF), np.uint64(0xB5026F5AA96619E9)


def mt19937_64_stream(seed, count):
    """The first `count` outputs of std::mt19937_64(seed), the twist and tempering vectorized with
    numpy (the twist splits into the three index ranges whose inputs are already final)."""
    mt = np.array(MT19937_64(seed).mt, dtype=np.uint64)
    out = np.empty(count, np.uint64)
    done = 0
    one = np.uint64(1)
    with np.errstate(over="ignore"):
        while done < count:
            for lo, hi, src in ((0, 156, 156), (156, 311, -156)):
                i = np.arange(lo, hi)
                x = (mt[i] & _MT_U) | (mt[i + 1] & _MT_L)
                mt[i] = mt[i + src] ^ (x >> one) ^ np.where((x & one) == one, _MT_A, np.uint64(0))
            x = (mt[311] & _MT_U) | (mt[0] & _MT_L)
            mt[311] = mt[155] ^ (x >> one) ^ (_MT_A if int(x) & 1 else np.uint64(0))
            y = mt.copy()
            y ^= (y >> np.uint64(29)) & np.uint64(0x5555555555555555)
            y ^= (y << np.uint64(17)) & np.uint64(0x71D67FFFEDA60000)
            y ^= (y << np.uint64(37)) & np.uint64(0xFFF7EEE000000000)
            y ^= y >> np.uint64(43)
            k = min(312, count - done)
            out[done:done + k] = y[:k]
            done += k
    return out


def uniforms(bits):
    """uniform doubles in [0, 1): (x >> 11) * 2^-53"""
    return (bits >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def batch_problem(p):
    """Problem p of the batched workload: stream mt19937_64(4000 + p); Nx, Ny ~ U{32..256}; then per
    element, in element order, z_e ~ N(0, 1) by Box-Muller (cos branch) from two uniforms u1, u2 as
    sqrt(-2 ln(1 - u1)) cos(2 pi u2); k_e = exp(z_e)."""
    head = uniforms(mt19937_64_stream(4000 + p, 2))
    nx, ny = (32 + int(u * 225) for u in head)
    u = uniforms(mt19937_64_stream(4000 + p, 2 + 2 * nx * ny)[2:]).reshape(-1, 2)
    z = np.sqrt(-2.0 * np.log1p(-u[:, 0])) * np.cos(2.0 * np.pi * u[:, 1])
    return nx, ny, np.exp(z)


def sine_modes(seed=2, modes=8):
    """T0(x) = sum_m 0.1 sin(a_m . x + b_m), a_m = pi * i_m with i_m ~ U{1..8}^3, b_m ~ U[0, 2pi);
    per mode the three integers are drawn before the phase."""
    g = MT19937_64(seed)
    A, B = [], []
    for _ in range(modes):
        A.append([np.pi * g.integer(1, 8) for _ in range(3)])
        B.append(2.0 * np.pi * g.uniform())
    return np.array(A), np.array(B)


def initial_condition(xyz, a2t, seed=2):
    A, B = sine_modes(seed)
    X = xyz.reshape(-1, 3)[a2t]
    return (0.1 * np.sin(X @ A.T + B[None, :])).sum(axis=1)


# ---------------------------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------------------------
class ClockSampler:
    """SM clock and clock-event reasons sampled by NVML (read-only queries) every 2 ms in a thread
    while the timed region runs; nvidia-smi's 100 ms minimum interval is longer than a timed region
    of a few steps.  Reports the median SM clock under load, the maximum SM clock and the reasons
    seen active."""
    REASONS = (("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"), ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
               ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"), ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap"),
               ("hw_power_brake", "nvmlClocksEventReasonHwPowerBrakeSlowdown"))

    def __init__(self, device):
        self.device = device
        self.thread = None
        self.samples, self.reasons = [], set()
        self.err = None

    def _run(self):
        import pynvml
        h = pynvml.nvmlDeviceGetHandleByIndex(self.device)
        while not self.stop_flag:
            try:
                self.samples.append(pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM))
                r = pynvml.nvmlDeviceGetCurrentClocksEventReasons(h)
                for name, const in self.REASONS:
                    if r & getattr(pynvml, const, 0):
                        self.reasons.add(name)
            except Exception as e:  # noqa: BLE001
                self.err = str(e)
                break
            time.sleep(0.002)

    def start(self):
        import threading
        try:
            import pynvml
            pynvml.nvmlInit()
            h = pynvml.nvmlDeviceGetHandleByIndex(self.device)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM)
        except Exception as e:  # noqa: BLE001
            self.err = f"nvml unavailable: {e}"
            return
        self.stop_flag = False
        self.thread = threading.Thread(target=self._run, daemon=True)
        self.thread.start()

    def stop(self):
        if self.thread is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [self.err or "not sampled"], "samples": 0}
        self.stop_flag = True
        self.thread.join()
        sm = self.samples
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": float(self.max_mhz),
                "reasons": sorted(self.reasons), "samples": len(sm), "source": "nvml, 2 ms"}


def measured_peak_hbm():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        return float(json.load(open(p))["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def ncu_traffic(kernel):
    """DRAM traffic per launch for a kernel from the committed ncu summary, or None."""
    p = os.path.join(ROOT, "profiles", "dram_traffic.json")
    if os.path.exists(p):
        d = json.load(open(p))
        if kernel in d:
            return d[kernel]
    return None


# ---------------------------------------------------------------------------------------------
# reference CPU path (oracle/_ref: the reference templates compiled unmodified) on the full workload
# ---------------------------------------------------------------------------------------------
def reference_steps(S, nsteps):
    """`nsteps` Backward-Euler steps of the S^3 workload from T0 through the reference's own
    BackwardEulerStage + BackwardEulerRunner (oracle/_ref, one core: the reference is
    single-threaded).  Returns the state after the last step, the per-step wall seconds of
    runner.step() and of its linear solve, the CG iterations per step, and the seconds spent before
    the first step (mesh, DOF map, CSR pattern, the stage's first matrix assembly in setDt)."""
    import oracle
    if not oracle.reference_available():
        return None
    t0 = time.perf_counter()
    r = oracle.Reference(3, 1, 2, [S] * 3, [0, 0, 0], [1, 1, 1], list(range(6)), bc_kind=0, rho=1.0, cp=1.0)
    # node coordinates from the oracle's block mesh (the reference's numbering): nothing of the
    # device package runs on this path
    xyz = oracle.BlockMesh(3, [S] * 3, [0, 0, 0], [1, 1, 1], 1).xyz
    t2a, a2t = r.dofmap()
    U0 = initial_condition(xyz, a2t)
    setup = time.perf_counter() - t0
    t1 = time.perf_counter()
    U, _, rc, st = r.backward_euler(1e-3, nsteps, U0, tol=1e-8, maxit=100000, stats=True)
    total = time.perf_counter() - t1
    return {"U": U, "U0": U0, "n": r.n, "nnz": r.nnz, "elements": r.nelem, "rc": rc, "step_s": st[:, 0],
            "solve_s": st[:, 1], "iters": st[:, 2], "setup_s": setup + total - float(st[:, 0].sum())}


def reference_config(S):
    """The workload description both arms print (the reference arm computes the sizes itself)."""
    n, nnz = (S - 1) ** 3, (3 * S - 5) ** 3
    return {"workload": WORKLOAD.format(S=S), "n_free": n, "nnz": nnz, "elements": S ** 3, "parallelism": "replicas",
            "l2": "inputs larger than L2 (CSR FP64 values + columns %.2f GB)" % (nnz * 12 / 1e9)}


def run_reference_arm(args, rank, world):
    """bench.py --impl reference: the reference's own Backward-Euler steps on the same 128^3 workload,
    timed on the host (one core), `--ref-steps` of them (each about half a minute) so that the arm
    ends within a few minutes whatever --steps asks for; the steps timed are the line's `steps`."""
    if rank != 0:
        return
    S = args.size
    nsteps = max(1, min(args.steps, args.ref_steps))
    try:
        import oracle
        if not oracle.reference_available():
            print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libresiduum_ref.so not built (reference tree absent at build time)"}))
            return
        ref = reference_steps(S, nsteps)
    except Exception as e:  # noqa: BLE001
        print(json.dumps({"impl": "reference", "unavailable": f"reference run failed: {e}"}))
        return
    ms = 1e3 * float(np.median(ref["step_s"]))
    sample = (f"{nsteps} Backward-Euler step(s) of the {S}^3 workload from T0 (dt = 1e-3, FP64 CG + Jacobi to 1e-8) "
              f"through the reference templates (oracle/_ref: BackwardEulerStage + BackwardEulerRunner::step), 1 core, "
              f"median of runner.step() wall times; CG iterations {[int(i) for i in ref['iters']]}; "
              f"setup before the first step {ref['setup_s']:.1f} s untimed")
    line = {"impl": "reference", "metric": METRIC, "value": ms, "unit": "ms", "n_gpus": world, "steps": nsteps,
            "warmup": 0, "ms_per_step": ms, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic", "config": reference_config(S),
            "requested": {"steps": args.steps, "warmup": args.warmup},
            "step_ms": [1e3 * float(t) for t in ref["step_s"]], "solve_ms": [1e3 * float(t) for t in ref["solve_s"]],
            "cpu_baseline": {"value": ms, "unit": "ms", "cores": 1, "kind": "reference", "sample": sample},
            "e2e": {"value": ms, "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def batch_share(count, world, rank):
    """The problems of the batched workload that rank `rank` of `world` solves: largest first, each to
    the rank with the fewest rows so far (ties to the lower rank).  Independent problems need no
    exchange, so ranks share nothing but the final timing."""
    rows = []
    for p in range(count):
        head = uniforms(mt19937_64_stream(4000 + p, 2))
        nx, ny = (32 + int(u * 225) for u in head)
        rows.append(((nx - 1) * (ny - 1), p))
    load = [0] * world
    mine = []
    for r, p in sorted(rows, key=lambda t: (-t[0], t[1])):
        k = min(range(world), key=lambda i: (load[i], i))
        load[k] += r
        if k == rank:
            mine.append(p)
    return sorted(mine)


def ranks_reduce(value, op, dist, device):
    """max or sum of a float over the ranks (the value itself on one rank)."""
    if dist is None:
        return value
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())


def _batch_cpu_worker(ps):
    """One process of the batched workload's CPU baseline: problems `ps` through the reference's own
    templates (oracle/_ref), each assembled (untimed) and then solved by the reference's FP64
    CG + Jacobi to 1e-8 from x0 = 0 (timed).  Returns (solve seconds, iterations)."""
    import oracle
    solve_s, iters = 0.0, 0
    for p in ps:
        nx, ny, ke = batch_problem(p)
        r = oracle.Reference(2, 1, 2, [nx, ny], [0, 0], [1, 1], [0, 1, 2, 3], bc_kind=0, src_kind=0, src_c=1.0, k_elem=ke)
        val = r.assemble_matrix("K")
        F = r.assemble_vector(0)
        rp, col = r.pattern()
        t0 = time.perf_counter()
        _, rep = oracle.ref_csr_solve(rp, col, val, F, tol=1e-8, maxit=100000)
        solve_s += time.perf_counter() - t0
        iters += int(rep["iterations"])
    return solve_s, iters


def batch_cpu_baseline(count):
    """The reference CPU solver over the whole batch with P = min(cores, 32) spawned processes (the
    reference is single-threaded), each taking every P-th problem of the largest-first order: the
    slowest process's solve seconds are the time for the batch at P cores."""
    import multiprocessing as mp
    import oracle
    if not oracle.reference_available():
        return None
    rows = []
    for p in range(count):
        head = uniforms(mt19937_64_stream(4000 + p, 2))
        nx, ny = (32 + int(u * 225) for u in head)
        rows.append(((nx - 1) * (ny - 1), p))
    order = [p for _, p in sorted(rows, key=lambda t: (-t[0], t[1]))]
    procs = max(1, min(os.cpu_count() or 1, 32))
    with mp.get_context("spawn").Pool(procs) as pool:
        res = pool.map(_batch_cpu_worker, [order[i::procs] for i in range(procs)])
    slowest = max(t for t, _ in res)
    return {"value": 1e3 * slowest, "unit": "ms", "cores": procs, "kind": "reference",
            "problems_per_s": count / slowest, "iterations_total": int(sum(i for _, i in res)),
            "sample": f"all {count} problems, FP64 CG + Jacobi to 1e-8 through the reference templates "
                      f"(oracle/_ref), {procs} spawned processes, solve time of the slowest (assembly untimed)"}


def run_batch(rsd, ctx, stream, count, reps, peak, rank=0, world=1, dist=None, device="cuda", cpu=False):
    """The batched workload: `count` unit-square Q1 problems (Nx, Ny ~ U{32..256}, log-normal
    per-element conductivity, unit source, T = 0 on the boundary) solved together by
    rsd_batch_solve, CG + Jacobi to 1e-8 (mixed: FP64-checked), x0 = 0.  With several ranks each
    solves its share (batch_share) and the time is the slowest rank's."""
    import torch
    from importlib import import_module
    bm = import_module("residuum_solver_b200.blockmesh")
    t0 = time.time()
    probs = []
    for p in batch_share(count, world, rank):
        nx, ny, ke = batch_problem(p)
        xyz, ien, rg = bm.block_mesh(2, [nx, ny], [0, 0], [1, 1], 1)
        h = rsd.Heat(ctx, rsd.Mesh(ctx, 2, 1, xyz, ien, rg), 2, k_elem=ke, src_expr="1",
                     dirichlet={t: "0" for t in range(4)})
        h.assemble_matrix(1.0)
        F = ctx.array(h.n)
        h.assemble_vector(0, F)
        probs.append((h, F))
    setup_s = time.time() - t0
    B = rsd.Batch(ctx, [h.K for h, _ in probs])
    xs = [ctx.array(h.n) for h, _ in probs]
    ns = np.array([h.n for h, _ in probs], dtype=np.float64)
    nnzs = np.array([h.nnz for h, _ in probs], dtype=np.float64)
    out = {"problems": count, "rows": int(ranks_reduce(ns.sum(), "sum", dist, device)),
           "nnz": int(ranks_reduce(nnzs.sum(), "sum", dist, device)), "setup_s": round(setup_s, 2), "ranks": world}
    for key, prec in (("mixed", rsd.MIXED), ("fp64", rsd.FP64)):
        cfg = rsd.SolverConfig.make(precision=prec, tol=1e-8, max_iters=100000)
        ts = []
        for r in range(reps + 1):
            for x in xs:
                x.zero()
            torch.cuda.synchronize()
            if dist is not None:
                dist.barrier()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            rr = B.solve([F for _, F in probs], xs, cfg)
            e1.record(stream)
            e1.synchronize()
            if r:
                ts.append(e0.elapsed_time(e1))
        its = np.array([q["iterations"] for q in rr], dtype=np.float64)
        refs = np.array([q["refinements"] for q in rr], dtype=np.float64)
        s = 4 if key == "mixed" else 8
        # PCG+Jacobi per iteration: SpMV nnz(s+4) + 4(n+1) + 2ns, and 11 vector passes of n*s;
        # each FP64 residual replacement one FP64 SpMV plus 4 n*8
        byts = float(np.sum(its * (nnzs * (s + 4) + 4 * (ns + 1) + 2 * ns * s + 11 * ns * s)
                            + refs * (nnzs * 12 + 4 * (ns + 1) + 2 * ns * 8 + 4 * ns * 8)))
        ms = ranks_reduce(float(np.median(ts)), "max", dist, device)
        byts = ranks_reduce(byts, "sum", dist, device)
        conv = ranks_reduce(0.0 if all(q["converged"] for q in rr) else 1.0, "max", dist, device) == 0.0
        out[key] = {"ms": ms, "problems_per_s": count / (ms * 1e-3), "all_converged": conv,
                    "iterations_total": int(ranks_reduce(its.sum(), "sum", dist, device)),
                    "iterations_max": int(ranks_reduce(its.max() if len(its) else 0, "max", dist, device)),
                    "refinements_total": int(ranks_reduce(refs.sum(), "sum", dist, device)),
                    "max_true_residual_rel": ranks_reduce(max([q["trueResidualRel"] for q in rr] or [0.0]), "max", dist, device),
                    "algorithmic_gbs": byts / (ms * 1e-3) / 1e9,
                    "frac_of_measured_hbm": byts / (ms * 1e-3) / 1e9 / (peak * world)}
    out["speedup_mixed_vs_fp64"] = out["fp64"]["ms"] / out["mixed"]["ms"]
    if cpu and rank == 0 and world == 1:
        try:
            out["cpu_baseline"] = batch_cpu_baseline(count)
        except Exception as e:  # noqa: BLE001
            out["cpu_baseline"] = {"value": None, "sample": f"failed: {e}"}
    out["how"] = ("one rsd_batch_solve call (one persistent launch), CUDA events around the call, median of "
                  f"{reps}; setup (meshes, patterns, assembly) outside the timed region")
    del B
    return out


def newton_cpu_baseline(rsd, ctx, stream, m):
    """The reference's own Newton (oracle/_ref: its NewtonRunner over SteadyStage with GMRES(30) +
    Jacobi, 1 core) on an m^3 Q2 sample of the Newton workload, beside this library's Newton on the
    same sample."""
    import oracle
    if not oracle.reference_available():
        return None
    r = oracle.Reference(3, 2, 3, [m] * 3, [0, 0, 0], [1, 1, 1], [0, 1], bc_kind=0, bc_val={0: 0.0, 1: 1.0},
                         src_kind=0, src_c=10.0, k_a=1.0, k_b=0.5)
    t0 = time.perf_counter()
    _, rep = r.newton(1e-10, 1e-10, 50, solver=1, precond=1, tol=1e-12, lin_maxit=100000, krylov=30)
    cpu_ms = 1e3 * (time.perf_counter() - t0)
    dev = run_newton(rsd, ctx, stream, m)
    return {"value": cpu_ms, "unit": "ms", "cores": 1, "kind": "reference", "newton_iterations": rep["iterations"],
            "device_same_sample_ms": {"fp64": dev["fp64"]["ms"], "mixed": dev["mixed"]["ms"]},
            "sample": f"the whole Newton solve on {m}^3 Q2 hexes ({r.n} rows) through the reference templates "
                      f"(oracle/_ref), 1 core; the device times are this library's Newton on the same mesh"}


def run_newton(rsd, ctx, stream, S):
    """Steady nonlinear heat on S^3 Q2 hexes: k(T) = 1 + 0.5 T, f = 10, T = 0 on x = 0 and 1 on x = 1,
    zero flux elsewhere; Newton to 1e-10 (absolute or relative) with GMRES(30) + Jacobi inner solves
    to 1e-12, x0 = 0, inner GMRES in FP64 and mixed (FP32 Arnoldi, FP64 restart residuals).  Checked
    against the 1D closed form T = 2(sqrt(1 + u) - 1), u = 6.25 x - 5 x^2."""
    import torch
    from importlib import import_module
    bm = import_module("residuum_solver_b200.blockmesh")
    t0 = time.time()
    xyz, ien, rg = bm.block_mesh(3, [S] * 3, [0, 0, 0], [1, 1, 1], 2)
    h = rsd.Heat(ctx, rsd.Mesh(ctx, 3, 2, xyz, ien, rg), 3, k_expr="1 + 0.5*T", dk_expr="0.5", src_expr="10",
                 dirichlet={0: "0", 1: "1"})
    setup_s = time.time() - t0
    U = ctx.array(h.n)
    t2a, a2t = h.dofmap()
    x = xyz.reshape(-1, 3)[a2t, 0]
    exact = 2.0 * (np.sqrt(1.0 + 6.25 * x - 5.0 * x * x) - 1.0)
    out = {"workload": f"{S}^3 Q2 hexes, k(T) = 1 + 0.5T, f = 10, Newton 1e-10, GMRES(30) + Jacobi 1e-12",
           "n_free": h.n, "nnz": h.nnz, "setup_s": round(setup_s, 2)}
    sols = {}
    for key, prec in (("fp64", rsd.FP64), ("mixed", rsd.MIXED)):
        cfg = rsd.SolverConfig.make(type=rsd.GMRES, krylov_dim=30, tol=1e-12, max_iters=100000, precision=prec)
        U.zero()
        h.newton(U, 1e-10, 1e-10, 50, cfg)          # warm-up (workspace setup)
        U.zero()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        rep = h.newton(U, 1e-10, 1e-10, 50, cfg)
        e1.record(stream)
        e1.synchronize()
        sols[key] = U.download()
        out[key] = {"ms": e0.elapsed_time(e1), "newton_iterations": rep["iterations"],
                    "gmres_iterations_total": rep["refinements"], "converged": bool(rep["converged"]),
                    "final_residual": rep["finalResidual"],
                    "max_error_vs_1d_closed_form": float(np.max(np.abs(sols[key] - exact)))}
    out["speedup_mixed_vs_fp64"] = out["fp64"]["ms"] / out["mixed"]["ms"]
    out["mixed_vs_fp64_max_rel_diff"] = float(np.max(np.abs(sols["mixed"] - sols["fp64"])) / np.max(np.abs(sols["fp64"])))
    return out


def fem_steady(rsd, ctx, stream, S, op, reps=3):
    """Steady linear heat on S^3 Q2 hexes (k = 1, f = 10, T = 0 on x = 0 and 1 on x = 1), CG + Jacobi
    in FP64 to 1e-8 from x0 = 0 with the assembled matrix (op CSR: assembly + solve) or the matrix-free
    operator (op FEM: the solve's products are element passes); median of reps event-timed stages."""
    import torch
    from importlib import import_module
    bm = import_module("residuum_solver_b200.blockmesh")
    xyz, ien, rg = bm.block_mesh(3, [S] * 3, [0, 0, 0], [1, 1, 1], 2)
    h = rsd.Heat(ctx, rsd.Mesh(ctx, 3, 2, xyz, ien, rg), 3, src_expr="10", dirichlet={0: "0", 1: "1"})
    cfg = rsd.SolverConfig.make(type=rsd.CG, precond=rsd.JACOBI, precision=rsd.FP64, tol=1e-8, max_iters=100000,
                                operator_type=op)
    U = ctx.array(h.n).zero()
    h.steady(U, cfg=cfg)            # warm-up (tables, maps, workspace)
    ts = []
    for _ in range(reps):
        U.zero()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        rep = h.steady(U, cfg=cfg)
        e1.record(stream)
        e1.synchronize()
        ts.append(e0.elapsed_time(e1))
    return h, U.download(), rep, float(np.median(ts))


def permuted_problem(rsd, bm, ctx, S, seed=7):
    """The S^3 Q1 Backward-Euler problem of the metric with its node numbers shuffled (seeded), so that
    the DOF numbering, which follows node order, scatters every row's columns: an unstructured-mesh
    matrix with no stencil slices.  K + M/dt assembled (dt = 1e-3)."""
    xyz, ien, rng = bm.block_mesh(3, [S] * 3, [0, 0, 0], [1, 1, 1], 1)
    nn = xyz.size // 3
    p = np.random.default_rng(seed).permutation(nn)          # new id of old node v is p[v]
    x2 = np.empty((nn, 3))
    x2[p] = xyz.reshape(nn, 3)
    h = rsd.Heat(ctx, rsd.Mesh(ctx, 3, 1, x2.reshape(-1), p[ien].astype(np.int64), rng), 2,
                 dirichlet={t: "0" for t in range(6)})
    h.assemble_matrix(1.0, 1.0 / 1e-3)
    return h


def time_spmv(ctx, stream, A, n, launches=20):
    """Average CUDA-event time (ms) of one FP64 and one FP32 SpMV over `launches` back-to-back launches
    (operands of n entries; the matrix is larger than L2, so it streams from HBM every launch)."""
    import torch
    x, y = ctx.to_device(np.cos(np.arange(n) * 0.37)), ctx.array(n)
    x32, y32 = ctx.to_device(np.cos(np.arange(n) * 0.37), np.float32), ctx.array(n, np.float32)
    A.sync_f32()
    out = {}
    for key, f in (("fp64", lambda: A.spmv(x, y)), ("fp32", lambda: A.spmv_f32(x32, y32))):
        for _ in range(3):
            f()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(launches):
            f()
        e1.record(stream)
        e1.synchronize()
        out[key] = e0.elapsed_time(e1) / launches
    return out


def run_unstructured_spmv(rsd, bm, ctx, stream, heat, S, peak):
    """SpMV on the metric's matrix (stencil slices) and on the same matrix with shuffled node numbers
    (16/32-bit column indices, gathered x): event-timed, with the CSR byte model (value + 4-byte column
    per entry, x read and y written once) and its fraction of the HBM peak."""
    hp = permuted_problem(rsd, bm, ctx, S)
    out = {"workload": f"{S}^3 Q1 K + M/dt, FP64 and FP32 SpMV, 20 launches each, structured vs node numbers shuffled (seed 7)"}
    for name, h in (("structured", heat), ("shuffled", hp)):
        t = time_spmv(ctx, stream, h.K, h.n)
        lay = h.K.layout()
        rec = {"n": h.n, "nnz": h.nnz, "stencil_slices": lay["stencil_slices"], "slices": lay["slices"],
               "sell_slots": lay["sell_slots"]}
        for key, ms in t.items():
            vb = 8 if key == "fp64" else 4
            model = h.nnz * (vb + 4) + 2 * h.n * vb
            rec[key] = {"us": 1e3 * ms, "csr_model_bytes": model, "csr_model_gbs": model / (ms * 1e-3) / 1e9,
                        "csr_model_frac": model / (ms * 1e-3) / 1e9 / peak}
        out[name] = rec
    out["note"] = ("csr_model counts 4-byte columns; the structured matrix's stencil slices read none, so its "
                   "model fraction overstates DRAM traffic (the DRAM-traffic figure is in the ncu summary)")
    del hp
    return out


def run_fem_operator(rsd, ctx, stream, S):
    """The matrix-free operator (operator type fem) against the assembled matrix on S^3 Q2 hexes: the
    whole steady stage both ways, and one operator product (sum-factorized element pass against the
    FP64 SpMV of the assembled K)."""
    import torch
    out = {"workload": f"{S}^3 Q2 hexes, k = 1, f = 10, T = 0 / 1 on x = 0 / 1, steady, CG + Jacobi FP64 to 1e-8"}
    sol = {}
    for key, op in (("csr", rsd.OP_CSR), ("fem", rsd.OP_FEM)):
        h, sol[key], rep, ms = fem_steady(rsd, ctx, stream, S, op)
        out[key] = {"ms": ms, "iterations": rep["iterations"], "converged": bool(rep["converged"]),
                    "true_residual_rel": rep["trueResidualRel"]}
    out["n_free"], out["nnz"], out["elements"] = h.n, h.nnz, S ** 3
    out["speedup_fem_vs_csr"] = out["csr"]["ms"] / out["fem"]["ms"]
    out["fem_vs_csr_max_rel_diff"] = float(np.max(np.abs(sol["fem"] - sol["csr"])) / np.max(np.abs(sol["csr"])))
    # one product each way, 20 back to back per event pair, median of 5
    v = ctx.to_device(np.random.default_rng(1).standard_normal(h.n))
    y = ctx.array(h.n)
    h.assemble_matrix(1.0, 0.0)

    def per_product(fn):
        ts = []
        for i in range(6):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(20):
                fn()
            e1.record(stream)
            e1.synchronize()
            if i:
                ts.append(e0.elapsed_time(e1) * 1e3 / 20)
        return float(np.median(ts))
    spmv_us = per_product(lambda: h.K.spmv(v, y))
    fem_us = per_product(lambda: h.assemble_vector(4, y, coef=0.0, operand=v))
    import ctypes
    rate = ctypes.c_double()
    rsd.check(rsd.lib().rsd_measure_fp64_rate(ctx.h, ctypes.byref(rate)))
    fp64_rate = rate.value   # TFLOP/s, measured on this GPU
    E = S ** 3
    # bytes: per element the 27 free rows (4 B) and the geometry record (64 B), the operand read and
    # the result written once; flops: about 693 multiply-adds per lane of the kernel (x contraction
    # 54, nine points of y/z contraction, flux and z back-projection 56 each, y/x back 135), 3 lanes
    # per element, counted as 2 flops each
    fem_bytes = E * (27 * 4 + 64) + 16 * h.n
    fem_flops = E * 3 * 693 * 2
    t_hbm = fem_bytes / (measured_peak_hbm()[0] * 1e3)
    t_fp64 = fem_flops / (fp64_rate * 1e6) if fp64_rate else None
    bound = max(t_hbm, t_fp64 or 0.0)
    out["product_us"] = {"csr_spmv_fp64": spmv_us, "fem_sum_factorized": fem_us, "speedup": spmv_us / fem_us}
    out["product_roofline"] = {"kernel": "k_apply_hex27_planes", "bytes": fem_bytes, "flops": fem_flops,
                               "hbm_us": t_hbm, "fp64_us": t_fp64, "bound": "fp64" if (t_fp64 or 0) > t_hbm else "hbm",
                               "roofline_us": bound, "achieved_us": fem_us, "frac": bound / fem_us,
                               "fp64_tflops": fp64_rate, "hbm_peak_gbs": measured_peak_hbm()[0],
                               "csr_bytes": h.nnz * 12 + 4 * (h.n + 1) + 16 * h.n,
                               "note": "three lanes per element, z contraction by shuffles; FP64 pipe is the bound"}
    return out


def fem_cpu_baseline(rsd, ctx, stream, m):
    """The reference's steady stage with operator type fem (FEMOperator + cg::Solver + Jacobi, 1 core)
    on an m^3 Q2 sample, beside this library's matrix-free stage on the same sample."""
    import oracle
    if not oracle.reference_available():
        return None
    r = oracle.Reference(3, 2, 3, [m] * 3, [0, 0, 0], [1, 1, 1], [0, 1], bc_kind=0, bc_val={0: 0.0, 1: 1.0},
                         src_kind=0, src_c=10.0)
    r.set_operator("fem")
    t0 = time.perf_counter()
    _, rep = r.steady(0, 1, 1e-8, 100000)
    cpu_ms = 1e3 * (time.perf_counter() - t0)
    _, _, drep, dev_ms = fem_steady(rsd, ctx, stream, m, rsd.OP_FEM)
    return {"value": cpu_ms, "unit": "ms", "cores": 1, "kind": "reference", "cg_iterations": rep["iterations"],
            "device_same_sample_ms": dev_ms, "device_iterations": drep["iterations"],
            "sample": f"the whole steady stage with the matrix-free operator on {m}^3 Q2 hexes ({r.n} rows) through "
                      f"the reference templates (oracle/_ref), 1 core; the device time is this library's on the same mesh"}


def fourier_theta(xyz, ien, npe, seed, modes=16, amp=0.5):
    """theta_e = sum_m amp sin(2 pi k_m . c_e + phi_m) at element centroids c_e; stream mt19937_64(seed),
    per mode the three integers k_m ~ U{1..4} and then phi_m ~ U[0, 2 pi)."""
    u = uniforms(mt19937_64_stream(seed, 4 * modes)).reshape(modes, 4)
    c = xyz.reshape(-1, 3)[ien.reshape(-1, npe)].mean(axis=1)
    th = np.zeros(len(c))
    for m in range(modes):
        k = 1 + np.floor(u[m, :3] * 4.0)
        th += amp * np.sin(2.0 * np.pi * (c @ k) + 2.0 * np.pi * u[m, 3])
    return th


def adjoint_cpu_baseline(rsd, ctx, stream, m):
    """One forward solve of the adjoint workload (k_e = exp(theta_e), f = 1, T = 0 on the boundary,
    CG + Jacobi to 1e-13) through the reference's own SteadyStage (oracle/_ref, 1 core) on an m^3
    sample, beside this library's forward solve on the same sample."""
    import torch
    import oracle
    from importlib import import_module
    if not oracle.reference_available():
        return None
    bm = import_module("residuum_solver_b200.blockmesh")
    xyz, ien, rg = bm.block_mesh(3, [m] * 3, [0, 0, 0], [1, 1, 1], 1)
    th = fourier_theta(xyz, ien, 8, 5)
    r = oracle.Reference(3, 1, 2, [m] * 3, [0, 0, 0], [1, 1, 1], list(range(6)), bc_kind=0, src_kind=0, src_c=1.0,
                         k_elem=np.exp(th))
    t0 = time.perf_counter()
    _, rep = r.steady(solver=0, precond=1, tol=1e-13, maxit=100000)
    cpu_ms = 1e3 * (time.perf_counter() - t0)
    h = rsd.Heat(ctx, rsd.Mesh(ctx, 3, 1, xyz, ien, rg), 2, src_expr="1", dirichlet={t: "0" for t in range(6)})
    cfg = rsd.SolverConfig.make(tol=1e-13, max_iters=100000)
    theta, T = ctx.to_device(th), ctx.array(h.n)
    ts = []
    for _ in range(3):
        T.zero()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        h.forward(theta, T, cfg)
        e1.record(stream)
        e1.synchronize()
        ts.append(e0.elapsed_time(e1))
    return {"value": cpu_ms, "unit": "ms", "cores": 1, "kind": "reference", "cg_iterations": rep["iterations"],
            "device_same_sample_ms": float(np.median(ts)),
            "sample": f"one forward solve (assembly, lift, CG + Jacobi to 1e-13) on {m}^3 Q1 hexes ({r.n} rows) through "
                      f"the reference templates (oracle/_ref), 1 core; the device time is this library's forward "
                      f"solve on the same mesh"}


def run_adjoint(rsd, ctx, stream, S, ndir):
    """Adjoint gradient on S^3 Q1 hexes: k_e = exp(theta_e) (16 seeded Fourier modes, seed 5), f = 1,
    T = 0 on the boundary, J = 0.5 ||T(theta) - T_obs||^2 over the free nodes with T_obs from a second
    theta (seed 55); forward and adjoint CG + Jacobi to 1e-13; central differences (h = 1e-6) along
    `ndir` directions d ~ N(0, 1) per element (seed 555, Box-Muller), normalised."""
    import torch
    from importlib import import_module
    bm = import_module("residuum_solver_b200.blockmesh")
    xyz, ien, rg = bm.block_mesh(3, [S] * 3, [0, 0, 0], [1, 1, 1], 1)
    h = rsd.Heat(ctx, rsd.Mesh(ctx, 3, 1, xyz, ien, rg), 2, src_expr="1", dirichlet={t: "0" for t in range(6)})
    ne, n = S ** 3, h.n
    th = fourier_theta(xyz, ien, 8, 5)
    cfg = rsd.SolverConfig.make(tol=1e-13, max_iters=100000)
    Tobs = ctx.array(n).zero()
    h.forward(ctx.to_device(fourier_theta(xyz, ien, 8, 55)), Tobs, cfg)
    tobs = Tobs.download()
    theta, T, grad, dJdT = ctx.to_device(th), ctx.array(n), ctx.array(ne), ctx.array(n)
    times = []
    for _ in range(3):
        T.zero()
        e0, e1, e2, e3 = (torch.cuda.Event(enable_timing=True) for _ in range(4))
        e0.record(stream)
        rf = h.forward(theta, T, cfg)
        e1.record(stream)
        dJdT.upload(T.download() - tobs)
        e2.record(stream)
        rb = h.backward(theta, T, dJdT, grad, cfg)
        e3.record(stream)
        e3.synchronize()
        times.append((e0.elapsed_time(e1), e2.elapsed_time(e3)))
    g = grad.download()
    u = uniforms(mt19937_64_stream(555, 2 * ne * ndir)).reshape(ndir, ne, 2)
    dirs = np.sqrt(-2.0 * np.log1p(-u[..., 0])) * np.cos(2.0 * np.pi * u[..., 1])
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)

    # central differences J(th + h d) - J(th - h d) from the increments delta = T(th +- h d) - T(th),
    # solved directly: K(th +- h d) delta = -(K(th +- h d) - K(th)) T, the right-hand side being the
    # diffusion operator of the conductivity differences k_e (exp(+-h d_e) - 1) applied to T.  Nothing
    # is formed as a difference of two nearly equal solutions (T+ - T- loses about cond(K) eps / h of
    # its digits at this conductivity contrast), and T + delta solves the perturbed system exactly
    # when T solves the base one; then
    #   J(th + h d) - J(th - h d) = 0.5 sum (d+ - d-) (d+ + d- + 2 (T - T_obs))
    t_base = T.download()
    ke = np.exp(th)
    v, dl = ctx.array(n), ctx.array(n)
    hstep = 1e-6

    def increment(d, sgn):
        h.set_k_elem(ctx.to_device(ke * np.expm1(sgn * hstep * d)))
        h.assemble_vector(1, v, U=T)
        h.set_k_elem(ctx.to_device(ke * np.exp(sgn * hstep * d)))
        h.assemble_matrix(1.0)
        rhs = ctx.to_device(-v.download())
        dl.zero()
        rsd.solve(ctx, h.K, rhs, dl, cfg)
        return dl.download()

    errs = []
    for d in dirs:
        dp, dm = increment(d, 1.0), increment(d, -1.0)
        fd = 0.5 * float(np.sum((dp - dm) * (dp + dm + 2.0 * (t_base - tobs)))) / (2.0 * hstep)
        errs.append(abs(fd - g @ d) / abs(fd))
    h.set_k_elem(ctx.to_device(ke))
    # the same directional derivatives without differencing (tangent-linear solve):
    # K dT = -(dK/dtheta . d) T, with (dK/dtheta . d) T the diffusion operator of the element
    # multipliers k_e d_e applied to T; dJ . d = (T - T_obs) . dT
    dT = ctx.array(n)
    terrs = []
    for d in dirs:
        h.set_k_elem(ctx.to_device(ke * d))
        h.assemble_vector(1, v, U=T)
        h.set_k_elem(ctx.to_device(ke))
        h.assemble_matrix(1.0)
        rhs = ctx.to_device(-v.download())
        dT.zero()
        rsd.solve(ctx, h.K, rhs, dT, cfg)
        tl = float((t_base - tobs) @ dT.download())
        terrs.append(abs(tl - g @ d) / abs(tl))
    fwd, bwd = (float(np.median([t[i] for t in times])) for i in (0, 1))
    return {"workload": f"{S}^3 Q1 hexes, k_e = exp(theta_e), J = 0.5||T - T_obs||^2, CG + Jacobi 1e-13",
            "n_free": n, "elements": ne, "forward_ms": fwd, "backward_ms": bwd,
            "forward_iterations": rf["iterations"], "adjoint_iterations": rb["iterations"],
            "fd_directions": ndir, "fd_max_rel_error": max(errs), "fd_median_rel_error": float(np.median(errs)),
            "tangent_linear_max_rel_error": max(terrs), "tangent_linear_median_rel_error": float(np.median(terrs))}


def run_transient_adjoint(rsd, ctx, stream, S, nsteps, ndir, cpu):
    """Transient adjoint on S^3 Q1 hexes: k_e = exp(theta_e) (16 seeded Fourier modes, seed 5), f = 1,
    T = 0 on the boundary, nsteps Backward-Euler steps of dt = 1e-3 from the sine-mode T0 (seed 2),
    J = 0.5 ||U_N - U_obs||^2 with U_obs = T0 / 2; CG + Jacobi to 1e-14.  The adjoint gradient against
    central differences (h = 1e-6) along `ndir` directions through the device steps, and against the FP64
    CPU adjoint on the reference's templates (oracle.ref_transient_adjoint) when `cpu`."""
    import torch
    from importlib import import_module
    bm = import_module("residuum_solver_b200.blockmesh")
    xyz, ien, rg = bm.block_mesh(3, [S] * 3, [0, 0, 0], [1, 1, 1], 1)
    h = rsd.Heat(ctx, rsd.Mesh(ctx, 3, 1, xyz, ien, rg), 2, src_expr="1", dirichlet={t: "0" for t in range(6)})
    ne, n, dt = S ** 3, h.n, 1e-3
    th = fourier_theta(xyz, ien, 8, 5)
    t2a, a2t = h.dofmap()
    u0 = initial_condition(xyz, a2t)
    uobs = 0.5 * u0
    cfg = rsd.SolverConfig.make(tol=1e-14, max_iters=100000)
    theta, U0, U, grad, dJdU = ctx.to_device(th), ctx.to_device(u0), ctx.array(n), ctx.array(ne), ctx.array(n)
    times = []
    for _ in range(3):
        e0, e1, e2, e3 = (torch.cuda.Event(enable_timing=True) for _ in range(4))
        e0.record(stream)
        rf = h.transient_forward(theta, U0, U, 0.0, dt, nsteps, cfg)
        e1.record(stream)
        dJdU.upload(U.download() - uobs)
        e2.record(stream)
        rb = h.transient_backward(theta, U0, dJdU, grad, 0.0, dt, nsteps, cfg)
        e3.record(stream)
        e3.synchronize()
        times.append((e0.elapsed_time(e1), e2.elapsed_time(e3)))
    g = grad.download()
    u = uniforms(mt19937_64_stream(555, 2 * ne * ndir)).reshape(ndir, ne, 2)
    dirs = np.sqrt(-2.0 * np.log1p(-u[..., 0])) * np.cos(2.0 * np.pi * u[..., 1])
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    hstep = 1e-6
    Ut = ctx.array(n)

    def J(t):
        h.transient_forward(ctx.to_device(t), U0, Ut, 0.0, dt, nsteps, cfg)
        return 0.5 * float(np.sum((Ut.download() - uobs) ** 2))
    errs = []
    for d in dirs:
        fd = (J(th + hstep * d) - J(th - hstep * d)) / (2 * hstep)
        errs.append(abs(fd - g @ d) / abs(fd))
    # the same with h = 1e-4: central differences' truncation error grows as h^2 while the forward
    # solves' 1e-14 stopping noise, divided by 2h, shrinks; at this size h = 1e-6 is noise-limited
    errs4 = []
    for d in dirs:
        fd = (J(th + 1e-4 * d) - J(th - 1e-4 * d)) / 2e-4
        errs4.append(abs(fd - g @ d) / abs(fd))
    fwd, bwd = (float(np.median([t[i] for t in times])) for i in (0, 1))
    out = {"workload": f"{S}^3 Q1 hexes, k_e = exp(theta_e), {nsteps} Backward-Euler steps dt = {dt}, J = 0.5||U_N - U_obs||^2, "
                       f"CG + Jacobi 1e-14",
           "n_free": n, "elements": ne, "forward_ms": fwd, "backward_ms": bwd, "states_held": rb["states_held"],
           "forward_iterations": rf["iterations"], "adjoint_iterations": rb["iterations"],
           "forward_iterations_in_backward": rb["refinements"], "fd_directions": ndir, "fd_max_rel_error": max(errs),
           "fd_median_rel_error": float(np.median(errs)), "fd_h1e-4_max_rel_error": max(errs4),
           "fd_h1e-4_median_rel_error": float(np.median(errs4))}
    if cpu:
        import oracle
        if oracle.reference_available():
            t0 = time.perf_counter()
            uN, Jr, gr, its = oracle.ref_transient_adjoint([S] * 3, th, u0, dt, nsteps, uobs, tol=1e-14)
            out["cpu_adjoint"] = {"ms": 1e3 * (time.perf_counter() - t0), "cores": 1, "kind": "reference",
                                  "max_rel_diff_gradient": float(np.max(np.abs(g - gr)) / np.max(np.abs(gr))),
                                  "max_rel_diff_state": float(np.max(np.abs(U.download() - uN)) / np.max(np.abs(uN))),
                                  "how": "forward steps by the reference's BackwardEulerStage, adjoint solves by its cg::Solver + "
                                         "Jacobi on its K + M/dt, element terms by its DiffusionForm (oracle/_ref), 1 core"}
    return out


METRIC = "time to a 1e-8 FP64-checked relative residual per Backward-Euler step, mixed FP32/FP64 CG+Jacobi (FP64 CG alongside)"
WORKLOAD = ("3D transient heat, unit cube, {S}^3 Q1 hexes, k = rho*cp = 1, Backward Euler dt = 1e-3, "
            "T0 = 8 seeded sine modes (amplitude 0.1, seed 2), Dirichlet T = 0 on all faces")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--size", type=int, default=128)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--ref-steps", type=int, default=2, help="reference Backward-Euler steps the reference arm times")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--reliable-delta", type=float, default=0.0)
    ap.add_argument("--batch", type=int, default=256, help="problems in the batched workload (0: skip it)")
    ap.add_argument("--newton", type=int, default=48, help="Q2 mesh size of the Newton workload (0: skip it)")
    ap.add_argument("--adjoint", type=int, default=96, help="mesh size of the adjoint workload (0: skip it)")
    ap.add_argument("--fem", type=int, default=48, help="Q2 mesh size of the matrix-free operator workload (0: skip it)")
    ap.add_argument("--fd-directions", type=int, default=20)
    ap.add_argument("--transient-adjoint", type=int, default=48, help="mesh size of the transient adjoint workload (0: skip it)")
    ap.add_argument("--transient-steps", type=int, default=10)
    ap.add_argument("--only", choices=["mixed", "fp64", "fem-product", "spmv-shuffled", "batch", "newton"], default=None,
                    help="run one solver path only (no e2e, no CPU leg), 4 matrix-free products on the "
                         "--fem Q2 mesh, 4 FP64 + 4 FP32 SpMV on the --size matrix with shuffled node "
                         "numbers, the batched workload of --batch problems (2 mixed and 2 FP64 batch "
                         "solves), or one mixed Newton solve of the --newton workload: for profiler captures")
    ap.add_argument("--unstructured", type=int, default=1, help="time SpMV on the shuffled-node matrix too (0: skip it)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        run_reference_arm(args, rank, world)
        return

    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    rsd = load_package()
    from importlib import import_module
    bm = import_module("residuum_solver_b200.blockmesh")
    ctx = rsd.Context(local)
    stream = torch.cuda.ExternalStream(ctx.stream(), device=local)

    if args.only == "fem-product":
        # the matrix-free workload's problem and 4 operator products on a seeded operand
        F = args.fem
        xq, iq, rq = bm.block_mesh(3, [F] * 3, [0, 0, 0], [1, 1, 1], 2)
        hq = rsd.Heat(ctx, rsd.Mesh(ctx, 3, 2, xq, iq, rq), 3, src_expr="10", dirichlet={0: "0", 1: "1"})
        v = ctx.to_device(np.random.default_rng(1).standard_normal(hq.n))
        y = ctx.array(hq.n)
        for _ in range(4):
            hq.assemble_vector(4, y, coef=0.0, operand=v)
        ctx.sync()
        if rank == 0:
            print(json.dumps({"only": args.only, "n_free": hq.n, "elements": F ** 3}))
        del hq
        ctx.close()
        if dist is not None:
            dist.destroy_process_group()
        return

    if args.only == "newton":
        S = args.newton
        xq, iq, rq = bm.block_mesh(3, [S] * 3, [0, 0, 0], [1, 1, 1], 2)
        hq = rsd.Heat(ctx, rsd.Mesh(ctx, 3, 2, xq, iq, rq), 3, k_expr="1 + 0.5*T", dk_expr="0.5", src_expr="10",
                      dirichlet={0: "0", 1: "1"})
        U = ctx.array(hq.n).zero()
        cfg = rsd.SolverConfig.make(type=rsd.GMRES, krylov_dim=30, tol=1e-12, max_iters=100000, precision=rsd.MIXED)
        rep = hq.newton(U, 1e-10, 1e-10, 50, cfg)
        ctx.sync()
        if rank == 0:
            print(json.dumps({"only": args.only, "n_free": hq.n, "newton_iterations": rep["iterations"],
                              "gmres_iterations_total": rep["refinements"], "converged": bool(rep["converged"])}))
        del hq
        ctx.close()
        if dist is not None:
            dist.destroy_process_group()
        return

    if args.only == "batch":
        out = run_batch(rsd, ctx, stream, args.batch, 1, measured_peak_hbm()[0])
        if rank == 0:
            print(json.dumps({"only": args.only, **{k: out[k] for k in ("problems", "rows", "nnz")},
                              **{k: {kk: out[k][kk] for kk in ("ms", "iterations_max", "all_converged")} for k in ("mixed", "fp64")}}))
        ctx.close()
        if dist is not None:
            dist.destroy_process_group()
        return

    if args.only == "spmv-shuffled":
        hp = permuted_problem(rsd, bm, ctx, args.size)
        time_spmv(ctx, stream, hp.K, hp.n, launches=1)
        if rank == 0:
            print(json.dumps({"only": args.only, "n_free": hp.n, "nnz": hp.nnz, **hp.K.layout()}))
        del hp
        ctx.close()
        if dist is not None:
            dist.destroy_process_group()
        return

    S = args.size
    xyz, ien, rng = bm.block_mesh(3, [S, S, S], [0, 0, 0], [1, 1, 1], 1)
    mesh = rsd.Mesh(ctx, 3, 1, xyz, ien, rng)
    heat = rsd.Heat(ctx, mesh, 2, k_const=1.0, rho=1.0, cp=1.0, dirichlet={t: "0" for t in range(6)})
    n, nnz = heat.n, heat.nnz
    t2a, a2t = heat.dofmap()
    U0 = initial_condition(xyz, a2t)
    U, Up = ctx.array(n), ctx.array(n)
    dt = 1e-3
    cfgs = {
        "mixed": rsd.SolverConfig.make(type=rsd.CG, precond=rsd.JACOBI, precision=rsd.MIXED, tol=1e-8, max_iters=100000,
                                       reliable_delta=args.reliable_delta),
        "fp64": rsd.SolverConfig.make(type=rsd.CG, precond=rsd.JACOBI, precision=rsd.FP64, tol=1e-8, max_iters=100000),
    }

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
            torch.cuda.synchronize()

    def run(cfg, steps, warmup, profile=False, clocks=None):
        U.upload(U0); Up.upload(U0)
        heat.set_time(0.0)
        for _ in range(warmup):
            heat.be_step(dt, U, Up, cfg)
        reps = []
        if profile:
            ctx.profile(True)
        barrier()
        if clocks:
            clocks.start()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            reps.append(heat.be_step(dt, U, Up, cfg))
        e1.record(stream)
        e1.synchronize()
        clk = clocks.stop() if clocks else None
        barrier()
        ms = e0.elapsed_time(e1) / steps
        prof = {}
        if profile:
            for fam in ("cg_persist", "spmv_dot_f32", "spmv_dot_f64", "cg_update", "cg_pupdate", "reliable_update",
                        "assemble_matrix", "assemble_vector"):
                prof[fam] = ctx.profile_get(fam)
            ctx.profile(False)
        return ms, reps, prof, clk

    clocks = ClockSampler(local)
    if args.only:
        ms, reps, prof, _ = run(cfgs[args.only], args.steps, args.warmup, profile=False)
        if rank == 0:
            print(json.dumps({"only": args.only, "ms_per_step": ms, "iterations": [r["iterations"] for r in reps],
                              "true_residual_rel": [r["trueResidualRel"] for r in reps]}))
        del heat, mesh
        ctx.close()
        if dist is not None:
            dist.destroy_process_group()
        return
    # timed: the mixed solves run as one persistent kernel each (the FP64 ones as cached CUDA graphs);
    # then the same steps once more with event timing around each kernel family (the persistent
    # kernel, the assembly), and once with the mixed iteration as one kernel per phase (plain
    # launches) for the phase breakdown
    ms_mx, reps_mx, _, clk = run(cfgs["mixed"], args.steps, args.warmup, clocks=clocks)
    ms_64, reps_64, _, clk64 = run(cfgs["fp64"], args.steps, args.warmup, clocks=ClockSampler(local))
    _, reps_pr, prof_mx, _ = run(cfgs["mixed"], args.steps, args.warmup, profile=True)
    os.environ["RSD_CG_PERSIST"] = "0"
    _, _, prof_ph, _ = run(cfgs["mixed"], args.steps, args.warmup, profile=True)
    del os.environ["RSD_CG_PERSIST"]
    _, _, prof_64, _ = run(cfgs["fp64"], args.steps, args.warmup, profile=True)

    # time to the FP64-checked 1e-8 residual of the first step's system alone: K + M/dt, b = M U0 / dt,
    # warm start x0 = U0; median of 5 solves per precision, each from the same x0
    heat.assemble_matrix(1.0, 1.0 / dt)
    b = ctx.array(n)
    U.upload(U0)
    heat.assemble_vector(2, b, U=U)
    rsd.check(rsd.lib().rsd_scal(ctx.h, n, 1.0 / dt, b.ptr))
    x = ctx.array(n)
    solve_t, solve_it, solve_tr = {}, {}, {}
    for key in ("mixed", "fp64"):
        ts = []
        for rep_i in range(7):
            rsd.check(rsd.lib().rsd_copy(ctx.h, n, U.ptr, x.ptr))
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            r = rsd.solve(ctx, heat.K, b, x, cfgs[key])
            e1.record(stream)
            e1.synchronize()
            if rep_i >= 2:
                ts.append(e0.elapsed_time(e1))
        solve_t[key] = float(np.median(ts))
        solve_it[key] = r["iterations"]
        solve_tr[key] = r["trueResidualRel"]

    unstructured = None
    if args.unstructured:
        unstructured = run_unstructured_spmv(rsd, bm, ctx, stream, heat, S, measured_peak_hbm()[0])

    batch = None
    if args.batch > 0:
        batch = run_batch(rsd, ctx, stream, args.batch, 3, measured_peak_hbm()[0], rank, world, dist, f"cuda:{local}",
                          cpu=not args.no_cpu)
    newton = run_newton(rsd, ctx, stream, args.newton) if args.newton > 0 else None
    if newton is not None and rank == 0 and world == 1 and not args.no_cpu:
        try:
            newton["cpu_baseline"] = newton_cpu_baseline(rsd, ctx, stream, 16)
        except Exception as e:  # noqa: BLE001
            newton["cpu_baseline"] = {"value": None, "sample": f"failed: {e}"}
    adjoint = run_adjoint(rsd, ctx, stream, args.adjoint, args.fd_directions) if args.adjoint > 0 else None
    if adjoint is not None and rank == 0 and world == 1 and not args.no_cpu:
        try:
            adjoint["cpu_baseline"] = adjoint_cpu_baseline(rsd, ctx, stream, 48)
        except Exception as e:  # noqa: BLE001
            adjoint["cpu_baseline"] = {"value": None, "sample": f"failed: {e}"}

    tadj = None
    if args.transient_adjoint > 0:
        tadj = run_transient_adjoint(rsd, ctx, stream, args.transient_adjoint, args.transient_steps, args.fd_directions,
                                     cpu=rank == 0 and world == 1 and not args.no_cpu)

    fem_op = None
    if args.fem > 0:
        fem_op = run_fem_operator(rsd, ctx, stream, args.fem)
        if rank == 0 and world == 1 and not args.no_cpu:
            try:
                fem_op["cpu_baseline"] = fem_cpu_baseline(rsd, ctx, stream, 16)
            except Exception as e:  # noqa: BLE001
                fem_op["cpu_baseline"] = {"value": None, "sample": f"failed: {e}"}

    # the configured run once: 50 steps from T0 with each solver, final states compared
    full_run = {}
    finals = {}
    for key in ("mixed", "fp64"):
        U.upload(U0); Up.upload(U0)
        heat.set_time(0.0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        reps50 = [heat.be_step(dt, U, Up, cfgs[key]) for _ in range(50)]
        e1.record(stream)
        e1.synchronize()
        finals[key] = U.download()
        full_run[key] = {"ms": e0.elapsed_time(e1), "all_converged": all(r["converged"] for r in reps50),
                         "iterations_total": int(sum(r["iterations"] for r in reps50)),
                         "max_true_residual_rel": max(r["trueResidualRel"] for r in reps50)}
    full_run["final_state_max_rel_diff"] = float(np.max(np.abs(finals["mixed"] - finals["fp64"])) / np.max(np.abs(finals["fp64"])))
    full_run["how"] = "50 Backward-Euler steps (dt = 1e-3) from T0, one CUDA-event pair around all of them, each solver"

    # end to end through the public API with host buffers: rsd_heat_be_step_host every step, which
    # uploads the state from pinned host memory, steps (its previous state is the state it starts
    # from, as BackwardEulerRunner::step keeps Uprev = U between steps) and copies the new state back
    hU = torch.from_numpy(U0.copy()).pin_memory()
    heat.set_time(0.0)
    for _ in range(args.warmup):            # the first call also allocates the device state it keeps
        heat.be_step_host(dt, hU, cfgs["mixed"])
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        heat.be_step_host(dt, hU, cfgs["mixed"])
    e1.record(stream)
    e1.synchronize()
    barrier()
    ms_e2e = e0.elapsed_time(e1) / args.steps

    def reduce_max(v):
        return ranks_reduce(v, "max", dist, f"cuda:{local}")

    ms_mx, ms_64, ms_e2e = reduce_max(ms_mx), reduce_max(ms_64), reduce_max(ms_e2e)
    solve_t = {k: reduce_max(v) for k, v in solve_t.items()}

    # the mixed iteration's phases run one kernel each: the FP32 SpMV (+ z.w) dominates them
    launches, tot = prof_ph["spmv_dot_f32"]
    avg_ms = tot / max(launches, 1)
    bytes_spmv32 = nnz * (4 + 4) + 4 * (n + 1) + 2 * n * 4
    peak, peak_kind = measured_peak_hbm()
    achieved = bytes_spmv32 / (avg_ms * 1e-3) / 1e9 if launches else None
    l64, t64 = prof_64["spmv_dot_f64"]
    bytes_spmv64 = nnz * (8 + 4) + 4 * (n + 1) + 2 * n * 8
    achieved64 = bytes_spmv64 / ((t64 / max(l64, 1)) * 1e-3) / 1e9 if l64 else None
    traffic = ncu_traffic("k_mx_spmv_dot")

    it_mx = [r["iterations"] for r in reps_mx]
    it_64 = [r["iterations"] for r in reps_64]
    solve_mx = prof_mx["cg_persist"][1] / args.steps
    solve_64 = sum(prof_64[f][1] for f in ("spmv_dot_f64", "cg_update", "cg_pupdate")) / args.steps
    # kernels run in the timed mixed steps: per step 8 outside the solve loop (Udot, K + M/dt with its
    # FP32 copy, right-hand side, lift, inverse diagonal, initial residual, stage residual, its norm)
    # and the persistent solve kernel
    gpu_launches = int(9 * len(reps_mx))

    # the reference's own first step of the same workload (one core), timed on the host, and parity
    # at the configured size: the device's first step from T0 in FP64 and mixed precision against it
    cpu = None
    parity = None
    if rank == 0 and world == 1 and not args.no_cpu:
        first = {}
        for key in ("fp64", "mixed"):
            U.upload(U0); Up.upload(U0)
            heat.set_time(0.0)
            rep1 = heat.be_step(dt, U, Up, cfgs[key])
            first[key] = (U.download(), rep1)
        try:
            ref = reference_steps(S, 1)
            if ref is not None:
                step_ms = 1e3 * float(ref["step_s"][0])
                cpu = {"value": step_ms, "unit": "ms", "cores": 1, "kind": "reference",
                       "sample": (f"the first Backward-Euler step of the {S}^3 workload from T0 through the reference "
                                  f"templates (oracle/_ref: BackwardEulerRunner::step), 1 core; its linear solve "
                                  f"{1e3 * float(ref['solve_s'][0]):.0f} ms, {int(ref['iters'][0])} CG iterations; setup before "
                                  f"the step {ref['setup_s']:.1f} s untimed")}
                uref = ref["U"]
                scale = float(np.max(np.abs(uref)))
                parity = {"reference_iterations": int(ref["iters"][0]),
                          "initial_state_identical": bool(np.array_equal(ref["U0"], U0)),
                          "how": "one step from T0, the device's state against the reference's state after its first step, max |diff| / max |ref|"}
                for key in ("fp64", "mixed"):
                    ud, rp = first[key]
                    parity[key] = {"max_rel_diff_vs_reference": float(np.max(np.abs(ud - uref))) / scale,
                                   "iterations": int(rp["iterations"]), "true_residual_rel": rp["trueResidualRel"]}
                parity["fp64"]["iterations_equal"] = parity["fp64"]["iterations"] == parity["reference_iterations"]
        except Exception as e:  # noqa: BLE001
            cpu = {"value": None, "unit": "ms", "cores": 1, "kind": "reference", "sample": f"failed: {e}"}

    # element assembly roofline of K + M/dt.  The all-affine row-gather kernel (k_asm_matrix_rows) forms
    # each entry from the reference-element integrals: per (element, row a, column b) NT + 1 = 7
    # multiply-adds and one more add (3D), E npe^2 17 flops, so it is HBM-bound.  Its bytes: the SELL
    # values written once in FP64 and in FP32 (slots x 12), per (element, row) the adjacency entry (4)
    # and the column-rank record (8), per element the geometry record (64), the row pointers (n x 4).
    # The path's own byte count (CSR values + coordinates + connectivity) is given beside it.
    import ctypes
    fp64 = ctypes.c_double()
    rsd.check(rsd.lib().rsd_measure_fp64_rate(ctx.h, ctypes.byref(fp64)))
    n_elem, n_nodes = S ** 3, (S + 1) ** 3
    lay = heat.K.layout()
    slots = lay["sell_slots"]
    asm_bytes = slots * 12 + n_elem * 8 * (4 + 8) + n_elem * 64 + 4 * n
    path_bytes = nnz * 8 + n_nodes * 3 * 8 + n_elem * 8 * 4
    asm_flops = n_elem * 64 * 17
    t_hbm = asm_bytes / (peak * 1e9) * 1e3
    t_fp64 = asm_flops / (fp64.value * 1e12) * 1e3
    asm_ms = prof_mx["assemble_matrix"][1] / max(prof_mx["assemble_matrix"][0], 1) if "assemble_matrix" in prof_mx else None
    asm_roof = {"kernel": "k_asm_matrix_rows_q1 (K + M/dt with its FP32 copy, one launch per step)", "bound": "hbm",
                "bytes": asm_bytes, "flops": asm_flops, "hbm_ms": t_hbm, "fp64_ms": t_fp64,
                "achieved_ms": asm_ms, "achieved_gbs": asm_bytes / (asm_ms * 1e6) if asm_ms else None,
                "frac": t_hbm / asm_ms if asm_ms else None, "peak_gbs": peak, "peak_kind": peak_kind,
                "path_bytes": path_bytes, "fp64_tflops": fp64.value, "layout": lay,
                "note": "frac = kernel bytes / measured HBM copy peak / event-timed duration; the executed flops "
                        "(reference-element integrals) need %s of the duration at the measured FP64 rate; ncu: the "
                        "L1/tex pipe on the element-record loads bounds it (k_asm_matrix_rows_q1_96.md)"
                        % (f"{100 * t_fp64 / asm_ms:.0f}%" if asm_ms else "a fraction")}

    # the dominant kernel's roofline on the bytes it moves: DRAM traffic per launch from the ncu
    # capture of this workload (dram__bytes_read.sum + dram__bytes_write.sum) over the event-timed
    # average launch.  The path's algorithmic byte count charges 4-byte column indices, which the
    # stencil-slice layout does not read, and a gathered vector that stays in L2: its figure is kept
    # beside it as an equivalent rate, not as a fraction of the HBM roofline.
    if traffic and avg_ms:
        achieved_dram = traffic / (avg_ms * 1e6)
    else:
        achieved_dram = None
    # the timed region's dominant kernel: k_mx_persist, one launch per mixed solve.  Its DRAM traffic
    # per CG iteration (replacements included) from the ncu capture of this workload, times the
    # iterations of the profiled solves, over their event-timed launches
    persist = ncu_traffic("k_mx_persist") or {}
    pl, pt = prof_mx["cg_persist"]
    it_pr = float(np.mean([r["iterations"] for r in reps_pr])) if reps_pr else None
    per_iter = persist.get("bytes_per_launch", 0) / persist["iterations"] if persist.get("iterations") else None
    p_avg_ms = pt / max(pl, 1)
    p_traffic = per_iter * it_pr if per_iter and it_pr else None
    p_achieved = p_traffic / (p_avg_ms * 1e6) if p_traffic and pl else None
    alg_iter = bytes_spmv32 + 10 * n * 4   # the SpMV's algorithmic bytes + the vector pass's ten FP32 vectors
    roofline = {"kernel": "k_mx_persist (mixed CG: FP32 SELL-32 SpMV + z.w, vector pass, FP64 replacements)", "bound": "hbm",
                "achieved": p_achieved, "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                "frac": p_achieved / peak if p_achieved else None,
                "frac_nominal_8tbs": p_achieved / 8000.0 if p_achieved else None,
                "traffic": p_traffic, "avg_launch_us": p_avg_ms * 1e3, "launches": pl, "iterations_per_launch": it_pr,
                "traffic_per_iteration": per_iter, "traffic_source": persist.get("source"),
                "algorithmic_bytes": alg_iter * it_pr if it_pr else None,
                "algorithmic_equiv_gbs": alg_iter * it_pr / (p_avg_ms * 1e6) if it_pr and pl else None,
                "note": "achieved = ncu DRAM bytes per CG iteration x iterations of the profiled solves / "
                        "CUDA-event average launch time on the solve stream",
                "spmv_phase": {"kernel": "k_mx_spmv_dot (the SpMV phase as its own kernel)", "traffic": traffic,
                               "avg_launch_us": avg_ms * 1e3, "launches": launches,
                               "achieved": achieved_dram, "frac": achieved_dram / peak if achieved_dram else None,
                               "algorithmic_bytes": bytes_spmv32, "algorithmic_equiv_gbs": achieved,
                               "algorithmic_equiv_frac": achieved / peak if achieved else None},
                "fp64_spmv": {"kernel": "k_cg_spmv_dot", "traffic": ncu_traffic("k_cg_spmv_dot"),
                              "avg_launch_us": 1e3 * t64 / max(l64, 1),
                              "achieved": (ncu_traffic("k_cg_spmv_dot") / (t64 / max(l64, 1) * 1e6)) if ncu_traffic("k_cg_spmv_dot") and l64 else None,
                              "algorithmic_bytes": bytes_spmv64, "algorithmic_equiv_gbs": achieved64}}
    if roofline["fp64_spmv"]["achieved"]:
        roofline["fp64_spmv"]["frac"] = roofline["fp64_spmv"]["achieved"] / peak

    line = {
        "metric": METRIC, "value": ms_mx, "unit": "ms", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_mx, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32+f64", "data": "synthetic",
        "config": {"workload": WORKLOAD.format(S=S), "n_free": n, "nnz": nnz, "elements": S ** 3, "parallelism": "replicas",
                   "l2": "inputs larger than L2 (CSR FP64 values + columns %.2f GB)" % (nnz * 12 / 1e9)},
        "fp64_ms_per_step": ms_64,
        "speedup_mixed_vs_fp64_step": ms_64 / ms_mx,
        "time_to_1e8_solve_ms": {"mixed": solve_t["mixed"], "fp64": solve_t["fp64"],
                                 "speedup_mixed_vs_fp64": solve_t["fp64"] / solve_t["mixed"],
                                 "iterations": solve_it, "true_residual_rel": solve_tr,
                                 "how": "first step's system, x0 = U0 on the device, CUDA events around rsd_solve (graph, warm), median of 5"},
        "solve_kernel_ms_per_step": {"mixed": solve_mx, "fp64": solve_64},
        "iterations": {"mixed": it_mx, "fp64": it_64},
        "reliable_updates": [r["refinements"] for r in reps_mx],
        "true_residual_rel": {"mixed": max(r["trueResidualRel"] for r in reps_mx), "fp64": max(r["trueResidualRel"] for r in reps_64)},
        "roofline": roofline,
        "assembly_roofline": asm_roof,
        "kernel_ms_per_step": {k: v[1] / args.steps for k, v in prof_mx.items()},
        "phase_kernel_ms_per_step": {k: v[1] / args.steps for k, v in prof_ph.items()},
        "kernel_ms_per_step_fp64": {k: v[1] / args.steps for k, v in prof_64.items()},
        "clocks_fp64": clk64,
        "full_run_50_steps": full_run,
        "batch": batch,
        "newton": newton,
        "fem_operator": fem_op,
        "adjoint": adjoint,
        "transient_adjoint": tadj,
        "spmv_unstructured": unstructured,
        "cpu_baseline": cpu,
        "parity_at_size": parity,
        "e2e": {"value": ms_e2e, "unit": "ms", "h2d_bytes_per_step": 8 * n, "d2h_bytes_per_step": 8 * n},
        "gpu_launches": gpu_launches,
        "clocks": clk,
    }
    if rank == 0:
        print(json.dumps(line))
    del heat, mesh
    ctx.close()
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
