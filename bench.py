"""Benchmark: Wilson-clover propagator solves on one B200 (N GPUs = N replicas).

Workload (the configuration the headline metric is quoted on): SU(3) fundamental
Wilson-clover operator on a 24^3 x 48 lattice, kappa = 0.137, c_sw = 1.7, seeded
near-unit links U = exp(i 0.25 H), antiperiodic in time; 44 right-hand sides
(12 spin-colour point sources at the origin + 32 Z2 x Z2 noise sources).  One
step solves all 44 systems D x = b to a true residual ||b - D x|| / ||b|| <= 1e-10
with the block even-odd mixed-precision BiCGStab (FP32 batched stencil, FP64 reliable
updates, every solution re-measured with the FP64 operator).

Prints one JSON line (rank 0).  --impl reference times the reference's own solver,
compiled from its sources, on the host cores instead (see ReferenceCPU).
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import re
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

DIMS = (24, 24, 24, 48)
KAPPA, CSW, EPS, SEED = 0.137, 1.7, 0.25, 1237
N_POINT, N_NOISE = 12, 32
TOL = 1e-10
METRIC = "solves/s @24^3x48 to res 1e-10 (mixed vs FP64); dslash HBM GB/s; p50/p99 ms"
PEAKS_FALLBACK = {"hbm_gbs": 6650.0, "which": "fallback"}
# algorithmic bytes per output half-site of the Schur stencil kernel that carries the
# clover term (out_o = T_oo y_o - kappa^2 H_oe a_e): 8 links (+ 2 sign-table bytes for the
# reconstructed formats), 1 neighbour spinor (each read once), the y spinor, T_oo, the output
STENCIL_BYTES = {0: 8 * 144 + 3 * 192 + 576, 1: 8 * 48 + 2 + 3 * 96 + 288, 2: 8 * 24 + 2 + 3 * 52 + 144}
STENCIL_BYTES_8REAL = 8 * 32 + 2 + 3 * 96 + 288  # FP32 with SU(3) links in 8 reals
# the batched kernel reads links and T once per site for the whole batch, in FP32 for either
# spinor storage (links in 12 reals + 2 sign-table bytes, or in all 18 reals: the 8 padding
# bytes of the fifth word are not counted), and three spinors (neighbour, y, out) per
# right-hand side
STENCIL_SITE_BYTES = {12: 8 * 48 + 2 + 288, 18: 8 * 72 + 288}
STENCIL_RHS_BYTES = {1: 3 * 96, 2: 3 * 52}
STENCIL_FLOPS = 1320 + 504 + 48  # hopping + clover apply + xpay, per site


def log(msg):
    print(msg, file=sys.stderr, flush=True)


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return {"hbm_gbs": float(d["hbm_gbs"]), "which": "measured"}
    return PEAKS_FALLBACK


_LINKS = None
_SYNTH = None


def synth_module():
    """leonardym_b200/synth.py (seeded host generators, numpy only) loaded on its own, so
    that the reference arm draws the same inputs without importing the package."""
    global _SYNTH
    if _SYNTH is None:
        import importlib.util
        spec = importlib.util.spec_from_file_location("lym_synth_standalone",
                                                      os.path.join(ROOT, "leonardym_b200", "synth.py"))
        _SYNTH = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(_SYNTH)
    return _SYNTH


def workload_links():
    global _LINKS
    if _LINKS is None:
        _LINKS = synth_module().fermion_links(DIMS, "su3", EPS, SEED)
    return _LINKS


def workload_sources(nc=3):
    synth = synth_module()
    srcs = []
    for alpha in range(4):
        for c in range(nc):
            srcs.append(synth.point_source(DIMS, nc, alpha, c))
    for k in range(N_NOISE):
        srcs.append(synth.z2_source(DIMS, nc, SEED, stream=(1 << 21) + k))
    return srcs


# Serving workload (the configs' serving loop): 8 resident seeded fields, one per
# (volume, representation), requests in a seeded Poisson stream of mean rate
# SERVE_RATE with kappa uniform in the representation's range and 1-16 sources each.
SERVE_VOLUMES = [(8, 8, 8, 8), (12, 12, 12, 12), (16, 16, 16, 32), (24, 24, 24, 48)]
SERVE_RATE = 200.0
SERVE_KAPPA = {"su3": (0.12, 0.135), "su2adj": (0.17, 0.185)}
SERVE_CSW = {"su3": 1.7, "su2adj": 1.5}
SERVE_EPS = {"su3": 0.25, "su2adj": 0.3}
SERVE_POOL = 4  # distinct sources per field (reused across requests; every request gets its own solutions)


def _percentiles(lat):
    lat = sorted(lat)
    return {"p50": lat[len(lat) // 2], "p99": lat[min(len(lat) - 1, int(0.99 * len(lat)))]}


def serving_stream(srv, fields, pools, rate, window_s, seed):
    """Open loop: requests arrive for window_s seconds at Poisson times of mean rate `rate`
    (seeded) and are submitted as they arrive; returns the completed sources per second
    over the whole run, per-request latency p50 / p99 (submit to completion, the server's
    own clock) and the largest FP64 true residual."""
    rng = np.random.default_rng(seed)
    t, arrivals = 0.0, []
    while True:
        t += rng.exponential(1.0 / rate)
        if t > window_s:
            break
        key = int(rng.integers(len(fields)))
        rep = fields[key][1]
        arrivals.append((t, key, float(rng.uniform(*SERVE_KAPPA[rep])), int(rng.integers(1, 17))))
    tickets = []
    t0 = time.perf_counter()
    for (ta, key, kappa, nsrc) in arrivals:
        delay = t0 + ta - time.perf_counter()
        if delay > 0:
            time.sleep(delay)
        srcs = [pools[key][j % SERVE_POOL] for j in range(nsrc)]
        tickets.append(srv.submit(key, kappa, SERVE_CSW[fields[key][1]], srcs)[0])
    lat, worst, nsolved, failed = [], 0.0, 0, 0
    for tk in tickets:
        ok, st = srv.wait(tk, timeout=1800.0)
        lat.append(st.latency_s * 1e3)
        worst = max(worst, st.max_true_residual)
        nsolved += st.nsrc
        failed += 0 if ok else 1
    elapsed = time.perf_counter() - t0
    return {"requests": len(tickets), "sources": nsolved, "arrival_window_s": window_s,
            "offered_requests_per_s": rate, "elapsed_s": elapsed,
            "throughput_solves_per_s": nsolved / elapsed, "throughput_requests_per_s": len(tickets) / elapsed,
            "latency_ms": _percentiles(lat) if lat else None, "max_true_residual": worst, "failed_requests": failed}


SERVE_MEAN_SOURCES = 8.5  # mean of the uniform 1..16 sources per request
SERVE_LOADS = (0.25, 0.5, 0.9)


def run_serving(window_s, sweep_window_s, batch=16, precision="single", solver="bicgstab"):
    """The configs' serving loop on one server: 8 resident seeded fields (4 volumes x 2
    representations), each lane warmed by one request; then the configs' Poisson stream
    (200 requests/s) for window_s seconds, whose completion rate is the server's capacity
    on this mix; then the same mix offered at 25 %, 50 % and 90 % of that capacity for
    sweep_window_s seconds each, where the latency is that of batching, not of a queue."""
    from leonardym_b200.server import SolveServer
    synth = synth_module()
    fields = [(dims, rep) for dims in SERVE_VOLUMES for rep in ("su3", "su2adj")]
    srv = SolveServer(batch=batch, precision=precision, solver=solver)
    pools = {}
    try:
        for key, (dims, rep) in enumerate(fields):
            srv.add_gauge(key, dims, rep, synth.fermion_links(dims, rep, SERVE_EPS[rep], SEED + 4 * key))
            pools[key] = [synth.gaussian_spinor(dims, 3, SEED + 100 * key + j) for j in range(SERVE_POOL)]
        # one lane at a time, so that each lane's first batch (which tunes its batched
        # stencil) runs on an otherwise idle GPU
        for key, (dims, rep) in enumerate(fields):
            srv.wait(srv.submit(key, SERVE_KAPPA[rep][0], SERVE_CSW[rep], pools[key][:2])[0], timeout=1800.0)
        out = serving_stream(srv, fields, pools, SERVE_RATE, window_s, SEED + 7)
        capacity = out["throughput_solves_per_s"]
        sweep = []
        if sweep_window_s > 0:
            for k, f in enumerate(SERVE_LOADS):
                r = serving_stream(srv, fields, pools, f * capacity / SERVE_MEAN_SOURCES, sweep_window_s,
                                   SEED + 8 + k)
                r["load_fraction_of_capacity"] = f
                sweep.append(r)
    finally:
        srv.close()
    out.update({"fields": [f"{'x'.join(map(str, d))} {r}" for d, r in fields],
                "solver": f"{SOLVER_NAMES[solver]}, {batch} slots per field, {precision} storage, continuous batching",
                "capacity_solves_per_s": capacity, "load_sweep": sweep})
    return out


def run_serving_headline(links, srcs, batch=16, precision="single", solver="bicgstab", per_request=4):
    """The headline's 44 sources served through SolveServer on one resident 24^3x48 SU(3)
    field (kappa 0.137, c_sw 1.7): 11 requests of 4 sources submitted together after one
    warm-up request; served solves/s over the whole run and per-request latency."""
    from leonardym_b200.server import SolveServer
    srv = SolveServer(batch=batch, precision=precision, solver=solver)
    try:
        srv.add_gauge(0, DIMS, "su3", links)
        srv.wait(srv.submit(0, KAPPA, CSW, srcs[:per_request])[0], timeout=1800.0)
        t0 = time.perf_counter()
        tickets = [srv.submit(0, KAPPA, CSW, srcs[k:k + per_request])[0] for k in range(0, len(srcs), per_request)]
        lat, worst, n = [], 0.0, 0
        for tk in tickets:
            ok, st = srv.wait(tk, timeout=1800.0)
            if not ok:
                raise RuntimeError(f"headline serving request failed: status {st.status}")
            lat.append(st.latency_s * 1e3)
            worst = max(worst, st.max_true_residual)
            n += st.nsrc
        elapsed = time.perf_counter() - t0
    finally:
        srv.close()
    return {"requests": len(tickets), "sources": n, "elapsed_s": elapsed, "served_solves_per_s": n / elapsed,
            "latency_ms": _percentiles(lat), "max_true_residual": worst,
            "solver": f"{SOLVER_NAMES[solver]}, {batch} slots, {precision} storage, continuous batching"}


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = os.path.join("/tmp", f"lym_clocks_{os.getpid()}.csv")

    def start(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.f.close()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9 or parts[0] != str(self.index):
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def traffic_from_profiles(prec, batch, link_reals):
    """DRAM bytes per launch of the batched stencil kernel from the committed ncu summary."""
    for name in sorted(os.listdir(os.path.join(ROOT, "profiles"))):
        m = re.search(rf"traffic_bytes_per_launch\[prec={prec},kernel=xpay,batch={batch},links={link_reals}\]:"
                      rf"\s*([0-9.eE+]+)",
                      open(os.path.join(ROOT, "profiles", name)).read())
        if m:
            return float(m.group(1))
    return None


class quiet_stdout:
    """Silences C-level stdout (the reference prints solver progress with std::cout)."""

    def __enter__(self):
        sys.stdout.flush()
        self.saved = os.dup(1)
        self.null = os.open(os.devnull, os.O_WRONLY)
        os.dup2(self.null, 1)

    def __exit__(self, *a):
        os.dup2(self.saved, 1)
        os.close(self.saved)
        os.close(self.null)


# the reference's Schur-residual precision, in units of (1e-10 ||b||)^2, that gives a true
# residual <= 1e-10 on the benchmark's system (see ReferenceCPU)
REF_PRECISION_FACTOR = 7e-4


def host_threads():
    n = os.environ.get("OMP_NUM_THREADS")
    return int(n) if n else len(os.sched_getaffinity(0))


class ReferenceCPU:
    """The reference's own FP64 even-odd BiCGStab, PreconditionedBiCGStab::solve
    (inverters/PreconditionedBiCGStab.cpp:33-100), compiled from its sources into
    oracle/_ref, on the host cores (OpenMP, every thread this process may use), on the
    benchmark's lattice and its first Z2 x Z2 noise source.  The Improved operator is held
    across solves (field strength built once, as a caller solving many sources on one
    gauge field holds it); every solve then pays the reference's own per-solve set-up
    (the even-odd operators' field strength and 12x12 inverses) and its iterations.  The
    reference stops on the squared residual of its Schur system, ||r||^2 < precision,
    which is not the true residual of D x = b: at precision (1e-10 ||b||)^2 it stops after
    263 steps at a true residual of 3.3e-9.  To reach the same 1e-10 true residual as the
    GPU solves, precision is REF_PRECISION_FACTOR (1e-10 ||b||)^2 (measured: 286 steps,
    9.2e-11); the converged solve's true residual is re-measured with the reference's FP64
    Improved operator and, should it miss 1e-10, the factor is tightened and the solve
    repeated.  The -march=native build is used when a probe of it succeeds on this host,
    else the portable one."""

    def __init__(self):
        from oracle import ref as R
        self.build = "su3_native" if R.runs_here("su3_native") else "su3"
        self.links = workload_links()
        self.b = workload_sources()[N_POINT]
        self.precision = REF_PRECISION_FACTOR * (TOL ** 2) * float(np.vdot(self.b, self.b).real)
        self.ref = R.Reference(DIMS, self.links, self.build)
        t0 = time.perf_counter()
        with quiet_stdout():
            self.ref.bench_prepare(KAPPA, CSW)
        self.prepare_s = time.perf_counter() - t0
        self.cores = host_threads()

    def full_solve(self):
        """One solve to a true residual <= 1e-10: wall time, the reference's own
        getLastSteps(), the re-measured true residual (at most two tighter repeats)."""
        for _ in range(3):
            with quiet_stdout():
                t0 = time.perf_counter()
                rc, x, steps = self.ref.bench_solve(self.b, self.precision, 5000)
                seconds = time.perf_counter() - t0
                y = self.ref.multiply("Improved", x, KAPPA, CSW, False)
            res = float(np.linalg.norm(self.b - y) / np.linalg.norm(self.b))
            if res <= TOL or rc != 1:
                break
            self.precision *= 0.5 * (TOL / res) ** 2
        return {"seconds": seconds, "steps": steps, "converged": rc == 1, "true_residual": res,
                "solves_per_s": 1.0 / seconds,
                "precision_factor": self.precision / ((TOL ** 2) * float(np.vdot(self.b, self.b).real))}

    def sample(self, max_steps):
        """The same solve stopped after max_steps iterations (its set-up included)."""
        with quiet_stdout():
            t0 = time.perf_counter()
            self.ref.bench_solve(self.b, self.precision, max_steps, keep_solution=False)
            return time.perf_counter() - t0

    def close(self):
        self.ref.bench_release()


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(world, x):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


REF_SAMPLE_STEPS = 8  # iterations of one bounded sample of the reference solve


def run_reference(args, world, rank):
    """The reference arm: only the reference's own code (oracle/_ref), no GPU.  First one
    solve to convergence (its wall time, iteration count and re-measured true residual go
    into the line as full_solve); then every step is a bounded sample, the same solve
    stopped after REF_SAMPLE_STEPS iterations.  A step's solves/s is
    1 / (setup + steps x per-iteration time), with setup the solve stopped at 0 iterations
    (timed twice before the warm-up), the per-iteration time from the step's sample and
    steps the converged solve's own count."""
    if rank != 0:
        return
    ref = ReferenceCPU()
    try:
        full = ref.full_solve()
        if not full["converged"] or full["true_residual"] > TOL:
            log(f"reference: solve did not reach the tolerance: {full}")
        setup = min(ref.sample(0) for _ in range(2))
        per_solve, sample_s = [], []
        for s in range(args.warmup + args.steps):
            t = ref.sample(REF_SAMPLE_STEPS)
            if s >= args.warmup:
                sample_s.append(t)
                per_solve.append(setup + full["steps"] * max(t - setup, 0.0) / REF_SAMPLE_STEPS)
    finally:
        ref.close()
    value = 1.0 / statistics.median(per_solve)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": 0,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": statistics.mean(sample_s) * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded)", "config": config_dict("reference-fp64-eo-bicgstab (PreconditionedBiCGStab)"),
        "full_solve": {**full, "build": ref.build, "cores": ref.cores},
        "cpu_baseline": {"value": value, "unit": "solves/s", "cores": ref.cores, "kind": "reference",
                         "sample": (f"the reference's PreconditionedBiCGStab::solve (oracle/_ref {ref.build} build) on "
                                    f"the 24^3x48 system of the first Z2 source: one converged solve "
                                    f"({full['seconds']:.1f} s, {full['steps']} steps by its getLastSteps(), true "
                                    f"residual {full['true_residual']:.2e}), then per step the same solve stopped "
                                    f"after {REF_SAMPLE_STEPS} iterations ({statistics.mean(sample_s):.2f} s; set-up "
                                    f"{setup:.2f} s), scaled to the converged solve's {full['steps']} steps")},
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def block_solver(args):
    """The solver id of the block solves: mixed-precision even-odd CG on (gamma5 S)^2 or
    BiCGStab on S, with single (FP32) or half (FP16 + norms) inner storage."""
    from leonardym_b200 import solvers as S
    return {("cg", "single"): S.SOLVER_EO_CG_MIXED_SINGLE, ("cg", "half"): S.SOLVER_EO_CG_MIXED_HALF,
            ("bicgstab", "single"): S.SOLVER_EO_BICGSTAB_MIXED_SINGLE,
            ("bicgstab", "half"): S.SOLVER_EO_BICGSTAB_MIXED_HALF}[(args.solver, args.precision)]


SOLVER_NAMES = {"cg": "block even-odd CG on (gamma5 S)^2", "bicgstab": "block even-odd BiCGStab on S"}


ENGINE_KEYS = ("iterating_s", "reliable_updates_s", "adding_s", "collecting_s", "graph_replays", "pauses",
               "reliable_updates", "batch_iterations", "slot_iterations")


def engine_stats(lib, ctx):
    out = (C.c_double * len(ENGINE_KEYS))()
    if lib.lym_context_engine_stats(ctx, out, len(ENGINE_KEYS)) != 0:
        raise RuntimeError("lym_context_engine_stats failed")
    return list(out)


def config_dict(solver):
    return {"workload": "su3-clover-24^3x48-kappa0.137-csw1.7-44rhs-tol1e-10", "lattice": "24x24x24x48",
            "representation": "SU(3) fundamental", "kappa": KAPPA, "csw": CSW, "links": "exp(i 0.25 H), seeded",
            "rhs": N_POINT + N_NOISE, "sources": "12 point + 32 Z2xZ2", "solver": solver, "tolerance": TOL,
            "l2": "inputs larger than L2: FP64 links 382 MB + FP32 links 127 MB + clover resident",
            "parallelism": "replicas (one independent solve stream per GPU)"}


def run_ours(args, world, rank, local):
    import torch

    import leonardym_b200 as L
    from leonardym_b200 import synth
    from leonardym_b200.solvers import SOLVER_EO_CG

    lib = L.lib()
    torch.cuda.set_device(local)
    solver = block_solver(args)
    sprec = 1 if args.precision == "single" else 2
    links = workload_links()
    srcs = workload_sources()
    nrhs = len(srcs)
    lat = L.Lattice(DIMS, "su3", device=local)
    op = L.ImprovedDiracWilsonOperator(lat, KAPPA, CSW, gamma5=False)
    op.setLattice(links)
    ctx, opid = lat.handle, op.op_id
    V = lat.V
    dev_src = torch.from_numpy(np.stack(srcs).view(np.float64).reshape(nrhs, V * 24)).to(f"cuda:{local}")
    dev_sol = torch.zeros_like(dev_src)
    torch.cuda.synchronize()  # the library's stream does not wait for torch's
    stats = L.SolveStats()
    bstats = (L.SolveStats * nrhs)()
    src_ptrs = (C.c_void_p * nrhs)(*[dev_src[k].data_ptr() for k in range(nrhs)])
    sol_ptrs = (C.c_void_p * nrhs)(*[dev_sol[k].data_ptr() for k in range(nrhs)])

    def check_block(rc, tag):
        if rc != 0:
            raise RuntimeError(f"{tag} block solve failed: {rc} {lib.lym_last_error(ctx)}")
        for k in range(nrhs):
            if bstats[k].true_residual > TOL:
                raise RuntimeError(f"{tag} solve {k}: true residual {bstats[k].true_residual:.3e} > {TOL}")

    def solve_all(record=None):
        rc = lib.lym_solve_block_device(ctx, opid, solver, -TOL, 20000, nrhs, src_ptrs, sol_ptrs, args.batch, bstats)
        check_block(rc, "device")
        if record is not None:
            for k in range(nrhs):
                record.append((bstats[k].seconds, bstats[k].iterations, bstats[k].true_residual))

    for _ in range(args.warmup):
        solve_all()
    sampler = ClockSampler(local)
    barrier(world)
    torch.cuda.synchronize()
    lib.lym_synchronize(ctx)
    launches0 = lib.lym_context_kernel_launches(ctx)
    eng0 = engine_stats(lib, ctx)
    sampler.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    rec = []
    for _ in range(args.steps):
        solve_all(rec)
    lib.lym_synchronize(ctx)
    ev1.record()
    torch.cuda.synchronize()
    clocks = sampler.stop()
    launches = int(lib.lym_context_kernel_launches(ctx) - launches0)
    eng = [(b - a) / args.steps for a, b in zip(eng0, engine_stats(lib, ctx))]
    elapsed = max_over_ranks(world, ev0.elapsed_time(ev1) / 1e3)
    barrier(world)
    value = world * nrhs * args.steps / elapsed
    lat_ms = sorted(r[0] * 1e3 for r in rec)
    iters = [r[1] for r in rec]

    # end to end through the host-buffer API, pinned host memory, copies inside the region
    nbytes = V * 24 * 8
    hsrc = [lib.lym_host_alloc(nbytes) for _ in range(nrhs)]
    hsol = [lib.lym_host_alloc(nbytes) for _ in range(nrhs)]
    for k in range(nrhs):
        C.memmove(hsrc[k], srcs[k].ctypes.data, nbytes)
    barrier(world)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    hsrc_ptrs = (C.c_void_p * nrhs)(*hsrc)
    hsol_ptrs = (C.c_void_p * nrhs)(*hsol)
    e0.record()
    for _ in range(args.steps):
        rc = lib.lym_solve_block(ctx, opid, solver, -TOL, 20000, nrhs, hsrc_ptrs, hsol_ptrs, args.batch, bstats)
        check_block(rc, "e2e")
    lib.lym_synchronize(ctx)
    e1.record()
    torch.cuda.synchronize()
    e2e_elapsed = max_over_ranks(world, e0.elapsed_time(e1) / 1e3)
    for p in hsrc + hsol:
        lib.lym_host_free(p)
    e2e_value = world * nrhs * args.steps / e2e_elapsed

    # plain FP64 single-RHS even-odd CG on the same systems (the comparison of the metric)
    t64 = []
    for k in (0, N_POINT):
        rc = lib.lym_solve_device(ctx, opid, SOLVER_EO_CG, -TOL, 20000, C.c_void_p(dev_src[k].data_ptr()),
                                  C.c_void_p(dev_sol[k].data_ptr()), None, C.byref(stats))
        t64.append(stats.seconds)
    fp64_value = world / statistics.mean(t64)

    # stencil roofline: CUDA events around launches of the dominant kernel (the batched
    # stencil of the block solve) on the library stream
    ms = C.c_double(0)
    lib.lym_time_stencil_batch(ctx, opid, sprec, 0, args.batch, 30, C.byref(ms))
    tby, tbz, tminb = C.c_int(), C.c_int(), C.c_int()
    if lib.lym_get_batch_tile(ctx, sprec, args.batch, 1, C.byref(tby), C.byref(tbz), C.byref(tminb)) != 0:
        raise RuntimeError(f"lym_get_batch_tile failed: {lib.lym_last_error(ctx)}")
    Vh = V // 2
    link_reals = 18 if tminb.value & 64 else 12
    bytes_launch = (STENCIL_SITE_BYTES[link_reals] + args.batch * STENCIL_RHS_BYTES[sprec]) * Vh
    achieved = bytes_launch / (ms.value * 1e-3) / 1e9
    pk = peaks()
    traffic = traffic_from_profiles(sprec, args.batch, link_reals)
    ms1, ms64, ms8 = C.c_double(0), C.c_double(0), C.c_double(0)
    lib.lym_time_stencil(ctx, opid, sprec, 0, 30, C.byref(ms1))
    lib.lym_time_stencil(ctx, opid, 0, 0, 20, C.byref(ms64))
    lib.lym_set_link_format(ctx, 8)
    lib.lym_time_stencil(ctx, opid, 1, 0, 30, C.byref(ms8))
    lib.lym_set_link_format(ctx, 12)

    cpu = None
    if rank == 0 and world == 1 and not args.skip_cpu:
        ref = ReferenceCPU()
        try:
            full = ref.full_solve()
        finally:
            ref.close()
        cpu = {"value": full["solves_per_s"], "unit": "solves/s", "cores": ref.cores, "kind": "reference",
               "sample": (f"one solve to convergence of the reference's PreconditionedBiCGStab::solve (oracle/_ref "
                          f"{ref.build} build) on this lattice and the first Z2 source: {full['seconds']:.1f} s, "
                          f"{full['steps']} steps by its getLastSteps(), true residual {full['true_residual']:.2e}")}
    # the propagator consumers of this workload's sources, after the timed region on their own
    # clock: MesonCorrelator (the 12 point sources) and ChiralCondensate (32 Z2 noise vectors)
    consumers = None
    if rank == 0:
        consumers = {}
        for name, fn in (("meson_correlator", lambda: L.MesonCorrelator(op, tolerance=TOL, batch=args.batch)),
                         ("chiral_condensate", lambda: L.ChiralCondensate(op, number_stochastic_estimators=N_NOISE,
                                                                          seed=SEED, tolerance=TOL,
                                                                          batch=args.batch))):
            t0 = time.perf_counter()
            res = fn().execute()
            consumers[f"{name}_s"] = time.perf_counter() - t0
            consumers[f"{name}_converged"] = bool(res["converged"])
        consumers["sources"] = {"meson_correlator": 12, "chiral_condensate": N_NOISE}
    lat.close()
    serving = serving24 = None
    if rank == 0 and args.serve_window > 0:  # after the timed region: its own clock
        serving = run_serving(args.serve_window, args.serve_sweep_window, batch=args.batch, precision=args.precision,
                              solver=args.solver)
        serving24 = run_serving_headline(links, srcs, batch=args.batch, precision=args.precision, solver=args.solver)
        serving24["served_over_fp64_eo_cg"] = serving24["served_solves_per_s"] / (fp64_value / world)
    if rank != 0:
        return
    line = {
        "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": elapsed / args.steps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32" if sprec == 1 else "f16",
        "data": "synthetic (seeded links and sources)",
        "config": config_dict(f"{SOLVER_NAMES[args.solver]}, {args.batch} right-hand sides per batched stencil, "
                              f"{args.precision} storage + FP64 reliable updates"),
        "fp64_eo_cg_solves_per_s": fp64_value,
        "mixed_over_fp64": value / world / (fp64_value / world),
        "latency_ms": {"p50": lat_ms[len(lat_ms) // 2], "p99": lat_ms[min(len(lat_ms) - 1, int(0.99 * len(lat_ms)))]},
        "iterations": {"median": statistics.median(iters), "max": max(iters)},
        "engine_per_step": dict({k: round(v, 4) for k, v in zip(ENGINE_KEYS, eng)},
                                batch_occupancy=round(eng[8] / (eng[7] * args.batch), 4) if eng[7] else None),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": pk["hbm_gbs"], "unit": "GB/s",
                     "frac": achieved / pk["hbm_gbs"], "traffic": traffic,
                     "kernel": (f"batched Schur stencil with clover, {args.batch} right-hand sides, "
                                f"{args.precision} storage, {ms.value * 1e3:.1f} us/launch"),
                     "algorithmic_bytes_per_launch": bytes_launch,
                     "variant": (f"column {tby.value}x{tbz.value}, "
                                 + ("staged (bulk copies)" if tminb.value & 32 else
                                    "staged (cp.async)" if tminb.value & 16 else "direct")
                                 + f" kernel, {tminb.value % 16} blocks/SM, "
                                 + ("18-real" if tminb.value & 64 else "12-real") + " links"),
                     "peak_source": f"{pk['which']} hbm_gbs",
                     "gflops": STENCIL_FLOPS * Vh * args.batch / (ms.value * 1e-3) / 1e9,
                     "single_rhs_kernel_gbs": STENCIL_BYTES[sprec] * Vh / (ms1.value * 1e-3) / 1e9,
                     "fp64_single_rhs_kernel_gbs": STENCIL_BYTES[0] * Vh / (ms64.value * 1e-3) / 1e9,
                     "single_rhs_kernel_8real_links_gbs": STENCIL_BYTES_8REAL * Vh / (ms8.value * 1e-3) / 1e9,
                     "single_rhs_kernel_us": {"fp32_12real": ms1.value * 1e3, "fp32_8real": ms8.value * 1e3,
                                              "fp64": ms64.value * 1e3}},
        "clocks": clocks,
        "gpu_launches": launches,
        "e2e": {"value": e2e_value, "unit": "solves/s", "h2d_bytes_per_step": nrhs * nbytes,
                "d2h_bytes_per_step": nrhs * nbytes},
        "cpu_baseline": cpu,
        "serving": serving,
        "serving_24c48": serving24,
        "consumers": consumers,
    }
    print(json.dumps(line), flush=True)


RHMC_DIMS = (48, 48, 48, 96)
RHMC_KAPPA, RHMC_CSW, RHMC_EPS, RHMC_SEED = 0.1365, 1.7, 0.25, 1239
RHMC_SHIFTS = list(np.logspace(-4, 0, 12))
RHMC_METRIC = "RHMC multishift solves/s @48^3x96, 12 shifts to res 1e-10 (FP16 inner vs FP64)"


def run_rhmc(args, world, rank, local, dims=RHMC_DIMS):
    """The configs' RHMC case: SU(3) Wilson-clover 48^3x96, kappa 0.1365, c_sw 1.7, 12 shifts
    log-spaced in [1e-4, 1] on the squared even-odd operator (the RHMC operator), every
    shift to a FP64 true residual 1e-10; one step = one multishift solve of one
    complex-normal source.  Links and source are seeded on the device (the host generator
    would take minutes at 10.6M sites)."""
    import torch

    import leonardym_b200 as L
    from leonardym_b200 import synth
    from leonardym_b200.solvers import MULTISHIFT

    lib = L.lib()
    torch.cuda.set_device(local)
    dev = f"cuda:{local}"
    prec = args.precision or "half"
    algo = MULTISHIFT[f"multishift_cg_mixed_{prec}"]
    lat = L.Lattice(dims, "su3", device=local)
    ctx = lat.handle
    links = synth.su3_fermion_links_device(dims, RHMC_EPS, RHMC_SEED, dev)
    if lib.lym_gauge_upload_device(ctx, 1, C.c_void_p(links.data_ptr())) != 0:
        raise RuntimeError(lib.lym_last_error(ctx))
    del links
    torch.cuda.empty_cache()
    opid = C.c_int(0)
    if lib.lym_operator_create(ctx, 1, 5, RHMC_KAPPA, RHMC_CSW, 1, C.byref(opid)) != 0:
        raise RuntimeError(lib.lym_last_error(ctx))
    opid = opid.value
    b = synth.gaussian_spinor_device(dims, 3, RHMC_SEED + 1, dev)
    bb = float(torch.vdot(b.flatten(), b.flatten()).real)
    eps = TOL * TOL * bb
    nsh = len(RHMC_SHIFTS)
    sh = np.ascontiguousarray(RHMC_SHIFTS, dtype=np.float64)
    sols = [torch.zeros_like(b) for _ in range(nsh)]
    torch.cuda.synchronize()  # the library's stream does not wait for torch's
    ptrs = (C.c_void_p * nsh)(*[x.data_ptr() for x in sols])
    st = L.SolveStats()

    def solve(algorithm=algo, src=b, out=ptrs, device=True):
        fn = lib.lym_multishift_device if device else lib.lym_multishift
        rc = fn(ctx, opid, algorithm, nsh, sh.ctypes.data_as(C.c_void_p), eps, 20000,
                C.c_void_p(src if isinstance(src, int) else src.data_ptr()), out, C.byref(st))
        if rc != 0:
            raise RuntimeError(f"multishift failed: {rc} {lib.lym_last_error(ctx)}")
        if st.true_residual > TOL:
            raise RuntimeError(f"multishift true residual {st.true_residual:.3e} > {TOL}")
        return st.seconds, st.steps, st.iterations

    for _ in range(args.warmup):
        log(f"rhmc: warm-up solve {solve()}")
    sampler = ClockSampler(local)
    barrier(world)
    torch.cuda.synchronize()
    lib.lym_synchronize(ctx)
    launches0 = lib.lym_context_kernel_launches(ctx)
    sampler.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    rec = [solve() for _ in range(args.steps)]
    lib.lym_synchronize(ctx)
    ev1.record()
    torch.cuda.synchronize()
    clocks = sampler.stop()
    launches = int(lib.lym_context_kernel_launches(ctx) - launches0)
    elapsed = max_over_ranks(world, ev0.elapsed_time(ev1) / 1e3)
    value = world * args.steps / elapsed

    # every shift's true residual, re-measured with the FP64 multiplyAdd of the operator
    out = torch.empty_like(b)
    worst = 0.0
    for x, s in zip(sols, RHMC_SHIFTS):
        lib.lym_multiply_add_device(ctx, opid, C.c_void_p(out.data_ptr()), C.c_void_p(x.data_ptr()),
                                    C.c_void_p(x.data_ptr()), float(s), 0.0)
        worst = max(worst, float(torch.linalg.vector_norm((b - out).flatten())) / np.sqrt(bb))
    if worst > 1.02 * TOL:
        raise RuntimeError(f"re-measured true residual {worst:.3e}")

    # end to end: pinned host source and solutions, copies inside the timed region
    nbytes = lat.V * 24 * 8
    log(f"rhmc: timed {args.steps} solves in {elapsed:.2f} s; end to end with pinned host buffers")
    hsrc = lib.lym_host_alloc(nbytes)
    hsol = [lib.lym_host_alloc(nbytes) for _ in range(nsh)]
    if not hsrc or not all(hsol):
        for p in [hsrc] + hsol:
            lib.lym_host_free(p)
        raise RuntimeError(f"pinned host allocation of {(nsh + 1) * nbytes / 1e9:.1f} GB failed")
    bh = b.cpu().numpy()
    C.memmove(hsrc, bh.ctypes.data, nbytes)
    del bh
    hptrs = (C.c_void_p * nsh)(*hsol)
    barrier(world)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        solve(src=hsrc, out=hptrs, device=False)
    lib.lym_synchronize(ctx)
    e1.record()
    torch.cuda.synchronize()
    e2e_value = world * args.steps / max_over_ranks(world, e0.elapsed_time(e1) / 1e3)
    for p in [hsrc] + hsol:
        lib.lym_host_free(p)

    # the RHMC consumers on the same system (RationalApproximation::evaluate and the solves of
    # NFlavorFermionAction::updateForce), device buffers, one call each after a warm-up call
    alphas = np.ascontiguousarray(np.linspace(0.05, 0.6, nsh)[::-1], dtype=np.float64)
    r_out = torch.empty_like(b)
    ys = [torch.empty_like(b) for _ in range(nsh)]
    yptrs = (C.c_void_p * nsh)(*[y.data_ptr() for y in ys])
    dop = C.c_int(0)
    lib.lym_operator_create(ctx, 1, 2, RHMC_KAPPA, RHMC_CSW, 1, C.byref(dop))
    consumer = {}
    for _ in range(2):
        t0 = time.perf_counter()
        if lib.lym_rational_evaluate_device(ctx, opid, algo, nsh, alphas.ctypes.data_as(C.c_void_p),
                                            sh.ctypes.data_as(C.c_void_p), eps, 20000, C.c_void_p(b.data_ptr()),
                                            C.c_void_p(r_out.data_ptr()), C.byref(st)) != 0:
            raise RuntimeError(lib.lym_last_error(ctx))
        consumer["rational_evaluate_s"] = time.perf_counter() - t0
        t0 = time.perf_counter()
        if lib.lym_rhmc_force_solves_device(ctx, opid, dop.value, algo, nsh, sh.ctypes.data_as(C.c_void_p), eps,
                                            20000, C.c_void_p(b.data_ptr()), ptrs, yptrs, C.byref(st)) != 0:
            raise RuntimeError(lib.lym_last_error(ctx))
        consumer["force_solves_s"] = time.perf_counter() - t0
    consumer["energy"] = float(torch.vdot(b.flatten(), r_out.flatten()).real)
    # the fermion force of one shift's (x, y) pair on the whole field (FermionForce::derivative)
    fop = C.c_int(0)
    lib.lym_operator_create(ctx, 1, 1, RHMC_KAPPA, RHMC_CSW, 1, C.byref(fop))
    force = torch.zeros((lat.V, 4, 3, 3), dtype=torch.complex128, device=dev)
    torch.cuda.synchronize()  # the library's stream does not wait for torch's
    for _ in range(2):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        if lib.lym_fermion_force_device(ctx, fop.value, C.c_void_p(sols[0].data_ptr()), C.c_void_p(ys[0].data_ptr()),
                                        float(alphas[0]), C.c_void_p(force.data_ptr())) != 0:
            raise RuntimeError(lib.lym_last_error(ctx))
        consumer["fermion_force_s"] = time.perf_counter() - t0
    # all 12 shifts' pairs in one pass (NFlavorFermionAction's sum over the shifts)
    for _ in range(2):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        if lib.lym_fermion_force_multi_device(ctx, fop.value, nsh, ptrs, yptrs, alphas.ctypes.data_as(C.c_void_p),
                                              C.c_void_p(force.data_ptr())) != 0:
            raise RuntimeError(lib.lym_last_error(ctx))
        consumer["fermion_force_12_pairs_s"] = time.perf_counter() - t0
    del ys, r_out, force
    torch.cuda.empty_cache()

    # the plain FP64 multishift CG on the same system (one solve)
    log("rhmc: FP64 multishift CG")
    fp64 = solve(algorithm=MULTISHIFT["multishift_cg"])
    # dominant kernel: the FP32 Schur stencil with the clover term of the shared Krylov phase
    sp = 1
    ms = C.c_double(0)
    lib.lym_time_stencil(ctx, opid, sp, 0, 30, C.byref(ms))
    Vh = lat.V // 2
    achieved = STENCIL_BYTES[sp] * Vh / (ms.value * 1e-3) / 1e9
    pk = peaks()
    lat.close()
    if rank != 0:
        return
    line = {
        "metric": RHMC_METRIC, "value": value, "unit": "multishift solves/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": elapsed / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (links and source seeded on the device)",
        "config": {"workload": "su3-clover-48^3x96-kappa0.1365-csw1.7-12shifts-tol1e-10",
                   "lattice": "x".join(str(d) for d in dims), "operator": "SquareEvenOddImproved (gamma5)",
                   "shifts": "12, log-spaced in [1e-4, 1]", "solver": f"multishift_cg_mixed_{prec}",
                   "l2": "inputs larger than L2: FP64 links 6.1 GB, spinors 2 GB each",
                   "parallelism": "replicas (one independent solve stream per GPU)"},
        "multishift_steps": [r[1] for r in rec], "total_iterations": [r[2] for r in rec],
        "worst_true_residual": worst,
        "rhmc_consumers": consumer,
        "fp64_multishift_cg_solves_per_s": 1.0 / fp64[0], "fp64_multishift_cg_iterations": fp64[2],
        "mixed_over_fp64": value / world * fp64[0],
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": pk["hbm_gbs"], "unit": "GB/s",
                     "frac": achieved / pk["hbm_gbs"], "traffic": None,
                     "kernel": (f"Schur stencil with clover, FP32 (shared Krylov phase), {ms.value * 1e3:.1f} "
                                f"us/launch"),
                     "algorithmic_bytes_per_launch": STENCIL_BYTES[sp] * Vh,
                     "peak_source": f"{pk['which']} hbm_gbs"},
        "clocks": clocks, "gpu_launches": launches,
        "e2e": {"value": e2e_value, "unit": "multishift solves/s", "h2d_bytes_per_step": nbytes,
                "d2h_bytes_per_step": nsh * nbytes},
        "cpu_baseline": None,
    }
    print(json.dumps(line), flush=True)


def run_profile(args):
    """Small fixed case for ncu captures: one block solve of the benchmark's first
    `batch` noise sources, then 10 launches each of the single-RHS and the batched
    stencil kernels (a few GB on the device)."""
    import leonardym_b200 as L
    lib = L.lib()
    if args.workload.startswith("rhmc"):
        return run_profile_rhmc(args)
    if args.workload == "consumers":
        return run_profile_consumers(args)
    lat = L.Lattice(DIMS, "su3", device=0)
    op = L.ImprovedDiracWilsonOperator(lat, KAPPA, CSW, gamma5=False)
    op.setLattice(workload_links())
    srcs = workload_sources()[N_POINT:N_POINT + args.batch]
    xs = [lat.new_vector() for _ in srcs]
    solver = block_solver(args)
    if args.tile:  # a fixed batched-stencil configuration instead of the autotuner's
        by, bz, minb = (int(v) for v in args.tile.split(","))
        lib.lym_set_batch_tile(lat.handle, by, bz, minb)
    bstats = (L.SolveStats * len(srcs))()
    sp_ = (C.c_void_p * len(srcs))(*[s.ctypes.data for s in srcs])
    xp_ = (C.c_void_p * len(srcs))(*[x.ctypes.data for x in xs])
    t0 = time.perf_counter()
    rc = lib.lym_solve_block(lat.handle, op.op_id, solver, -TOL, 20000, len(srcs), sp_, xp_, args.batch, bstats)
    t_solve = time.perf_counter() - t0
    st = bstats[0]
    ms = C.c_double(0)
    sp = 1 if args.precision == "single" else 2
    lib.lym_time_stencil(lat.handle, op.op_id, sp, 0, 10, C.byref(ms))
    msb, msc = C.c_double(0), C.c_double(0)
    lib.lym_time_stencil_batch(lat.handle, op.op_id, sp, 0, args.batch, 10, C.byref(msb))
    lib.lym_time_stencil_batch(lat.handle, op.op_id, sp, 1, args.batch, 10, C.byref(msc))
    tby, tbz, tminb = C.c_int(), C.c_int(), C.c_int()
    lib.lym_get_batch_tile(lat.handle, sp, args.batch, 1, C.byref(tby), C.byref(tbz), C.byref(tminb))
    print(f"profile case: rc {rc}, block solve {t_solve:.3f} s, updates {st.reliable_updates}, "
          f"iterations {st.iterations}, true residual {st.true_residual:.2e}, "
          f"stencil {ms.value * 1e3:.1f} us, batched stencil ({args.batch}) {msb.value * 1e3:.1f} us "
          f"(T^-1 half {msc.value * 1e3:.1f} us), tile {tby.value},{tbz.value},{tminb.value}")
    lat.close()
    if rc != 0:
        sys.exit(1)


def run_profile_consumers(args):
    """Small case for ncu captures of the consumer kernels on 24^3x48 (links and sources
    seeded on the device, a few GB on the device): one fermion force over 12 weighted pairs,
    the meson contractions of 12 spinors, the condensate dot products of 32 pairs."""
    import torch

    import leonardym_b200 as L
    from leonardym_b200 import synth
    lib = L.lib()
    lat = L.Lattice(DIMS, "su3", device=0)
    ctx = lat.handle
    links = synth.su3_fermion_links_device(DIMS, RHMC_EPS, RHMC_SEED, "cuda:0")
    lib.lym_gauge_upload_device(ctx, 1, C.c_void_p(links.data_ptr()))
    del links
    opid = C.c_int(0)
    lib.lym_operator_create(ctx, 1, 1, KAPPA, CSW, 0, C.byref(opid))
    vecs = [synth.gaussian_spinor_device(DIMS, 3, 100 + k, "cuda:0") for k in range(24)]
    X, Y = vecs[:12], vecs[12:]
    w = np.linspace(0.05, 0.6, 12)
    xp = (C.c_void_p * 12)(*[v.data_ptr() for v in X])
    yp = (C.c_void_p * 12)(*[v.data_ptr() for v in Y])
    force = torch.zeros((lat.V, 4, 3, 3), dtype=torch.complex128, device="cuda:0")
    torch.cuda.synchronize()  # the library's stream does not wait for torch's
    t0 = time.perf_counter()
    rc = lib.lym_fermion_force_multi_device(ctx, opid.value, 12, xp, yp, w.ctypes.data_as(C.c_void_p),
                                            C.c_void_p(force.data_ptr()))
    t_force = time.perf_counter() - t0
    Lt = DIMS[3]
    pion, scalar, ps = np.zeros(Lt), np.zeros(Lt), np.zeros(Lt)
    rc |= lib.lym_meson_contractions_device(ctx, xp, pion.ctypes.data, scalar.ctypes.data, ps.ctypes.data)
    d = np.zeros(2 * 12)
    rc |= lib.lym_dots_device(ctx, 12, xp, yp, 1, d.ctypes.data)
    print(f"consumers profile case: rc {rc}, fermion force (12 pairs) {t_force:.3f} s, pion[0] {pion[0]:.6e}")
    lat.close()
    if rc != 0:
        sys.exit(1)


def run_profile_rhmc(args):
    """Small case for ncu captures of the RHMC multishift: one solve of the 12-shift system
    on 24^3x48 (links and source seeded on the device, about 10 GB on the device)."""
    import torch

    import leonardym_b200 as L
    from leonardym_b200 import synth
    from leonardym_b200.solvers import MULTISHIFT
    lib = L.lib()
    prec = args.precision or "half"
    lat = L.Lattice(DIMS, "su3", device=0)
    ctx = lat.handle
    links = synth.su3_fermion_links_device(DIMS, RHMC_EPS, RHMC_SEED, "cuda:0")
    lib.lym_gauge_upload_device(ctx, 1, C.c_void_p(links.data_ptr()))
    del links
    opid = C.c_int(0)
    lib.lym_operator_create(ctx, 1, 5, RHMC_KAPPA, RHMC_CSW, 1, C.byref(opid))
    b = synth.gaussian_spinor_device(DIMS, 3, RHMC_SEED + 1, "cuda:0")
    bb = float(torch.vdot(b.flatten(), b.flatten()).real)
    sols = [torch.zeros_like(b) for _ in RHMC_SHIFTS]
    torch.cuda.synchronize()  # the library's stream does not wait for torch's
    ptrs = (C.c_void_p * len(sols))(*[x.data_ptr() for x in sols])
    sh = np.ascontiguousarray(RHMC_SHIFTS, dtype=np.float64)
    st = L.SolveStats()
    rc = lib.lym_multishift_device(ctx, opid.value, MULTISHIFT[f"multishift_cg_mixed_{prec}"], len(sols),
                                   sh.ctypes.data_as(C.c_void_p), TOL * TOL * bb, 20000, C.c_void_p(b.data_ptr()),
                                   ptrs, C.byref(st))
    print(f"rhmc profile case: rc {rc}, {st.seconds:.3f} s, multishift steps {st.steps}, iterations "
          f"{st.iterations}, reliable updates {st.reliable_updates}, true residual {st.true_residual:.2e}")
    lat.close()
    if rc != 0:
        sys.exit(1)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default=None, choices=["single", "half"],
                    help="inner storage (default: single for the propagator solves, half for rhmc)")
    ap.add_argument("--workload", default="propagators", choices=["propagators", "rhmc", "rhmc-small", "consumers"],
                    help="propagators: the 24^3x48 block solves (the headline); rhmc: the 48^3x96 multishift; "
                         "rhmc-small: the same at 24^3x48")
    ap.add_argument("--solver", default="bicgstab", choices=["cg", "bicgstab"],
                    help="the block solver of the timed solves")
    ap.add_argument("--batch", type=int, default=16, help="right-hand sides per batched stencil (power of 2 <= 32)")
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--profile", action="store_true", help="small fixed case for ncu captures")
    ap.add_argument("--serve-window", type=float, default=0.25,
                    help="seconds of the configs' 200 requests/s Poisson stream (0: skip the serving measurements)")
    ap.add_argument("--serve-sweep-window", type=float, default=15.0,
                    help="seconds of arrivals at each load of the sweep below the measured capacity (0: no sweep)")
    ap.add_argument("--tile", default="", help="with --profile: batched stencil column and variant 'by,bz,minb'")
    args = ap.parse_args()
    if args.workload == "propagators" and args.precision is None:
        args.precision = "single"
    if args.profile:
        run_profile(args)
        return
    world, rank, local = dist_setup()
    try:
        if args.impl == "reference":
            run_reference(args, world, rank)
        elif args.workload.startswith("rhmc"):
            run_rhmc(args, world, rank, local, RHMC_DIMS if args.workload == "rhmc" else DIMS)
        else:
            run_ours(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
