"""Benchmark: batched 2D x Fourier Helmholtz solve, Helmholtz DOF/s on B200.

Workload (the configuration the headline metric is quoted on): 16x16
uniform quads on [0,1]^2, GLL order N=10 (N_P=11), N_Z=64 planes (modes
k=0..31), per-mode constant lambda^2 + (beta k)^2 with LAMBDA2=1, BETA=1,
Dirichlet u=0 on the x/y edges, forcing i.i.d. uniform[-1,1] per unique node
from seed 20261203.  One step = one full condensed direct solve of every
mode (elliptic/helmholtz.cpp:29-52, src/field.cpp:598-709) in plain FP64.
DOF per step = unique nodes per plane x N_Z = 25921 x 64.

value: device time of the solve with the Fourier forcing resident in HBM
(CUDA events on the library stream, L2 flushed between steps).
e2e:   the public host-buffer call stx_elliptic_solve_host (pinned forcing
in, forward FFT, solve, inverse FFT, solution out), wall clock.

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
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
sys.path.insert(0, ROOT)

WORKLOAD = dict(n=16, np_=11, nz=64, lambda2=1.0, beta=1.0, seed=20261203)
METRIC = "Helmholtz DOF/s (batched 2D x Fourier, plain FP64 direct)"
UNIT = "DOF/s"


def make_session(d):
    from semtex_b200 import sessions
    w = WORKLOAD
    return sessions.helmholtz_session(os.path.join(d, "c2"), w["n"], w["np_"], nz=w["nz"],
                                      lambda2=w["lambda2"], beta=w["beta"])


def forcing_per_unique_node(x, y, nz, seed):
    from semtex_b200 import sessions
    return sessions.forcing_per_unique_node(x, y, nz, seed)


def dist_init(backend="nccl"):
    """One process per GPU (torchrun env); a short timeout so that ranks
    waiting on a lost peer end with an error."""
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return ws, rank, local


def max_over_ranks(value, ws, device):
    """The largest of the ranks' values (the job's time is its slowest rank's)."""
    if ws <= 1:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return t.item()


def job_rate(units_per_rank, ws, seconds):
    """Whole-job throughput of ws replicas that each processed
    units_per_rank in at most `seconds` (weak scaling)."""
    return units_per_rank * ws / seconds


def clocks_start():
    try:
        f = open(os.path.join(tempfile.gettempdir(), f"clk_{os.getpid()}.csv"), "w")
        p = subprocess.Popen(
            ["nvidia-smi", "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
             "--format=csv,noheader,nounits", "-lms", "200"], stdout=f, stderr=subprocess.DEVNULL)
        return p, f
    except Exception:
        return None, None


def clocks_stop(p, f, gpu_index):
    if p is None:
        return None
    p.terminate()
    p.wait(timeout=10)
    f.close()
    sm, mx, reasons = [], None, set()
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    for ln in open(f.name):
        parts = [s.strip() for s in ln.split(",")]
        if len(parts) < 8 or parts[0] != str(gpu_index):
            continue
        try:
            sm.append(float(parts[1]))
            mx = float(parts[2])
        except ValueError:
            continue
        for nm, v in zip(names, parts[4:8]):
            if v.lower() == "active":
                reasons.add(nm)
    os.unlink(f.name)
    if not sm:
        return None
    return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
            "samples": len(sm)}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


def c2_parity(ctx, U):
    """Relative error of the timed solution (Fourier space, device) against
    the oracle's checksums of the same workload (tests/golden/baseline/c2.npz:
    norm, seeded Gaussian projections and sampled values of the oracle's
    physical-space solution), or None when the fixture is absent."""
    import semtex_b200 as S
    gold = os.path.join(ROOT, "tests", "golden")
    if not os.path.exists(os.path.join(gold, "baseline", "c2.npz")):
        return None
    sys.path.insert(0, gold)
    import make_baseline_fixtures as FX
    W = ctx.new_field("parity")
    ctx.sync()
    W.data.copy_(U.data)
    import torch
    torch.cuda.synchronize()
    W.transform(S.INVERSE)
    e = FX.errors(W.to_numpy(), FX.load("c2")["c"])
    return {"vs": "oracle checksums of the same forcing (norm, 4 Gaussian projections, 256 samples)",
            "rel_err": max(e.values()), "detail": e}


def load_dns_traffic(workload):
    """DRAM bytes (read + write) of one steady DNS step, from the committed
    ncu summary of the same workload (profiles/dns_traffic.json), or None."""
    p = os.path.join(ROOT, "profiles", "dns_traffic.json")
    if os.path.exists(p):
        return json.load(open(p)).get("dram_bytes_per_step", {}).get(workload)
    return None


def load_profile_traffic(phase):
    """DRAM bytes (read + write) of one launch of a solve phase, from the
    committed ncu summary of the same workload (profiles/c2_solve_traffic.json)."""
    p = os.path.join(ROOT, "profiles", "c2_solve_traffic.json")
    if os.path.exists(p):
        return json.load(open(p)).get("dram_bytes_per_phase", {}).get(phase)
    return None


# ---------------------------------------------------------------------------
# CPU arms (the oracle restatement of the reference path; the reference itself
# does not build here)
# ---------------------------------------------------------------------------

def _oracle_plane_worker(args):
    """Oracle solves of `planes`, each repeated `nrep` times after a one-off setup.

    Returns per-repetition seconds (summed over this worker's planes)."""
    session, planes, seed, nrep = args
    from threadpoolctl import threadpool_limits
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import semtex_oracle as O
    with threadpool_limits(1):
        S = O.read_session(session)
        P = O.Problem(S)
        c = "c"
        f, _ = forcing_per_unique_node(P.M.x, P.M.y, P.nz, seed)
        F = O.dft_forward(f)
        bl = P.bc_lines(c)
        beta = S.tokens["BETA"]
        systems = {k: O.MatrixSys(P.M, P.N[c], S.tokens["LAMBDA2"], (beta * (k >> 1)) ** 2)
                   for k in planes}
        out = []
        for _ in range(nrep):
            t0 = time.perf_counter()
            for k in planes:
                O.solve_plane(P.M, P.N[c], P.B[c], systems[k], F[k], np.zeros_like(F[k]), bl[k])
            out.append(time.perf_counter() - t0)
    return out


def dns_session(d, workload):
    """The DNS workloads' sessions (the builders and seeds of the tests)."""
    from semtex_b200 import sessions
    if workload in ("c3", "c3d"):
        return sessions.taylor_green_session(os.path.join(d, workload), 24, 9, 96, re=1600.0, dt=1e-3, nstep=200,
                                             extra={"DEALIAS": 1} if workload == "c3d" else None)
    return sessions.channel_session(os.path.join(d, "c5"), 16, 8, 9, 32, re=500.0, dt=5e-3, nstep=100)


def oracle_dns_sample(workload, modes, nsteps):
    """CPU baseline of a DNS workload: the oracle restatement of integrate()
    on one core, at full size, with the Helmholtz solves of the Fourier modes
    `modes` only (None: every mode).  Matrix setup is excluded, and the
    N_TIME - 1 start-up steps (whose Jacobi-PCG solves differ from a steady
    step's) are skipped: the run starts at full order from the initial state,
    with zero history, which changes the values of a steady step but not its
    work.  `nsteps` steady steps are timed.  The solve time of the sample is
    scaled to all solved planes; the rest of the step (nonlinear terms,
    transforms, waveProp, setPForce, project) runs in full.
    Returns (seconds per step, description)."""
    from threadpoolctl import threadpool_limits
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import semtex_oracle as O
    from semtex_b200 import sessions
    import semtex_b200 as SB
    with tempfile.TemporaryDirectory() as d:
        p = dns_session(d, workload)
        S = O.read_session(p)
        # the numbering (the `.num` input of the reference's dns) from the
        # library's host enumerate, the same maps as the oracle's own
        # (tests/test_numbering.py), whose -O3 search is slow at this size
        P = O.Problem(S, numbering={c: SB.numbering(p, c)["btog"] for c in S.fields})
        if workload == "c5":
            ic = sessions.channel_initial(P.M.x, P.M.y, np.arange(P.nz) * 2 * np.pi / P.nz)
        else:
            funcs = O.user_functions(S)
            ic = {c: P.evaluate(funcs[c], 0.0) for c in S.fields if c in funcs}
        D = O.DNS(P, ic, modes=modes)
        D.step = D.nord - 1
        with threadpool_limits(1):
            P.solve_seconds = 0.0
            t0 = time.perf_counter()
            D.advance(nsteps)
            total = time.perf_counter() - t0
        solved = P.nz - 1 if P.nz > 1 else 1
        sampled = solved if modes is None else sum(1 if (m == 0 or P.nz == 1) else 2 for m in modes)
        per_step = ((total - P.solve_seconds) + P.solve_seconds * solved / sampled) / nsteps
    what = (f"{nsteps} steady steps of the oracle restatement at full size, 1 thread, setup excluded, "
            "started at full order")
    if modes is not None:
        what += (f"; Helmholtz solves of modes {list(modes)} only ({sampled} of {solved} planes per field), "
                 f"their time scaled to all planes")
    return per_step, what


def cpu_sample(session, planes, workers, seed, nrep=1):
    """Oracle solves of `planes` spread over `workers` spawned processes.

    Returns the per-repetition wall time of the slowest worker."""
    if workers <= 1:
        return _oracle_plane_worker((session, planes, seed, nrep))
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    chunks = [planes[i::workers] for i in range(workers)]
    chunks = [c for c in chunks if c]
    with ctx.Pool(len(chunks)) as pool:
        res = pool.map(_oracle_plane_worker, [(session, ch, seed, nrep) for ch in chunks])
    return [max(r[i] for r in res) for i in range(nrep)]


def run_reference(args):
    ws, rank, _ = int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")), 0
    if rank != 0:
        return
    w = WORKLOAD
    cores = os.cpu_count() or 1
    with tempfile.TemporaryDirectory() as d:
        session = make_session(d)
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import semtex_oracle as O
        S = O.read_session(session)
        P = O.Problem(S)
        _, nuniq = forcing_per_unique_node(P.M.x, P.M.y, 1, w["seed"])
        planes = [k for k in range(w["nz"]) if k != 1][: max(cores, 1)]
        reps = cpu_sample(session, planes, cores, w["seed"], args.warmup + args.steps)
        times = reps[args.warmup:]
    tot = sum(times)
    value = nuniq * len(planes) * len(times) / tot
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot / len(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": config_block(),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": f"{len(planes)} of {w['nz'] - 1} solved planes per step, one "
                                   f"process per core; condensed-system setup excluded"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def config_block():
    w = WORKLOAD
    return {"workload": "c2: batched 2D x Fourier Helmholtz, 16x16 quads, N_P=11, N_Z=64, "
                        "lambda2=1+k^2, Dirichlet 0, U[-1,1] forcing",
            "elements": w["n"] * w["n"], "np": w["np_"], "nz": w["nz"],
            "solver": "element + patch static condensation, dense interface inverse per mode (FP64)",
            "l2": "flushed between timed steps (256 MB write)", "parallelism": "replicas"}


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------

def run_ours(args):
    import ctypes as C
    import torch
    ws, rank, local = dist_init()
    torch.cuda.set_device(local)
    import semtex_b200 as S
    from semtex_b200 import _lib
    w = WORKLOAD
    d = tempfile.mkdtemp()
    session = make_session(d)
    t0 = time.perf_counter()
    over = {"STX_TWOLEVEL": 0} if args.solver == "band" else {}
    tuning = {}
    if not args.untuned and args.solver != "band":
        from semtex_b200 import autotune
        tuning = autotune.tuned_overrides(session, "c", w["lambda2"])
        over.update(tuning)
    if args.mode_groups:
        over["STX_MODE_GROUPS"] = args.mode_groups
    ctx = S.Context(session, over or None, device=local)
    x, y = ctx.mesh_coords()
    f, nuniq = forcing_per_unique_node(x, y, ctx.nz, w["seed"])
    sysm = S.ModalMatrixSys(ctx, "c", w["lambda2"], w["beta"])
    setup_s = time.perf_counter() - t0
    # DOF over the solved planes (the Nyquist plane is never solved), counted
    # as the reference arm counts them
    dof = nuniq * (ctx.nz - 1 if ctx.nz > 1 else 1)
    F = ctx.new_field("f").load_physical(f).transform(S.FORWARD).zero_nyquist()
    U = ctx.new_field("c")
    stream = ctx.torch_stream()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{local}")
    phase = (C.c_float * 4)()
    launches = C.c_int()
    L = _lib.lib()

    def solve():
        _lib.check(L.stx_field_solve(sysm.handle, F.ptr(), U.ptr(), C.c_double(1e-12), 1000, None))

    def solve_profiled():
        # the phases of a solve run one after another here (no mode groups)
        _lib.check(L.stx_field_solve_profiled(sysm.handle, F.ptr(), U.ptr(), phase, None))
        return list(phase)

    _lib.check(L.stx_modal_launches(sysm.handle, C.byref(launches)))
    for _ in range(args.warmup):
        solve()
    if ws > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    clk_p, clk_f = clocks_start()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    for e0, e1 in ev:
        with torch.cuda.stream(stream):
            flush.fill_(1.0)
        e0.record(stream)
        solve()
        e1.record(stream)
    torch.cuda.synchronize()
    t_total = sum(e0.elapsed_time(e1) for e0, e1 in ev) / 1e3
    # per-phase breakdown (events between the phases of a sequential solve)
    phases = []
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            flush.fill_(1.0)
        phases.append(solve_profiled())
    torch.cuda.synchronize()
    t_total = max_over_ranks(t_total, ws, f"cuda:{local}")
    parity = c2_parity(ctx, U)
    if ws > 1:
        torch.distributed.barrier()
    # -- end to end through the host-buffer calls: every step copies its
    # forcing in from pinned host memory and its solution out; the K steps
    # go through the pipelined batch call (the copies of step i +- 1 overlap
    # the solve of step i), and one step at a time through the single call
    fh = torch.from_numpy(np.ascontiguousarray(f)).pin_memory()
    uh = [torch.empty_like(fh).pin_memory() for _ in range(2)]
    fins, fouts = [fh] * args.steps, [uh[i % 2] for i in range(args.steps)]
    S.solve_host_batch(sysm, [fh] * max(2, args.warmup), [uh[i % 2] for i in range(max(2, args.warmup))])
    _lib.check(_lib.lib().stx_elliptic_solve_host(sysm.handle, C.c_void_p(fh.data_ptr()),
                                                  C.c_void_p(uh[0].data_ptr())))
    if ws > 1:
        torch.distributed.barrier()
    e0 = time.perf_counter()
    S.solve_host_batch(sysm, fins, fouts)
    e_total = time.perf_counter() - e0
    e0 = time.perf_counter()
    for _ in range(args.steps):
        _lib.check(_lib.lib().stx_elliptic_solve_host(sysm.handle, C.c_void_p(fh.data_ptr()),
                                                      C.c_void_p(uh[0].data_ptr())))
    e_single = time.perf_counter() - e0
    e_total = max_over_ranks(e_total, ws, f"cuda:{local}")
    e_single = max_over_ranks(e_single, ws, f"cuda:{local}")
    clocks = clocks_stop(clk_p, clk_f, local)
    if rank != 0:
        if ws > 1:
            torch.distributed.destroy_process_group()
        return
    ph = np.array(phases)
    mb = (C.c_double * 4)()
    _lib.check(_lib.lib().stx_modal_bytes(sysm.handle, mb))
    names = ["element condensation", "skeleton solve", "skeleton solve (2nd half)", "element recovery"]
    ms = ph.mean(axis=0)
    # the skeleton solve's two halves are one phase for the roofline
    phase_ms = [ms[0], ms[1] + ms[2], ms[3]]
    phase_bytes = [mb[0], mb[1] + mb[2], mb[3]]
    phase_names = [names[0], names[1], names[3]]
    top = int(np.argmax(phase_ms))
    peak, kind = measured_peaks()
    achieved = phase_bytes[top] / (phase_ms[top] / 1e3) / 1e9
    traffic = load_profile_traffic(phase_names[top])
    # CPU baseline: the oracle on one core over a bounded sample of planes
    cpu = None
    if not args.no_cpu_baseline:
        planes = [0, 2, 3, 20, 21, 62, 63]
        secs = cpu_sample(session, planes, 1, w["seed"], 3)
        cpu = {"value": nuniq * len(planes) / min(secs), "unit": UNIT, "cores": 1, "kind": "port",
               "sample": f"{len(planes)} of {w['nz'] - 1} solved planes (modes 0,1,10,31), "
                         "oracle restatement: per-element condensation + LAPACK dpbtrs, 1 thread"}
    line = {
        "metric": METRIC, "value": job_rate(dof * args.steps, ws, t_total), "unit": UNIT, "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t_total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": config_block(),
        "e2e": {"value": job_rate(dof * args.steps, ws, e_total), "unit": UNIT,
                "h2d_bytes_per_step": int(fh.numel() * 8), "d2h_bytes_per_step": int(uh[0].numel() * 8),
                "call": "stx_elliptic_solve_host_batch (pipelined: copies of neighbouring steps overlap a solve)",
                "single_call": {"value": job_rate(dof * args.steps, ws, e_single),
                                "call": "stx_elliptic_solve_host, one step per call"}},
        "roofline": {"bound": "hbm", "kernel": phase_names[top], "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak, "peak_kind": kind, "traffic": traffic,
                     "algorithmic_bytes_per_launch": phase_bytes[top],
                     "whole_solve": {"achieved": sum(phase_bytes) / (t_total / args.steps) / 1e9,
                                     "algorithmic_bytes": sum(phase_bytes)}},
        # phases of a solve with its mode groups run one after another (the
        # timed solves overlap the groups' phases on parallel streams)
        "phases": {n: {"ms": float(t), "bytes": float(b), "GB/s": float(b / (t / 1e3) / 1e9)}
                   for n, t, b in zip(phase_names, phase_ms, phase_bytes)},
        "sequential_ms": float(sum(phase_ms)),
        "setup_s": setup_s, "families": ctx.families(),
        "gpu_launches": int(launches.value) * args.steps,
        "clocks": clocks, "cpu_baseline": cpu, "parity": parity,
        "tuning": {"table": "semtex_b200/autotune_table.json", "tokens": tuning},
    }
    if args.dns_steps > 0 and ws == 1:
        line["mixed"] = run_mixed(ctx, sysm, F, args, flush, stream, dof)
        cb = not args.no_cpu_baseline
        line["dns"] = run_dns(args.dns_steps, 3, local, "c3", cb)
        line["dns_c3_dealiased"] = run_dns(args.dns_steps, 3, local, "c3d", cb)
        line["dns_c5"] = run_dns(args.dns_steps, 3, local, "c5", cb)
        line["dns_mixed_c3_dealiased"] = run_dns_mixed(args.dns_steps, 3, local, "c3d")
        line["batch_c4"] = run_batch(args.dns_steps, 3, local, not args.untuned)
        line["adjoint_c5"] = run_adjoint(local)
    print(json.dumps(line))
    if ws > 1:
        torch.distributed.destroy_process_group()


def run_mixed(ctx, sysm, F, args, flush, stream, dof):
    """The same c2 solve with STX_MIXED: the skeleton solve's packed inverses
    in FP32 (sums in FP64) and two FP64 iterative refinements of the skeleton
    solution.  Same timing rules as the FP64 line; the error is the relative
    L2 difference from the FP64 solution of the same forcing (which matches
    the oracle to 1e-10)."""
    import ctypes as C
    import torch
    import semtex_b200 as S
    from semtex_b200 import _lib
    L = _lib.lib()
    w = WORKLOAD
    sysx = S.ModalMatrixSys(ctx, "c", w["lambda2"], w["beta"], method=S.MIXED)
    U64, U32 = ctx.new_field("u64"), ctx.new_field("u32")
    _lib.check(L.stx_field_solve(sysm.handle, F.ptr(), U64.ptr(), C.c_double(1e-12), 1000, None))

    def solve():
        _lib.check(L.stx_field_solve(sysx.handle, F.ptr(), U32.ptr(), C.c_double(1e-12), 1000, None))

    for _ in range(args.warmup):
        solve()
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    for e0, e1 in ev:
        with torch.cuda.stream(stream):
            flush.fill_(1.0)
        e0.record(stream)
        solve()
        e1.record(stream)
    torch.cuda.synchronize()
    t = sum(e0.elapsed_time(e1) for e0, e1 in ev) / 1e3
    err = float(torch.linalg.norm(U32.data - U64.data) / torch.linalg.norm(U64.data))
    launches = C.c_int()
    _lib.check(L.stx_modal_launches(sysx.handle, C.byref(launches)))
    out = {"metric": METRIC.replace("plain FP64 direct", "FP32 skeleton inverses + FP64 refinement"),
           "value": dof * args.steps / t, "unit": UNIT, "ms_per_step": 1e3 * t / args.steps,
           "refinements": 2,
           "rel_l2_vs_fp64": err, "dtype": "f32 matrices, f64 sums / residuals / refinement",
           "gpu_launches": int(launches.value) * args.steps}
    sysx.close()
    return out


DNS_WORKLOADS = {
    "c3": "c3: Taylor-Green 24x24x96, N_P=9, Re=1600, D_T=1e-3, N_TIME=3 (no dealiasing)",
    "c3d": "c3: Taylor-Green 24x24x96, N_P=9, Re=1600, D_T=1e-3, N_TIME=3, 3/2-rule dealiased products",
    "c5": "c5: channel [0,2pi]x[-1,1]x[0,2pi) 16x8x32, N_P=9, Re=500, D_T=5e-3, N_TIME=3, "
          "no-slip walls with high-order pressure BCs, u=1-y^2 + seeded 1e-3 perturbation",
}


def run_dns(steps, warmup=3, local=0, workload="c3", cpu_baseline=False):
    """Secondary measurement: DNS steps/s, plain FP64 direct solves,
    alternating skew-symmetric advection.  c3: 3D Taylor--Green (24x24
    periodic quads, N_P=9, N_Z=96, Re=1600, D_T=1e-3, N_TIME=3).  c5: plane
    channel (16x8 quads periodic in x, N_P=9, N_Z=32, Re=500, D_T=5e-3,
    N_TIME=3, walls <D> u=v=w=0 / <H> p, base flow plus a seeded stream-
    function perturbation).  The first N_TIME-1 steps use the reference's
    temporary PCG systems and are excluded; the timed steps are device time
    (CUDA events on the library stream); steady steps run as the library's
    captured CUDA graph of one step cycle."""
    import torch
    import semtex_b200 as S
    from semtex_b200 import sessions
    d = tempfile.mkdtemp()
    p = dns_session(d, workload)
    t0 = time.perf_counter()
    ctx = S.Context(p, device=local)
    D = S.DNS(ctx, 1)
    setup = time.perf_counter() - t0
    if workload in ("c3", "c3d"):
        funcs = S._user_functions(p)
        ic = {c: ctx.evaluate(funcs[c], 0.0) for c in ctx.fields if c in funcs}
    else:
        x, y = ctx.mesh_coords()
        z = np.arange(ctx.nz) * 2 * np.pi / ctx.nz
        ic = sessions.channel_initial(x, y, z)
    D.restart(ic, 0.0)
    # start-up steps and warm-up, then the steps in which the steady step
    # cycle (14 steps for c3, 42 for c5) is captured as a CUDA graph and
    # replayed: 84 steps end on a cycle boundary, as the timed steps do
    D.advance(2 + warmup)
    D.advance(84)
    stream = ctx.torch_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ctx.sync()
    e0.record(stream)
    D.advance(steps)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1) / steps
    period, glaunch = D.graph_info()
    # roofline: algorithmic bytes of one steady step over its device time.
    # Field passes (F = one field, nz planes of plane_size doubles):
    # nonlinear 2 ncom, waveProp (2 N_TIME + 1) ncom, setPForce ndim + 1,
    # project 2 ncom + 1; plus the solves: the pressure system's
    # stx_modal_bytes, the velocity system's once (its matrices are read once
    # for all components) plus 3 F per further component (forcing read by the
    # condensation and the recovery, solution written)
    ncom = len(ctx.fields) - 1
    ndim = 3 if ctx.nz > 1 else 2
    nord = int(ctx.token("N_TIME"))
    F = 8.0 * ctx.plane_size * ctx.nz
    passes = 2 * ncom + (2 * nord + 1) * ncom + (ndim + 1) + (2 * ncom + 1)
    vb, pb = sum(D.system_bytes(ctx.fields[0])), sum(D.system_bytes(ctx.fields[ncom]))
    step_bytes = passes * F + pb + vb + (ncom - 1) * 3 * F
    peak, kind = measured_peaks()
    achieved = step_bytes / (ms / 1e3) / 1e9
    traffic = load_dns_traffic(workload)
    out = {"metric": "DNS steps/s", "value": 1e3 / ms, "ms_per_step": ms, "steps": steps,
           "workload": DNS_WORKLOADS[workload], "setup_s": setup,
           "graph": {"cycle_steps": period, "launches": glaunch},
           "roofline": {"bound": "hbm", "kernel": "whole step", "achieved": achieved, "peak": peak,
                        "unit": "GB/s", "frac": achieved / peak, "peak_kind": kind,
                        "algorithmic_bytes_per_step": step_bytes,
                        "model": {"field_bytes": F, "field_passes": passes, "pressure_solve_bytes": pb,
                                  "velocity_solve_bytes": vb + (ncom - 1) * 3 * F},
                        "traffic": traffic}}
    D.close()
    ctx.close()
    if cpu_baseline:
        # c5: two modes, two steps; c3: the highest mode, one step (a Fourier
        # mode's planes cost the same to solve, mode 0 aside)
        modes, nst = ((1, 15), 2) if workload == "c5" else ((47,), 1)
        sec, what = oracle_dns_sample(workload, modes, nst)
        out["cpu_baseline"] = {"value": 1.0 / sec, "unit": "steps/s", "cores": 1, "kind": "port",
                               "sample": what}
    return out


def run_dns_mixed(steps, warmup=3, local=0, workload="c3d"):
    """Secondary measurement: the DNS with mixed-precision steady velocity
    solves (token STX_DNS_MIXED = 1: FP32 packed skeleton inverses, sums in
    FP64, two FP64 refinements; pressure solves, field passes, FFTs and the
    time integration in FP64) against the plain FP64 DNS on the same
    workload and schedule.  Both run 2 start-up + warm-up + 84 graph-capture
    steps, then `steps` timed steps (device time, CUDA events on the library
    stream); the error is the relative L2 difference of every field from the
    FP64 run after the same steps (the FP64 run matches the oracle)."""
    import torch
    import semtex_b200 as S
    d = tempfile.mkdtemp()
    p = dns_session(d, workload)
    res = {}
    fields = {}
    for name, ov in (("fp64", None), ("mixed", {"STX_DNS_MIXED": 1})):
        ctx = S.Context(p, overrides=ov, device=local)
        D = S.DNS(ctx, 1)
        funcs = S._user_functions(p)
        D.restart({c: ctx.evaluate(funcs[c], 0.0) for c in ctx.fields if c in funcs}, 0.0)
        D.advance(2 + warmup)
        D.advance(84)
        stream = ctx.torch_stream()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ctx.sync()
        e0.record(stream)
        D.advance(steps)
        e1.record(stream)
        e1.synchronize()
        res[name] = e0.elapsed_time(e1) / steps
        fields[name] = {c: D.field(c) for c in ctx.fields}
        D.close()
        ctx.close()
    err = {c: float(np.linalg.norm(fields["mixed"][c] - fields["fp64"][c]) /
                    max(np.linalg.norm(fields["fp64"][c]), 1e-300)) for c in fields["fp64"]}
    return {"metric": "DNS steps/s", "value": 1e3 / res["mixed"], "ms_per_step": res["mixed"],
            "steps": steps, "workload": DNS_WORKLOADS[workload],
            "dtype": "f32 skeleton inverses of the velocity systems; f64 everything else",
            "fp64_ms_per_step": res["fp64"], "ratio_to_fp64": res["fp64"] / res["mixed"],
            "rel_l2_vs_fp64": err, "after_steps": 2 + warmup + 84 + steps}


def run_adjoint(local=0, steps=100, every=10):
    """Secondary measurement: the discrete adjoint of the c5 channel
    workload (16x8 quads, N_P=9, N_Z=32, Re=500, D_T=5e-3, N_TIME=3): a
    100-step recorded run with full-state checkpoints every 10 steps, then
    the gradient of the perturbation kinetic energy at the end w.r.t. the
    initial velocity (stx_dns_adjoint_backward: segments recomputed from
    their checkpoints, steps transposed), and the tangent-linear derivative
    along a second seeded perturbation (stx_dns_adjoint_tangent).  Device
    time by CUDA events on the library stream around each C-ABI call (the
    calls include their host copies of the seed and gradient, 3 fields
    each).  The gradient's directional derivative is compared with the
    tangent-linear one (they agree to round-off when the adjoint is the
    exact transpose)."""
    import torch
    import semtex_b200 as S
    from semtex_b200 import sessions
    import ctypes as C
    from semtex_b200 import _lib
    d = tempfile.mkdtemp()
    p = dns_session(d, "c5")
    ctx = S.Context(p, device=local)
    x, y = ctx.mesh_coords()
    z = np.arange(ctx.nz) * 2 * np.pi / ctx.nz
    u0 = {c: v for c, v in sessions.channel_initial(x, y, z).items() if c != "p"}
    alt = sessions.channel_initial(x, y, z, seed=7)
    shape = (ctx.nz, ctx.nel, ctx.np, ctx.np)
    base = {"u": np.broadcast_to(1 - y * y, shape), "v": np.zeros(shape), "w": np.zeros(shape)}
    dirn = {c: alt[c] - base[c] for c in "uvw"}
    q4 = np.empty(ctx.nel * ctx.np * ctx.np)
    _lib.check(_lib.lib().stx_mesh_mass(ctx.handle, C.c_void_p(q4.ctypes.data)))
    q4 = q4.reshape(1, ctx.nel, ctx.np, ctx.np)
    stream = ctx.torch_stream()

    def timed(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ctx.sync()
        e0.record(stream)
        r = fn()
        e1.record(stream)
        e1.synchronize()
        return r, e0.elapsed_time(e1)

    D = S.DNS(ctx, 1)
    A = S.DNSAdjoint(D, checkpoint_every=every)
    res = {}
    for rep in range(2):  # the first pass sets up the start-up systems
        D.restart(u0, 0.0)
        _, fwd_ms = timed(lambda: D.advance(steps))
        D.restart(u0, 0.0)
        _, rec_ms = timed(lambda: A.record(steps))
        uT = {c: D.field(c) for c in "uvw"}
        dE = {c: q4 * (uT[c] - base[c]) for c in "uvw"}
        grad, bwd_ms = timed(lambda: A.backward(dE))
        tl, tan_ms = timed(lambda: A.tangent(dirn))
        res = {"forward_ms": fwd_ms, "record_ms": rec_ms, "backward_ms": bwd_ms, "tangent_ms": tan_ms,
               "grad": grad, "tl": tl}
    dot = sum(float(np.vdot(res["grad"][c], dirn[c])) for c in "uvw")
    tld = sum(float(np.vdot(dE[c], res["tl"][c])) for c in "uvw")
    _, _, ck_bytes = A.info()
    A.close()
    D.close()
    ctx.close()
    return {"metric": "adjoint gradient time", "workload": DNS_WORKLOADS["c5"] + "; 100 steps, checkpoints every 10",
            "objective": "perturbation kinetic energy at the end (Q4-weighted, about u = 1 - y^2)",
            "forward_ms": res["forward_ms"], "record_ms": res["record_ms"], "backward_ms": res["backward_ms"],
            "tangent_ms": res["tangent_ms"],
            "gradient_ms": res["record_ms"] + res["backward_ms"],
            "backward_over_forward": res["backward_ms"] / res["forward_ms"],
            "checkpoint_bytes": ck_bytes,
            "adjoint_vs_tangent_rel": abs(dot - tld) / abs(tld)}


def dns_probe(workload):
    """Two start-up and three steady steps of a DNS workload with the graph
    replay off (every kernel a plain launch): the run the DNS traffic
    profile captures."""
    import semtex_b200 as S
    from semtex_b200 import sessions
    d = tempfile.mkdtemp()
    p = dns_session(d, workload)
    ctx = S.Context(p, {"STX_DNS_GRAPH": 0})
    D = S.DNS(ctx, 1)
    if workload == "c5":
        x, y = ctx.mesh_coords()
        ic = sessions.channel_initial(x, y, np.arange(ctx.nz) * 2 * np.pi / ctx.nz)
    else:
        funcs = S._user_functions(p)
        ic = {c: ctx.evaluate(funcs[c], 0.0) for c in ctx.fields if c in funcs}
    D.restart(ic, 0.0)
    D.advance(5)
    ctx.sync()
    D.close()
    ctx.close()


def run_batch(steps, warmup=3, local=0, tuned=True):
    """Secondary measurement: the uneven batch (64 independent 2D Helmholtz
    problems, n x n quads with n uniform in 4..32, order N uniform in 6..12,
    lambda^2 log-uniform in [0.1, 100], Dirichlet zero, U[-1,1] forcing per
    unique node, seeded).  Helmholtz DOF/s of the whole batch, device time
    (CUDA events), L2 flushed between steps, for (a) one replay of the
    captured CUDA graph (stx_batch_launch) and (b) the same 64 DIRECT solves
    issued one stx_field_solve call at a time from the host."""
    import ctypes as C
    import torch
    import semtex_b200 as S
    from semtex_b200 import sessions
    from semtex_b200._lib import lib
    d = tempfile.mkdtemp()
    specs = sessions.uneven_batch()
    batch_tuning = {}
    if tuned:
        from semtex_b200 import autotune
        batch_tuning = autotune.tuned_batch_overrides(specs)
    t0 = time.perf_counter()
    items, ctxs, dof = [], [], 0
    for i, sp in enumerate(specs):
        path = sessions.helmholtz_session(os.path.join(d, f"p{i}"), sp["n"], sp["np"], lambda2=sp["lambda2"])
        ctx = S.Context(path, batch_tuning or None, device=local)
        x, y = ctx.mesh_coords()
        f, nu = sessions.forcing_per_unique_node(x, y, 1, sp["seed"])
        dof += nu
        sys_ = S.ModalMatrixSys(ctx, "c", sp["lambda2"])
        items.append((sys_, ctx.new_field("f").load_physical(f), ctx.new_field("u")))
        ctxs.append(ctx)
    B = S.Batch(items)
    setup = time.perf_counter() - t0
    dev = f"cuda:{local}"
    main = torch.cuda.ExternalStream(B.stream, device=dev)
    side = [torch.cuda.ExternalStream(c.stream, device=dev) for c in ctxs]
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    calls = [(s.handle, fF.ptr(), fU.ptr()) for s, fF, fU in items]
    solve = lib().stx_field_solve

    def one_loop():
        ev0 = torch.cuda.Event()
        ev0.record(main)
        for st in side:
            st.wait_event(ev0)
        for h, pf, pu in calls:
            rc = solve(h, pf, pu, 0.0, 0, None)
            if rc:
                raise RuntimeError(f"stx_field_solve failed ({rc})")
        for st in side:
            ev = torch.cuda.Event()
            ev.record(st)
            main.wait_event(ev)

    def timed(fn):
        ms = []
        for k in range(warmup + steps):
            with torch.cuda.stream(main):
                flush.fill_(1.0)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(main)
            fn()
            e1.record(main)
            e1.synchronize()
            if k >= warmup:
                ms.append(e0.elapsed_time(e1))
        return statistics.mean(ms)

    ms_graph = timed(B.launch)
    ms_loop = timed(one_loop)
    out = {"metric": "Helmholtz DOF/s (uneven batch, one CUDA graph)", "value": dof / (ms_graph * 1e-3),
           "unit": "DOF/s", "ms_per_step": ms_graph, "steps": steps,
           "per_problem_calls": {"value": dof / (ms_loop * 1e-3), "ms_per_step": ms_loop},
           "problems": len(specs), "dof": dof, "elements": sum(sp["n"] ** 2 for sp in specs),
           "kernel_nodes": B.kernel_nodes, "tuning": batch_tuning,
           "workload": "c4: 64 Dirichlet Helmholtz problems on [0,1]^2, n in 4..32, N in 6..12, "
                       "lambda^2 log-uniform [0.1,100], seed 20261203",
           "setup_s": setup}
    B.close()
    for sys_, _, _ in items:
        sys_.close()
    for c in ctxs:
        c.close()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--dns-steps", type=int, default=84,
                    help="timed steps of the secondary measurements (mixed-precision c2, DNS c3 / c5, "
                         "batch c4); 0 skips them")
    ap.add_argument("--mode-groups", type=int, default=0,
                    help="Fourier-mode groups solved on parallel streams (0: library default)")
    ap.add_argument("--untuned", action="store_true",
                    help="ignore the autotuner's table (semtex_b200/autotune_table.json)")
    ap.add_argument("--solver", default="twolevel", choices=["twolevel", "band"],
                    help="band: the single banded-Cholesky skeleton solve (for comparison)")
    ap.add_argument("--workload", default="c2",
                    choices=["c2", "dns", "dns_c5", "dns_mixed", "batch_c4", "adjoint_c5", "dns_probe_c3",
                             "dns_probe_c5"],
                    help="dns / dns_c5 / dns_mixed / batch_c4: run only that secondary measurement (one JSON "
                         "line); "
                         "dns_probe_c3 / _c5: 2 start-up + 3 steady steps with graph replay off, nothing "
                         "timed (a run to profile every kernel of a step)")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload.startswith("dns_probe_"):
        dns_probe(args.workload[len("dns_probe_"):])
    elif args.workload in ("dns", "dns_c5"):
        import torch
        torch.cuda.set_device(0)
        print(json.dumps(run_dns(max(1, args.dns_steps), args.warmup, 0,
                                 "c3" if args.workload == "dns" else "c5", not args.no_cpu_baseline)))
    elif args.workload == "dns_mixed":
        import torch
        torch.cuda.set_device(0)
        print(json.dumps(run_dns_mixed(max(1, args.dns_steps), args.warmup, 0, "c3d")))
    elif args.workload == "adjoint_c5":
        import torch
        torch.cuda.set_device(0)
        print(json.dumps(run_adjoint(0)))
    elif args.workload == "batch_c4":
        import torch
        torch.cuda.set_device(0)
        print(json.dumps(run_batch(max(1, args.dns_steps), args.warmup, 0, not args.untuned)))
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
