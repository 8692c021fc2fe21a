"""Autotuner of the direct solve's launch configuration.

The solve's speed on a given problem shape depends on choices that the
library otherwise makes from byte and shared-memory models: the patch size of
the two-level condensation (session token STX_PATCH_CAP), the elements per
chunk of the element kernels (STX_CHUNK), the Fourier-mode groups run on
parallel streams (STX_MODE_GROUPS), the warps per block of the packed
skeleton products (STX_SYM_WARPS), how many product warps are scheduled
per full wave (STX_SYM_OCC, percent) and whether the products run their
register-capped build (STX_SYM_REGCAP: more resident warps, a few spills).  ``tune`` measures them on the device
by coordinate descent -- each knob in turn over its values with the others
held at the best so far, the device time of stx_field_solve (CUDA events,
the least of several solves of a resident forcing, each after a 256 MB
write that flushes L2, as the benchmark times its solves: the mean moves
between processes, e.g. with how two mode-group streams happen to overlap,
the least time much less) deciding -- and records every
trial and the winner in a JSON table keyed by the problem's shape.
``tuned_overrides`` returns the winner for a session from that table (empty
when the shape was never tuned), for Context(..., overrides=...).  A batch
of independent problems is tuned as a whole (``tune_batch``: one setting for
every problem, timed as the batch's graph replay), since problems that run
side by side compete for the GPU: settings best for each problem alone made
the 64-problem benchmark batch slower (0.69 against 0.56 ms).

The committed table (semtex_b200/autotune_table.json) holds the
benchmark workloads' entries; ``python -m semtex_b200.autotune session
field lambda2`` tunes another shape into it.
"""

from __future__ import annotations

import argparse
import json
import os

import numpy as np

TABLE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "autotune_table.json")

# knob -> candidate values (the library's defaults first)
SPACE = {
    "STX_PATCH_CAP": [None, 8, 16, 36, 64],
    "STX_CHUNK": [None, 16, 8],
    "STX_ELEM_TWOBLOCK": [None, 1],
    "STX_MODE_GROUPS": [None, 1, 3, 4],
    "STX_STAGGER": [None, 1],
    "STX_SYM_REGCAP": [None, 1],
    "STX_SYM_WARPS": [None, 2, 8],
    "STX_SYM_OCC": [None, 50, 200],
    "STX_PDL": [None, 0],
}


def signature(session: str, field: str, lambda2: float, overrides: dict | None = None) -> str:
    """Shape key of a solve: elements, N_P, N_Z, the field's numbering sizes
    (host only: no device needed) and whether the system is singular-prone
    (lambda2 = 0)."""
    from . import numbering
    ov = dict(overrides or {})
    n = numbering(session, field, ov)
    nel, next_ = n["btog"].shape
    np_ = next_ // 4 + 1
    nz = _token(session, "N_Z", ov)
    return f"nel{nel}-np{np_}-nz{int(nz)}-ng{n['nglobal']}-ns{n['nsolve']}-lam{'0' if lambda2 == 0 else '+'}"


def _token(session, name, ov):
    if name in ov:
        return float(ov[name])
    for ln in open(session):
        s = ln.split("#")[0].strip()
        if s.startswith(name) and "=" in s and s.split("=")[0].strip() == name:
            try:
                return float(s.split("=", 1)[1].split()[0])
            except ValueError:
                pass
    return 1.0


def load_table(path: str = TABLE) -> dict:
    if os.path.exists(path):
        with open(path) as f:
            return json.load(f)
    return {"entries": {}}


def save_table(table: dict, path: str = TABLE):
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        json.dump(table, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def tuned_overrides(session: str, field: str, lambda2: float, path: str = TABLE) -> dict:
    """The tuned tokens for this session's shape, or {} if it was never tuned."""
    entry = load_table(path)["entries"].get(signature(session, field, lambda2))
    return dict(entry["best"]) if entry else {}


def coordinate_descent(measure, space: dict = SPACE, rounds: int = 1):
    """Minimise measure(config) over the product space by coordinate descent.

    config maps knob -> value (None = library default, left out of the
    overrides).  Returns (best config, best time, trials [(config, time)])."""
    best = {k: v[0] for k, v in space.items()}
    measure(dict(best))  # discarded: the first solves of a run start on an idle GPU
    best_t = measure(dict(best))
    trials = [(dict(best), best_t)]
    for _ in range(rounds):
        changed = False
        for knob, values in space.items():
            for v in values:
                if v == best[knob]:
                    continue
                cand = dict(best)
                cand[knob] = v
                t = measure(dict(cand))
                trials.append((dict(cand), t))
                if t < best_t:
                    best, best_t, changed = cand, t, True
        if not changed:
            break
    return best, best_t, trials


def _overrides(config: dict) -> dict:
    return {k: v for k, v in config.items() if v is not None}


def _l2_flush_buffer(device: int):
    """A 256 MB device buffer whose write evicts L2 (126 MB) between timed solves."""
    import torch
    return torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{device}")


def solve_time_ms(session: str, field: str, lambda2: float, overrides: dict, reps: int = 11, device: int = 0,
                  seed: int = 1) -> float:
    """Least device time (ms) of `reps` stx_field_solve calls with a
    resident random forcing under `overrides`, L2 flushed before each (a
    failed configuration: +inf)."""
    import ctypes as C
    import torch
    from . import Context, FORWARD, ModalMatrixSys, StxError
    from ._lib import check, lib
    try:
        ctx = Context(session, overrides or None, device=device)
    except StxError:
        return float("inf")
    try:
        sysm = ModalMatrixSys(ctx, field, lambda2)
    except StxError:
        ctx.close()
        return float("inf")
    rng = np.random.default_rng(seed)
    f = rng.uniform(-1, 1, (ctx.nz, ctx.nel, ctx.np, ctx.np))
    F = ctx.new_field("f").load_physical(f).transform(FORWARD).zero_nyquist()
    U = ctx.new_field("u")
    stream = ctx.torch_stream()
    flush = _l2_flush_buffer(device)
    times = []
    for k in range(reps + 2):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            flush.fill_(float(k))
        e0.record(stream)
        check(lib().stx_field_solve(sysm.handle, F.ptr(), U.ptr(), C.c_double(0.0), 0, None))
        e1.record(stream)
        e1.synchronize()
        if k >= 2:
            times.append(e0.elapsed_time(e1))
    ok = sysm.status() == 0
    sysm.close()
    ctx.close()
    return min(times) if ok else float("inf")


def tune(session: str, field: str, lambda2: float, space: dict = SPACE, reps: int = 11, device: int = 0,
         path: str | None = TABLE, label: str = "") -> dict:
    """Tune one shape on the device; record it in the table at `path` (None:
    do not record).  Returns the table entry."""
    def measure(config):
        return solve_time_ms(session, field, lambda2, _overrides(config), reps, device)

    best, best_t, trials = coordinate_descent(measure, space)
    entry = {"label": label, "best": _overrides(best), "best_ms": best_t, "default_ms": trials[0][1],
             "trials": [[_overrides(c), t] for c, t in trials]}
    if path:
        table = load_table(path)
        table["entries"][signature(session, field, lambda2)] = entry
        save_table(table, path)
    return entry


# knobs of a batch of single-plane problems (mode groups do not apply)
BATCH_SPACE = {k: v for k, v in SPACE.items() if k not in ("STX_MODE_GROUPS", "STX_STAGGER")}


def batch_signature(specs) -> str:
    """Key of a batch of problems: their (n, N_P) list in order."""
    import hashlib
    key = ";".join(f"{s['n']}x{s['np']}" for s in specs)
    return "batch-" + hashlib.sha1(key.encode()).hexdigest()[:16] + f"-{len(specs)}"


def batch_time_ms(specs, overrides: dict, reps: int = 11, device: int = 0) -> float:
    """Least device time (ms) of `reps` replays of the batch's CUDA graph
    (stx_batch_launch, L2 flushed before each) with the same overrides on every problem (+inf when a
    problem rejects them).  The problems are the uneven-batch dicts of
    sessions.uneven_batch (n, np, lambda2, seed), Dirichlet zero."""
    import tempfile
    import torch
    from . import Batch, Context, ModalMatrixSys, StxError, sessions
    items, ctxs = [], []
    with tempfile.TemporaryDirectory() as d:
        try:
            for i, sp in enumerate(specs):
                p = sessions.helmholtz_session(os.path.join(d, f"p{i}"), sp["n"], sp["np"], lambda2=sp["lambda2"])
                ctx = Context(p, overrides or None, device=device)
                ctxs.append(ctx)
                x, y = ctx.mesh_coords()
                f, _ = sessions.forcing_per_unique_node(x, y, 1, sp["seed"])
                items.append((ModalMatrixSys(ctx, "c", sp["lambda2"]), ctx.new_field("f").load_physical(f),
                              ctx.new_field("u")))
        except StxError:
            for c in ctxs:
                c.close()
            return float("inf")
    B = Batch(items)
    main = torch.cuda.ExternalStream(B.stream, device=f"cuda:{device}")
    flush = _l2_flush_buffer(device)
    times = []
    for k in range(reps + 2):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(main):
            flush.fill_(float(k))
        e0.record(main)
        B.launch()
        e1.record(main)
        e1.synchronize()
        if k >= 2:
            times.append(e0.elapsed_time(e1))
    ok = all(s.status() == 0 for s, _, _ in items)
    B.close()
    for s, _, _ in items:
        s.close()
    for c in ctxs:
        c.close()
    return min(times) if ok else float("inf")


def tune_batch(specs, space: dict = BATCH_SPACE, reps: int = 11, device: int = 0, path: str | None = TABLE,
               label: str = "") -> dict:
    """Tune one setting of the knobs for a whole batch, timed as the batch
    runs (its graph replay: the problems' kernels run side by side, so a
    setting that is best for a problem alone need not be best in the batch).
    Recorded under batch_signature(specs)."""
    def measure(config):
        return batch_time_ms(specs, _overrides(config), reps, device)

    best, best_t, trials = coordinate_descent(measure, space)
    entry = {"label": label, "best": _overrides(best), "best_ms": best_t, "default_ms": trials[0][1],
             "trials": [[_overrides(c), t] for c, t in trials]}
    if path:
        table = load_table(path)
        table["entries"][batch_signature(specs)] = entry
        save_table(table, path)
    return entry


def tuned_batch_overrides(specs, path: str = TABLE) -> dict:
    """The tuned tokens of a batch, or {} if it was never tuned."""
    entry = load_table(path)["entries"].get(batch_signature(specs))
    return dict(entry["best"]) if entry else {}


def tune_benchmark_workloads(path: str = TABLE, device: int = 0, only: str | None = None):
    """Tune the benchmark's Helmholtz workloads into the table: the batched
    2D x Fourier solve (16x16 quads, N_P=11, N_Z=64) and the uneven batch
    (64 problems, seed 20261203) as one batch."""
    import tempfile
    from . import sessions
    with tempfile.TemporaryDirectory() as d:
        if only in (None, "c2"):
            p = sessions.helmholtz_session(os.path.join(d, "c2"), 16, 11, nz=64, lambda2=1.0, beta=1.0)
            e = tune(p, "c", 1.0, device=device, path=path, label="c2")
            print("c2", json.dumps({k: e[k] for k in ("best", "best_ms", "default_ms")}), flush=True)
        if only not in (None, "c4"):
            return
        e = tune_batch(sessions.uneven_batch(), device=device, path=path, label="c4 uneven batch")
        print("c4", json.dumps({k: e[k] for k in ("best", "best_ms", "default_ms")}), flush=True)


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("session", nargs="?")
    ap.add_argument("field", nargs="?")
    ap.add_argument("lambda2", type=float, nargs="?")
    ap.add_argument("--label", default="")
    ap.add_argument("--table", default=TABLE)
    ap.add_argument("--benchmark", action="store_true", help="tune the benchmark's Helmholtz workloads")
    ap.add_argument("--only", choices=["c2", "c4"], help="with --benchmark: one of the two workloads")
    a = ap.parse_args()
    if a.benchmark:
        tune_benchmark_workloads(a.table, only=a.only)
        return
    e = tune(a.session, a.field, a.lambda2, path=a.table, label=a.label)
    print(json.dumps({k: e[k] for k in ("best", "best_ms", "default_ms")}))


if __name__ == "__main__":
    main()
