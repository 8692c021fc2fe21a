"""Oracle checksums of the benchmark-size workloads (c2, c3, c3 with 3/2-rule
products, c5, the c4 batch), for GPU parity tests at full size.

The full oracle fields are too large to commit (c3: 36 MB per field), and the
oracle takes minutes at these sizes, so each field is reduced to numbers that
carry its relative L2 error:

- ``norm``: the 2-norm of the whole field;
- ``proj``: its inner products with four seeded standard-normal vectors (for
  a difference d, <d, r> has standard deviation ||d||, so a projection
  error over ||field|| estimates the relative L2 error of the whole field);
- ``idx`` / ``val``: the values at 256 seeded positions.

Fields are physical space, flattened [nz, nel, np, np].  ``checksums`` below
is the one routine both this script and the tests use.  Every input is
regenerated from the package's seeded session builders, so the GPU side needs
nothing but this file's output (tests/golden/baseline/*.npz).

Usage: python tests/golden/make_baseline_fixtures.py [c2|c3|c3d|c5|c4 ...]
"""

from __future__ import annotations

import os
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
OUT = os.path.join(HERE, "baseline")
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)

NPROJ, NSAMPLE, SEED = 4, 256, 20261203

# workload definitions shared with the tests
C2 = dict(n=16, np_=11, nz=64, lambda2=1.0, beta=1.0, seed=20261203)
C3_STEPS = 5
C5_STEPS = 10


def probes(n):
    """Seeded projection vectors [NPROJ, n] and sample positions [NSAMPLE]."""
    rng = np.random.default_rng(SEED + n)
    R = rng.standard_normal((NPROJ, n))
    idx = np.sort(rng.choice(n, size=min(NSAMPLE, n), replace=False))
    return R, idx


def checksums(a):
    a = np.ascontiguousarray(a, dtype=np.float64).ravel()
    R, idx = probes(a.size)
    return {"norm": np.linalg.norm(a), "proj": R @ a, "idx": idx, "val": a[idx]}


def errors(got, ref, scale=None):
    """Relative errors of a field `got` against the checksums `ref`, relative
    to `scale` (default: the reference field's 2-norm): projections (max),
    samples (2-norm over the samples, scaled by the samples' share of the
    field), norm."""
    c = checksums(got)
    scale = max(float(ref["norm"]) if scale is None else float(scale), 1e-300)
    e_proj = float(np.max(np.abs(c["proj"] - ref["proj"]))) / scale
    share = np.sqrt(len(ref["idx"]) / max(np.asarray(got).size, 1))
    e_val = float(np.linalg.norm(c["val"] - ref["val"])) / (scale * share)
    e_norm = abs(float(c["norm"]) - float(ref["norm"])) / scale
    return {"proj": e_proj, "sample": e_val, "norm": e_norm}


def load(name):
    z = np.load(os.path.join(OUT, f"{name}.npz"))
    out = {}
    for k in z.files:
        fld, _, item = k.partition(".")
        out.setdefault(fld, {})[item] = z[k]
    return out


def _save(name, fields, meta=None):
    os.makedirs(OUT, exist_ok=True)
    arrs = {}
    for fld, a in fields.items():
        for item, v in checksums(a).items():
            arrs[f"{fld}.{item}"] = v
    for k, v in (meta or {}).items():
        arrs[f"meta.{k}"] = np.asarray(v)
    np.savez_compressed(os.path.join(OUT, f"{name}.npz"), **arrs)


# ---- the workloads (the same builders and seeds as bench.py) --------------

def c2_session(d):
    from semtex_b200 import sessions
    w = C2
    return sessions.helmholtz_session(os.path.join(d, "c2"), w["n"], w["np_"], nz=w["nz"],
                                      lambda2=w["lambda2"], beta=w["beta"])


def c3_session(d, dealias):
    from semtex_b200 import sessions
    return sessions.taylor_green_session(os.path.join(d, "c3d" if dealias else "c3"), 24, 9, 96, re=1600.0,
                                         dt=1e-3, nstep=200, extra={"DEALIAS": 1} if dealias else None)


def c5_session(d):
    from semtex_b200 import sessions
    return sessions.channel_session(os.path.join(d, "c5"), 16, 8, 9, 32, re=500.0, dt=5e-3, nstep=100)


def c5_initial(x, y, nz):
    from semtex_b200 import sessions
    return sessions.channel_initial(x, y, np.arange(nz) * 2 * np.pi / nz)


def c4_problem(d, i, sp):
    from semtex_b200 import sessions
    return sessions.helmholtz_session(os.path.join(d, f"p{i}"), sp["n"], sp["np"], lambda2=sp["lambda2"])


def make_c2(d):
    import semtex_oracle as O
    from semtex_b200 import sessions
    p = c2_session(d)
    P = O.Problem(O.read_session(p))
    f, _ = sessions.forcing_per_unique_node(P.M.x, P.M.y, P.nz, C2["seed"])
    _, U = O.elliptic(p, forcing_phys=f)
    _save("c2", {"c": U})


def make_dns(d, name):
    import semtex_oracle as O
    if name == "c5":
        p = c5_session(d)
        P = O.Problem(O.read_session(p))
        D = O.DNS(P, c5_initial(P.M.x, P.M.y, P.nz))
        steps = C5_STEPS
    else:
        p = c3_session(d, name == "c3d")
        S = O.read_session(p)
        P = O.Problem(S)
        funcs = O.user_functions(S)
        D = O.DNS(P, {c: P.evaluate(funcs[c], 0.0) for c in S.fields if c in funcs})
        steps = C3_STEPS
    D.advance(steps)
    _save(name, D.physical(), {"steps": steps, "time": D.time})


def make_c4(d):
    import semtex_oracle as O
    from semtex_b200 import sessions
    fields = {}
    for i, sp in enumerate(sessions.uneven_batch()):
        p = c4_problem(d, i, sp)
        P = O.Problem(O.read_session(p))
        f, _ = sessions.forcing_per_unique_node(P.M.x, P.M.y, 1, sp["seed"])
        _, U = O.elliptic(p, forcing_phys=f)
        fields[f"p{i}"] = U
    _save("c4", fields)


def main(cases):
    for c in cases:
        t0 = time.time()
        with tempfile.TemporaryDirectory() as d:
            if c == "c2":
                make_c2(d)
            elif c in ("c3", "c3d", "c5"):
                make_dns(d, c)
            elif c == "c4":
                make_c4(d)
            else:
                raise SystemExit(f"unknown case {c}")
        print(f"{c}: {time.time() - t0:.1f} s", flush=True)


if __name__ == "__main__":
    main(sys.argv[1:] or ["c2", "c5", "c4", "c3", "c3d"])
