"""FEML session writer for rectangular quad meshes (the role of `rectmesh`).

Produces the session files the benchmarks and tests run: an nx x ny grid of
quads on [x0,x1] x [y0,y1], optional periodic pairing in x and/or y, one
boundary group per remaining side kind, tokens and a USER section.
"""

from __future__ import annotations

import numpy as np


def rect_session(path, nx, ny, x=(0.0, 1.0), y=(0.0, 1.0), tokens=None, fields="c",
                 periodic_x=False, periodic_y=False, bcs=None, user=None, xs=None, ys=None,
                 wall_group="w", force=None, side_groups=None, group_names=None, history=None):
    """Write a session file.

    bcs: {group_char: {field: "<D> value" | "<N> value" | "<H>"}} applied to
    every non-periodic boundary side (group `wall_group`), or None for no BCs.
    xs / ys: explicit node coordinates along x / y (length nx+1 / ny+1).
    force: lines of a <FORCE> section ("CONST_X = 0.1", ...), or None.
    side_groups: {"bottom" | "top" | "left" | "right": group char} overriding
    `wall_group` on those sides; group_names: {group char: descriptor}
    ("wall" by default; "outflow" and "axis" are the reserved ones).
    history: (id, x, y, z) points of a <HISTORY> section, or None.
    """
    side_groups = side_groups or {}
    group_names = group_names or {}
    xs = np.linspace(x[0], x[1], nx + 1) if xs is None else np.asarray(xs, float)
    ys = np.linspace(y[0], y[1], ny + 1) if ys is None else np.asarray(ys, float)
    lines = []
    if user:
        lines.append("<USER>")
        lines += [f"\t{u}" for u in user]
        lines.append("</USER>\n")
    lines.append("<FIELDS>")
    lines.append("\t" + " ".join(fields))
    lines.append("</FIELDS>\n")
    lines.append("<TOKENS>")
    for k, v in (tokens or {}).items():
        lines.append(f"\t{k} = {v}")
    lines.append("</TOKENS>\n")
    if force is not None:
        lines.append("<FORCE>")
        lines += [f"\t{f}" for f in force]
        lines.append("</FORCE>\n")
    if history:
        lines.append(f"<HISTORY NUMBER={len(history)}>")
        lines += [f"\t{i}\t{hx:.17g}\t{hy:.17g}\t{hz:.17g}" for (i, hx, hy, hz) in history]
        lines.append("</HISTORY>\n")
    if bcs:
        lines.append(f"<GROUPS NUMBER={len(bcs)}>")
        for i, g in enumerate(bcs):
            lines.append(f"\t{i + 1}\t{g}\t{group_names.get(g, 'wall')}")
        lines.append("</GROUPS>\n")
        lines.append(f"<BCS NUMBER={len(bcs)}>")
        for i, (g, spec) in enumerate(bcs.items()):
            lines.append(f"\t{i + 1}\t{g}\t{len(spec)}")
            for f, s in spec.items():
                kind, _, val = s.partition(" ")
                tag = kind.strip("<>")
                lines.append(f"\t\t<{tag}>\t{f} = {val.strip() or 0}\t</{tag}>")
        lines.append("</BCS>\n")
    nn = (nx + 1) * (ny + 1)
    lines.append(f"<NODES NUMBER={nn}>")

    def nid(i, j):
        return j * (nx + 1) + i + 1

    for j in range(ny + 1):
        for i in range(nx + 1):
            lines.append(f"\t{nid(i, j)}\t{xs[i]:.17g}\t{ys[j]:.17g}\t0")
    lines.append("</NODES>\n")
    lines.append(f"<ELEMENTS NUMBER={nx * ny}>")

    def eid(i, j):
        return j * nx + i + 1

    for j in range(ny):
        for i in range(nx):
            lines.append(f"\t{eid(i, j)}\t<Q>\t{nid(i, j)} {nid(i + 1, j)} {nid(i + 1, j + 1)} "
                         f"{nid(i, j + 1)}\t</Q>")
    lines.append("</ELEMENTS>\n")
    surf = []
    # side 1 = bottom (y0), 2 = right (x1), 3 = top (y1), 4 = left (x0)
    for i in range(nx):
        if periodic_y:
            surf.append((eid(i, 0), 1, f"<P>\t{eid(i, ny - 1)} 3\t</P>"))
        elif bcs:
            surf.append((eid(i, 0), 1, f"<B>\t{side_groups.get('bottom', wall_group)}\t</B>"))
            surf.append((eid(i, ny - 1), 3, f"<B>\t{side_groups.get('top', wall_group)}\t</B>"))
    for j in range(ny):
        if periodic_x:
            surf.append((eid(0, j), 4, f"<P>\t{eid(nx - 1, j)} 2\t</P>"))
        elif bcs:
            surf.append((eid(0, j), 4, f"<B>\t{side_groups.get('left', wall_group)}\t</B>"))
            surf.append((eid(nx - 1, j), 2, f"<B>\t{side_groups.get('right', wall_group)}\t</B>"))
    lines.append(f"<SURFACES NUMBER={len(surf)}>")
    for k, (e, s, body) in enumerate(surf):
        lines.append(f"\t{k + 1}\t{e}\t{s}\t{body}")
    lines.append("</SURFACES>")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")
    return path


def helmholtz_session(path, n, np_, nz=1, lambda2=1.0, beta=1.0, extra=None, user=None, xs=None, ys=None):
    """Dirichlet-zero Helmholtz problem on [0,1]^2 (configs c1, c2, c4)."""
    tok = {"N_P": np_, "N_Z": nz, "LAMBDA2": lambda2, "BETA": beta, "TOL_REL": 1e-12}
    tok.update(extra or {})
    return rect_session(path, n, n, tokens=tok, fields="c", bcs={"w": {"c": "<D> 0.0"}},
                        user=user, xs=xs, ys=ys)


def taylor_green_session(path, n, np_, nz, re=1600.0, dt=1e-3, nstep=200, extra=None, force=None):
    """3D-periodic Taylor--Green vortex on [0, 2 pi]^3 (config c3)."""
    tok = {"N_P": np_, "N_Z": nz, "BETA": 1, "KINVIS": f"1.0/{re}", "D_T": dt, "N_TIME": 3,
           "N_STEP": nstep, "TOL_REL": 1e-13}
    tok.update(extra or {})
    user = ["u = sin(x)*cos(y)*cos(z)", "v = -cos(x)*sin(y)*cos(z)", "w = 0", "p = 0"]
    return rect_session(path, n, n, x=(0.0, 2 * np.pi), y=(0.0, 2 * np.pi), tokens=tok,
                        fields="uvwp", periodic_x=True, periodic_y=True, user=user, force=force)


def channel_session(path, nx=16, ny=8, np_=9, nz=32, re=500.0, dt=5e-3, nstep=100, ntime=3, extra=None,
                    force=None, history=None):
    """Plane channel [0, 2 pi] x [-1, 1] x [0, 2 pi), periodic in x and z,
    no-slip walls at y = +-1 with high-order pressure BCs (config c5)."""
    tok = {"N_P": np_, "N_Z": nz, "BETA": 1, "KINVIS": f"1.0/{re}", "D_T": dt, "N_TIME": ntime,
           "N_STEP": nstep, "TOL_REL": 1e-13}
    tok.update(extra or {})
    fields = "uvwp" if nz > 1 else "uvp"
    bc = {"u": "<D> 0", "v": "<D> 0", "p": "<H> 0"}
    if nz > 1:
        bc["w"] = "<D> 0"
    return rect_session(path, nx, ny, x=(0.0, 2 * np.pi), y=(-1.0, 1.0), tokens=tok, fields=fields,
                        periodic_x=True, bcs={"w": bc}, force=force, history=history)


def channel_initial(x, y, z, seed=20261203, amplitude=1e-3, modes=3):
    """Base flow u = 1 - y^2 plus a divergence-free perturbation from a seeded
    random stream function psi(x, y; z) = (1 - y^2)^2 sum a cos(kx x + b)
    cos(kz z + c):  u' = dpsi/dy, v' = -dpsi/dx, w' = 0, all zero at the
    walls; scaled so that max |u'| = amplitude.  x, y are node coordinates
    [nel, np, np]; z the plane positions.  Returns {u, v, w, p} arrays
    [nz, nel, np, np]."""
    rng = np.random.default_rng(seed)
    X = x[None]
    Y = y[None]
    Z = np.asarray(z, float)[:, None, None, None]
    g = (1 - Y * Y) ** 2
    dg = -4 * Y * (1 - Y * Y)
    up = np.zeros(Z.shape[:1] + x.shape)
    vp = np.zeros_like(up)
    for kx in range(1, modes + 1):
        for kz in range(0, modes if len(z) > 1 else 1):
            a, b, c = rng.uniform(-1, 1), rng.uniform(0, 2 * np.pi), rng.uniform(0, 2 * np.pi)
            cx, sx = np.cos(kx * X + b), np.sin(kx * X + b)
            cz = np.cos(kz * Z + c)
            up += a * dg * cx * cz
            vp += a * kx * g * sx * cz
    s = amplitude / max(np.abs(up).max(), 1e-300)
    base = np.broadcast_to(1 - Y * Y, up.shape)
    return {"u": base + s * up, "v": s * vp, "w": np.zeros_like(up), "p": np.zeros_like(up)}


def forcing_per_unique_node(x, y, nz, seed):
    """U[-1,1] per unique (x, y, z) node, identical on coincident element
    copies.  x, y are node coordinates [nel, np, np]; returns the forcing
    [nz, nel, np, np] and the number of unique nodes per plane."""
    key = np.round(x * 1e9).astype(np.int64) * 4000000007 + np.round(y * 1e9).astype(np.int64)
    uniq, inv = np.unique(key.ravel(), return_inverse=True)
    rng = np.random.default_rng(seed)
    vals = rng.uniform(-1.0, 1.0, (nz, len(uniq)))
    return vals[:, inv].reshape((nz,) + x.shape), len(uniq)


def uneven_batch(count=64, seed=20261203, n_range=(4, 32), order_range=(6, 12), lambda2_range=(0.1, 100.0)):
    """The uneven batch of independent 2D Helmholtz problems (config c4):
    n x n quads on [0,1]^2 with n uniform in n_range, polynomial order N
    uniform in order_range (N_P = N + 1), lambda^2 log-uniform in
    lambda2_range, Dirichlet zero; forcing seeds follow.  Returns a list of
    dicts (n, np, lambda2, seed)."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = int(rng.integers(n_range[0], n_range[1] + 1))
        order = int(rng.integers(order_range[0], order_range[1] + 1))
        lam = float(np.exp(rng.uniform(np.log(lambda2_range[0]), np.log(lambda2_range[1]))))
        out.append({"n": n, "np": order + 1, "lambda2": lam, "seed": seed + 1 + i})
    return out
