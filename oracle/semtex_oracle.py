"""CPU oracle for the Semtex spectral-element--Fourier hot path (TEST INFRASTRUCTURE).

This module is the checker, not the product.  Only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg import it.
It restates, in numpy/scipy, the reference algorithm of the path that the
CUDA library accelerates:

* FEML session reading and token evaluation  (src/feml.cpp:64-330,
  femlib/initial.y:138-249, femlib/defaults.h:10-96)
* straight-sided quad meshing with a Coons patch (src/mesh.cpp:723-882)
* GLL quadrature and derivative operators     (femlib/polylib.c:312-575)
* element geometric factors                    (src/element.cpp:1253-1408)
* elemental Helmholtz matrix / operator        (src/element.cpp:1411-1622)
* static condensation                          (src/element.cpp:131-214)
* banded Cholesky boundary system              (src/matrix.cpp:132-267)
* Field::solve DIRECT / JACPCG                 (src/field.cpp:598-809)
* z-direction real DFT, packed Re0,Nyq,Re1,Im1 (femlib/fourier.c:40-165)
* the DNS velocity-correction step             (dns/integrate.cpp:66-289,
  dns/nonlinear.cpp:38-530)
* body forcing, SVV                            (dns/fieldforce.cpp, src/svv.cpp)
* cylindrical coordinates with axis BCs        (src/element.cpp:1389-1399,
  src/field.cpp:1127-1227, src/bcmgr.cpp:153-180, src/edge.cpp:98-256)
* computed outflow BCs                         (src/bcmgr.cpp:998-1633;
  parity unpinned: the reference has no golden for them)
* history points and wall forces               (src/history.cpp:45-78,
  src/element.cpp:1061-1203, src/auxfield.cpp:1621-1700,
  src/field.cpp:392-458, src/edge.cpp:259-378; parity unpinned: no
  reference golden holds them)

The banded factorisation and solve call LAPACK dpbtrf/dpbtrs through scipy,
the same routines the reference calls (src/matrix.cpp:252, src/field.cpp:693).

Node numbering is this module's own (connectivity + reverse Cuthill--McKee)
where a field has essential nodes: it differs from the reference `enumerate`
output only in round-off.  A field without essential nodes has a singular k=0
system whose pinned node (src/matrix.cpp:160-162) is the highest-numbered
solve node; where the discrete Neumann data are not compatible (high-order
pressure BCs) the pin changes the whole solution, not only a constant.  Such
fields take the reference's own `enumerate -O3` numbering (`reference_map`,
`enumerate_o3`), which reproduces the regress goldens of the kovas sessions
in every field.
"""

from __future__ import annotations

import math
import os
import re
import time
from dataclasses import dataclass, field as dfield

import numpy as np
import scipy.linalg as sla
from scipy.sparse import csr_matrix
from scipy.sparse.csgraph import reverse_cuthill_mckee

EPSDP = 6.0e-14          # veclib/cveclib.h:58
EPSSP = 6.0e-7

# ---------------------------------------------------------------------------
# Tokens and expressions (femlib/defaults.h, femlib/initial.y)
# ---------------------------------------------------------------------------

DEFAULT_TOKENS = {
    "E": 2.71828182845904523536, "DEG": 57.29577951308232087721,
    "PI": 3.14159265358979323844, "TWOPI": 6.28318530717958647688,
    "EULER": 0.57721566490153286061, "GOLDEN": 1.61803398874989484820,
    "t": 0.0, "D_T": 0.01, "TOL_REL": 1.0e-8, "TOL_ABS": 1.0e-8,
    "TOL_POS": 1.0e-5, "z": 0.0, "BETA": 1.0, "LAMBDA2": 0.0,
    "KINVIS": 1.0, "REFVIS": 1.0, "RHO": 1.0, "GRAVITY": 9.81,
    "X_SHIFT": 0.0, "Y_SHIFT": 0.0, "X_SCALE": 1.0, "Y_SCALE": 1.0,
    "SVV_MN": -1, "SVV_EPSN": 0.0, "SVV_MZ": -1, "SVV_EPSZ": 0.0,
    "ITERATIVE": 0, "TBCS": 0, "CYLINDRICAL": 0, "VERBOSE": 0,
    "CHKPOINT": 1, "IO_FLD": 500, "IO_HIS": 10, "IO_CFL": 50, "IO_MDL": 50,
    "N_P": 5, "N_TIME": 2, "N_STEP": 1, "N_Z": 1, "I_PROC": 0, "N_PROC": 1,
    "STEP_MAX": 500, "NR_MAX": 20, "FFX": 0.0, "FFY": 0.0, "FFZ": 0.0,
}

_FUNCS = {
    "cos": np.cos, "sin": np.sin, "tan": np.tan, "exp": np.exp,
    "sinh": np.sinh, "cosh": np.cosh, "tanh": np.tanh, "abs": np.abs,
    "floor": np.floor, "ceil": np.ceil, "acos": np.arccos, "asin": np.arcsin,
    "atan": np.arctan, "log": np.log, "log10": np.log10, "sqrt": np.sqrt,
    "int": np.rint, "sgn": np.sign,
    "heav": lambda x: np.where(np.asarray(x) >= 0.0, 1.0, 0.0),
}


class Tokens(dict):
    """Token table with the reference defaults and its expression grammar.

    Grammar of femlib/initial.y:196-249: '^' is right-associative power with
    higher precedence than unary minus, which python's '**' shares.
    """

    def __init__(self):
        super().__init__(DEFAULT_TOKENS)

    def evaluate(self, expr: str, **variables):
        src = expr.strip().replace("^", "**")
        if "&" in src or "~" in src:
            raise ValueError(f"operator not supported by the oracle: {expr}")
        names = dict(_FUNCS)
        names.update(self)
        names.update(variables)
        return eval(src, {"__builtins__": {}}, names)  # noqa: S307 (test oracle)

    def assign(self, line: str):
        name, expr = line.split("=", 1)
        self[name.strip()] = float(self.evaluate(expr))

    def ivalue(self, name):
        return int(round(float(self[name])))


# ---------------------------------------------------------------------------
# FEML session (src/feml.cpp, src/mesh.cpp:129-470, src/bcmgr.cpp:100-110)
# ---------------------------------------------------------------------------

@dataclass
class Session:
    name: str
    tokens: Tokens
    fields: str
    groups: dict                 # group char -> descriptor string
    bcs: dict                    # group char -> {field: (kind, expr)}
    nodes: np.ndarray            # [Nn, 3]
    elements: np.ndarray         # [nel, 4] zero-based node ids (CCW)
    surfaces: list               # (elmt, side, 'B', group) | (elmt, side, 'P', (me, ms))
    user: list = dfield(default_factory=list)
    force: list | None = None    # raw lines of the FORCE section, None if absent


def _section(text: str, name: str):
    m = re.search(r"<\s*" + name + r"\b([^>]*)>(.*?)</\s*" + name + r"\s*>",
                  text, re.S | re.I)
    if not m:
        return None, None
    return m.group(1), m.group(2)


def _lines(body: str):
    out = []
    for ln in body.splitlines():
        s = ln.strip()
        if s and not s.startswith("#"):
            out.append(s)
    return out


def read_session(path: str, overrides: dict | None = None) -> Session:
    """Read a FEML session file (src/feml.cpp:64-330, src/mesh.cpp:129-470)."""
    text = open(path).read()
    tok = Tokens()
    _, body = _section(text, "TOKENS")
    if body:
        for ln in body.splitlines():
            if "=" in ln and not ln.strip().startswith("#"):
                tok.assign(ln)
    for k, v in (overrides or {}).items():
        tok[k] = float(v)
    if tok.ivalue("IO_FLD") > tok.ivalue("N_STEP"):
        tok["IO_FLD"] = tok["N_STEP"]
    if tok.ivalue("N_TIME") > 3:
        tok["N_TIME"] = 3
    _, body = _section(text, "FIELDS")
    fields = "".join(body.split())
    groups = {}
    _, body = _section(text, "GROUPS")
    if body:
        for ln in _lines(body):
            parts = ln.split()
            groups[parts[1]] = parts[2]
    bcs = {}
    _, body = _section(text, "BCS")
    if body:
        lines = _lines(body)
        i = 0
        while i < len(lines):
            parts = lines[i].split()
            g, nf = parts[1], int(parts[2])
            entry = {}
            for j in range(nf):
                m = re.match(r"<\s*([A-Z])\s*>\s*(\w)\s*=?\s*(.*?)\s*</\s*[A-Z]\s*>",
                             lines[i + 1 + j])
                kind, fname, expr = m.group(1), m.group(2), m.group(3)
                entry[fname] = (kind, expr)
            bcs[g] = entry
            i += 1 + nf
    _, body = _section(text, "NODES")
    nodes = np.array([[float(v) for v in ln.split()[1:4]] for ln in _lines(body)])
    _, body = _section(text, "ELEMENTS")
    elems = []
    for ln in _lines(body):
        m = re.match(r"(\d+)\s*<\s*Q\s*>\s*(\d+)\s+(\d+)\s+(\d+)\s+(\d+)", ln)
        elems.append([int(m.group(k)) - 1 for k in range(2, 6)])
    surfaces = []
    _, body = _section(text, "SURFACES")
    if body:
        for ln in _lines(body):
            m = re.match(r"\d+\s+(\d+)\s+(\d+)\s*<\s*([BP])\s*>\s*(.*?)\s*</", ln)
            e, s, kind, rest = int(m.group(1)) - 1, int(m.group(2)) - 1, m.group(3), m.group(4)
            if kind == "B":
                surfaces.append((e, s, "B", rest.strip()))
            else:
                me, ms = rest.split()
                surfaces.append((e, s, "P", (int(me) - 1, int(ms) - 1)))
    _, curves = _section(text, "CURVES")
    if curves and _lines(curves):
        raise NotImplementedError("curved sides are outside the oracle's scope")
    _, body = _section(text, "USER")
    user = _lines(body) if body else []
    _, body = _section(text, "FORCE")
    force = None if body is None else [ln.rstrip("\r") for ln in body.split("\n")[1:]]
    name = os.path.basename(path)
    return Session(name, tok, fields, groups, bcs, nodes, np.array(elems, int),
                   surfaces, user, force)


def force_value(S: Session, token: str):
    """FEML::valueFromSection on the FORCE section (src/feml.cpp:519-560):
    the first line whose first word (words end at tab, '=' or space) is
    `token` gives the text after it up to the next '='.  A '#' line is read
    together with the line after it and both are skipped.  None if absent."""
    lines = S.force or []
    k = 0
    while k < len(lines):
        s = lines[k]
        k += 1
        if s.startswith("#"):
            k += 1
            continue
        m = re.match(r"[\t= ]*([^\t= ]+)", s)
        if not m or m.group(1) != token:
            continue
        rest = s[m.end(1) + 1:] if m.end(1) < len(s) else ""
        rest = rest.lstrip("=")
        val = rest.split("=", 1)[0]
        return val if val else None
    return None


# ---------------------------------------------------------------------------
# GLL quadrature (femlib/polylib.c:312-575): zeros, weights, derivative matrix
# ---------------------------------------------------------------------------

def _legendre(n, x):
    p0, p1 = np.ones_like(x), x.copy()
    if n == 0:
        return p0
    for k in range(2, n + 1):
        p0, p1 = p1, ((2 * k - 1) * x * p1 - (k - 1) * p0) / k
    return p1


def gll(np_: int):
    """GLL points z, weights w, derivative D[i,j] = h_j'(z_i) (row-major)."""
    N = np_ - 1
    if np_ == 2:
        z = np.array([-1.0, 1.0])
    else:
        # interior points: zeros of P_N'(x) via the Jacobi P^{(1,1)}_{N-1}
        # companion (Golub--Welsch) eigenvalues, then Newton polish.
        n = N - 1
        k = np.arange(1, n)
        b = np.sqrt(k * (k + 2.0) / ((2 * k + 1.0) * (2 * k + 3.0)))
        J = np.diag(b, 1) + np.diag(b, -1)
        zi = np.sort(np.linalg.eigvalsh(J)) if n > 1 else np.array([0.0])
        for _ in range(6):
            # P_N'(x) = N (x P_N - P_{N-1}) / (x^2 - 1)
            pn, pn1 = _legendre(N, zi), _legendre(N - 1, zi)
            d1 = N * (zi * pn - pn1) / (zi * zi - 1.0)
            d2 = (2 * zi * d1 - N * (N + 1) * pn) / (1.0 - zi * zi)
            zi = zi - d1 / d2
        z = np.concatenate([[-1.0], zi, [1.0]])
    PN = _legendre(N, z)
    w = 2.0 / (N * (N + 1) * PN * PN)
    D = np.zeros((np_, np_))
    for i in range(np_):
        for j in range(np_):
            if i != j:
                D[i, j] = PN[i] / (PN[j] * (z[i] - z[j]))
    D[0, 0] = -N * (N + 1) / 4.0
    D[N, N] = N * (N + 1) / 4.0
    return z, w, D


def svv_derivative(z, w, D, eps, mN, nu):
    """SVV-modified derivative MI diag(sqrt S) MF D (SVV::operators,
    src/svv.cpp:126-185): MF, MI the GLL Legendre transform pair
    (femlib/operators.c:317-490, C_k = 1/gamma_k of the discrete norms),
    S_k = 1 + eps/nu exp(-((N-k)/(mN-k))^2) for k > mN (SVV::coeffs,
    :20-52).  None when SVV is off."""
    np_ = len(z)
    N = np_ - 1
    if not (0 <= mN < N and eps > EPSDP):
        return None
    S = np.zeros(np_)
    for k in range(mN + 1, np_):
        S[k] = math.exp(-((N - k) / (1.0 * mN - k)) ** 2)
    S = 1.0 + eps / nu * S
    L = np.array([_legendre(k, z) for k in range(np_)])        # L[k, j] = P_k(z_j)
    C = np.array([0.5 * (2 * k + 1) if k < N else 0.5 * N for k in range(np_)])
    MF = C[:, None] * w[None, :] * L
    MI = L.T
    return MI @ (np.sqrt(S)[:, None] * MF) @ D


def svv_z(nz, num_modes, eps, mN, nu):
    """SVV::coeffs_z (src/svv.cpp:55-90): factors of beta^2 k^2 for the
    viscous systems' modes, N = nMode - 1."""
    N = (nz + 1) // 2 - 1
    S = np.zeros(num_modes)
    if 0 <= mN < N and eps > EPSDP:
        for i in range(num_modes):
            if i > mN:
                S[i] = math.exp(-((N - i) / (1.0 * mN - i)) ** 2)
        return 1.0 + eps / nu * S
    return np.ones(num_modes)


# ---------------------------------------------------------------------------
# Mesh and element geometry
# ---------------------------------------------------------------------------

class Mesh:
    """Element node locations and connectivity for straight-sided quads."""

    def __init__(self, S: Session, np_: int):
        self.S, self.np = S, np_
        self.nel = len(S.elements)
        self.z, self.w, self.D = gll(np_)
        nel, z = self.nel, self.z
        tok = S.tokens
        # viscous operators take the SVV-stabilised derivative (src/element.cpp:1454-1455)
        self.Dv = self.D
        if tok["SVV_EPSN"] > EPSDP:
            if tok["SVV_MN"] > np_:
                raise ValueError("SVV_MN exceeds N_P")      # dns/drive.cpp:244-245
            Dv = svv_derivative(self.z, self.w, self.D, tok["SVV_EPSN"], int(tok["SVV_MN"]), tok["KINVIS"])
            if Dv is not None:
                self.Dv = Dv
        x = np.zeros((nel, np_, np_))
        y = np.zeros((nel, np_, np_))
        for e in range(nel):
            P = S.nodes[S.elements[e], :2]
            # side k runs from vertex k to vertex k+1 (src/mesh.cpp:804-844):
            # Coons patch of straight sides == bilinear map of the 4 vertices.
            r = z[None, :]
            s = z[:, None]
            for arr, c in ((x, 0), (y, 1)):
                arr[e] = 0.25 * ((1 - r) * (1 - s) * P[0, c] + (1 + r) * (1 - s) * P[1, c]
                                 + (1 + r) * (1 + s) * P[2, c] + (1 - r) * (1 + s) * P[3, c])
        if abs(tok["X_SHIFT"]) > EPSDP:
            x += tok["X_SHIFT"]
        if abs(tok["Y_SHIFT"]) > EPSDP:
            y += tok["Y_SHIFT"]
        if abs(tok["X_SCALE"] - 1.0) > EPSDP:
            x *= tok["X_SCALE"]
        if abs(tok["Y_SCALE"] - 1.0) > EPSDP:
            y *= tok["Y_SCALE"]
        self.x, self.y = x, y
        self._factors()
        # Cylindrical coordinates (x axial, y radial, z azimuthal): the
        # quadrature of Q1-Q4 premultiplied by r = y; Q8 keeps the plain
        # mass, which weights forcing (src/element.cpp:1389-1399, 800-806)
        self.cyl = tok.ivalue("CYLINDRICAL") > 0
        self.Q8 = self.Q4.copy()
        if self.cyl:
            for nm in ("Q1", "Q2", "Q3", "Q4"):
                setattr(self, nm, getattr(self, nm) * self.y)
        self._connect()

    # -- src/element.cpp:1253-1408 (Element::mapping)
    def _factors(self):
        D, w = self.D, self.w
        x, y = self.x, self.y
        dxdr = x @ D.T
        dxds = D @ x
        dydr = y @ D.T
        dyds = D @ y
        jac = dxdr * dyds - dxds * dydr
        if jac.min() < 4 * EPSDP:
            raise ValueError("Jacobian of element nonpositive")
        WW = np.outer(w, w)[None]
        self.Q1 = (dxds * dxds + dyds * dyds) / jac * WW
        self.Q2 = (dxdr * dxdr + dydr * dydr) / jac * WW
        self.Q3 = (-dydr * dyds - dxdr * dxds) / jac * WW
        self.Q4 = jac * WW
        self.drdx = dyds / jac
        self.drdy = -dxds / jac
        self.dsdx = -dydr / jac
        self.dsdy = dxdr / jac
        eps = 4 * EPSDP
        for nm in ("drdx", "drdy", "dsdx", "dsdy", "Q3"):
            a = getattr(self, nm)
            for e in range(self.nel):
                if np.linalg.norm(a[e]) < eps:
                    a[e] = 0.0

    # -- element-boundary node traverse (femlib/mapping.c:46-132)
    def emap(self):
        n = self.np
        em = [0]
        k = 0
        for _ in range(1, n):
            k += 1
            em.append(k)
        for _ in range(1, n):
            k += n
            em.append(k)
        for _ in range(1, n):
            k -= 1
            em.append(k)
        for _ in range(1, n - 1):
            k -= n
            em.append(k)
        for i in range(1, n - 1):
            for j in range(1, n - 1):
                em.append(i * n + j)
        return np.array(em, int)

    def _connect(self):
        """Side mates: shared vertex pairs (internal) or <P> surfaces."""
        S = self.S
        nel = self.nel
        self.mate = {}
        key = {}
        for e in range(nel):
            for s in range(4):
                a, b = S.elements[e][s], S.elements[e][(s + 1) % 4]
                key.setdefault((a, b), []).append((e, s))
        for e in range(nel):
            for s in range(4):
                a, b = S.elements[e][s], S.elements[e][(s + 1) % 4]
                for (me, ms) in key.get((b, a), []):
                    self.mate[(e, s)] = (me, ms)
        self.group = {}
        for (e, s, kind, val) in S.surfaces:
            if kind == "B":
                self.group[(e, s)] = val
            else:
                self.mate[(e, s)] = val
                self.mate[val] = (e, s)

    def side_nodes(self, s):
        """Row-major indices of the np nodes of side s, CCW (src/element.h:162)."""
        n = self.np
        if s == 0:
            return [j for j in range(n)]
        if s == 1:
            return [i * n + n - 1 for i in range(n)]
        if s == 2:
            return [(n - 1) * n + (n - 1 - j) for j in range(n)]
        return [(n - 1 - i) * n for i in range(n)]


class Numbering:
    """Global numbering of element-boundary nodes for one field.

    Role of the `.num` NumberSys (src/numbersys.h, src/bcmgr.cpp:586-826):
    btog[e, i] for the 4(np-1) boundary nodes of element e in emap order,
    bmask (1 = essential), solve nodes numbered first, RCM-ordered.
    """

    def __init__(self, M: Mesh, fld: str, rcm: bool = True, mclass: int = 0, btog=None):
        """btog: a precomputed map (the `.num` file's contents, as the
        reference's dns reads it) used instead of this restatement's RCM /
        `enumerate -O3` ordering; the CPU timings pass one to skip the -O3
        search, which tries every node as root."""
        S, n, nel = M.S, M.np, M.nel
        nm = n - 1
        next_ = 4 * nm
        parent = list(range(len(S.nodes)))

        def find(a):
            while parent[a] != a:
                parent[a] = parent[parent[a]]
                a = parent[a]
            return a

        for (e, s), (me, ms) in M.mate.items():
            a, b = S.elements[e][s], S.elements[e][(s + 1) % 4]
            c, d = S.elements[me][ms], S.elements[me][(ms + 1) % 4]
            for u, v in ((a, d), (b, c)):
                ru, rv = find(u), find(v)
                if ru != rv:
                    parent[max(ru, rv)] = min(ru, rv)
        gid = -np.ones((nel, next_), int)
        vid = {}
        nxt = 0
        for e in range(nel):
            for s in range(4):
                r = find(S.elements[e][s])
                if r not in vid:
                    vid[r] = nxt
                    nxt += 1
                gid[e, s * nm] = vid[r]
        done = {}
        for e in range(nel):
            for s in range(4):
                if (e, s) in done:
                    ids = done[(e, s)]
                else:
                    ids = list(range(nxt, nxt + nm - 1))
                    nxt += nm - 1
                    if (e, s) in M.mate:
                        done[M.mate[(e, s)]] = ids[::-1]
                gid[e, s * nm + 1: s * nm + nm] = ids
        nglobal = nxt
        ess = np.zeros(nglobal, bool)
        for (e, s), g in M.group.items():
            if (e, s) in M.mate:
                continue
            bc = S.bcs.get(g, {}).get(fld)
            if bc and (axis_kind(bc[0], fld, mclass) == "D" or (bc[0] == "O" and fld == "p")):
                for t in range(n):
                    ess[gid[e, (s * nm + t) % next_]] = True
        solve_nodes = np.where(~ess)[0]
        ess_nodes = np.where(ess)[0]
        nsolve = len(solve_nodes)
        order = solve_nodes
        if rcm and nsolve > 1:
            loc = -np.ones(nglobal, int)
            loc[solve_nodes] = np.arange(nsolve)
            rows, cols = [], []
            for e in range(nel):
                g = loc[gid[e]]
                g = np.unique(g[g >= 0])
                rr, cc = np.meshgrid(g, g)
                rows.append(rr.ravel())
                cols.append(cc.ravel())
            A = csr_matrix((np.ones(sum(len(r) for r in rows)),
                            (np.concatenate(rows), np.concatenate(cols))),
                           shape=(nsolve, nsolve))
            perm = reverse_cuthill_mckee(A, symmetric_mode=True)
            order = solve_nodes[perm]
        newid = np.empty(nglobal, int)
        newid[order] = np.arange(nsolve)
        newid[ess_nodes] = nsolve + np.arange(len(ess_nodes))
        self.btog = newid[gid]
        if btog is not None:
            self.btog = np.asarray(btog, int).reshape(nel, next_)
        elif rcm and not len(ess_nodes):
            # no essential nodes: the k=0 system of this field is singular and
            # its pinned node (the highest number) decides the solution, so
            # the reference's own numbering is used
            self.btog = enumerate_o3(reference_map(M))
        self.bmask = ess[gid].astype(int)
        self.emask = self.bmask.any(axis=1).astype(int)
        self.nglobal, self.nsolve = nglobal, nsolve
        bw = 0
        for e in range(nel):
            g = self.btog[e][self.btog[e] < nsolve]
            if len(g):
                bw = max(bw, g.max() - g.min())
        self.nband = bw + 1
        em = M.emap()
        mass = np.zeros(nglobal)
        for e in range(nel):
            np.add.at(mass, self.btog[e], _dssum_weight(M, e)[em[:next_]])
        self.imass = 1.0 / mass


def _choose_node(per, n1, n2):
    """Mesh::chooseNode (src/mesh.cpp:479-531): periodic representative of a
    vertex pair, the lower node id among the alternatives (fixPeriodic,
    :538-554, changes nothing)."""
    p1, p2 = per[n1], per[n2]
    if p1 is None:
        if p2 is None:
            pn = min(n1, n2)
            per[n1] = per[n2] = pn
        elif p2 != n2:
            pn = n1 if n1 < p2 else p2
            per[n1] = per[n2] = pn
            per[p2] = pn
        else:
            pn = min(n1, n2)
            per[n1] = per[n2] = pn
    elif p1 != n1:
        if p2 is None:
            pn = p1 if p1 < n2 else n2
            per[n2] = per[n1] = pn
            per[p1] = pn
        elif p2 != n2:
            pn = p1 if p1 < p2 else p2
            per[n1] = per[n2] = pn
            per[p1] = pn
            per[p2] = pn
        else:
            pn = p1 if p1 < n2 else n2
            per[n2] = per[n1] = pn
            per[p1] = pn
    else:
        if p2 is None:
            pn = min(n1, n2)
            per[n1] = per[n2] = pn
        elif p2 != n2:
            pn = n1 if n1 < p2 else n2
            per[n2] = per[n1] = pn
            per[p1] = pn
        else:
            pn = min(n1, n2)
            per[n1] = per[n2] = pn


def reference_map(M: "Mesh"):
    """Mesh::buildMap (src/mesh.cpp:884-990, Side::connect :994-1030): the
    reference's initial global numbers of element-boundary nodes, [nel, next]
    in boundary-major order (side s, knot t at s*(np-1) + t)."""
    S, n, nel = M.S, M.np, M.nel
    nm, ni = n - 1, n - 2
    per = [None] * len(S.nodes)
    for (e, s, kind, val) in S.surfaces:
        if kind == "P":
            me, ms = val
            _choose_node(per, S.elements[e][s], S.elements[me][(ms + 1) % 4])
            _choose_node(per, S.elements[e][(s + 1) % 4], S.elements[me][ms])
    vg = [-1] * len(S.nodes)
    sg = {}
    nxt = 0

    def vertex(v):
        nonlocal nxt
        p = per[v]
        if p is not None:
            if vg[p] < 0:
                vg[p] = nxt
                nxt += 1
            if vg[v] < 0:
                vg[v] = vg[p]
        if vg[v] < 0:
            vg[v] = nxt
            nxt += 1

    for e in range(nel):
        for s in range(4):
            vertex(S.elements[e][s])
            if ni:
                m = M.mate.get((e, s))
                if m is not None and m in sg:
                    sg[(e, s)] = sg[m][::-1]
                else:
                    sg[(e, s)] = list(range(nxt, nxt + ni))
                    nxt += ni
            vertex(S.elements[e][(s + 1) % 4])
    out = np.empty((nel, 4 * nm), int)
    for e in range(nel):
        for s in range(4):
            out[e, s * nm] = vg[S.elements[e][s]]
            out[e, s * nm + 1: s * nm + nm] = sg.get((e, s), [])
    return out


def _sparspak_rcm(root, adj, deg):
    """RCM of the component of root (George & Liu, SPARSPAK RCM/DEGREE as in
    femlib/netlib.f:1678-1890): breadth-first levels, each node's new
    neighbours in adjacency order, stably sorted by degree; reversed."""
    mask = np.ones(len(adj), bool)
    mask[root] = False
    perm = [root]
    lvlend = 0
    while True:
        lbegin, lvlend = lvlend, len(perm)
        for i in range(lbegin, lvlend):
            fnbr = len(perm)
            for nb in adj[perm[i]]:
                if mask[nb]:
                    mask[nb] = False
                    perm.append(nb)
            if len(perm) - fnbr > 1:
                perm[fnbr:] = sorted(perm[fnbr:], key=lambda v: deg[v])
        if len(perm) <= lvlend:
            break
    return perm[::-1]


_O3_CACHE = {}


def enumerate_o3(bmap):
    """`enumerate -O3` of a field without essential nodes (utility/
    enumerate.cpp:694-831, connectivSC :883-920, globalBandwidth :923-964):
    every node in turn as the RCM root, the first with the least global
    bandwidth kept.  bmap [nel, next] holds Mesh::buildMap numbers; returns
    the renumbered map (the chosen root becomes the highest number).  The
    fields of one mesh often share a map: results are cached by map."""
    key = (bmap.shape, np.ascontiguousarray(bmap, dtype=np.int64).tobytes())
    if key not in _O3_CACHE:
        _O3_CACHE[key] = _enumerate_o3(bmap)
    return _O3_CACHE[key].copy()


def _enumerate_o3(bmap):
    nel, nxt = bmap.shape
    nsolve = int(bmap.max()) + 1
    adj = [[] for _ in range(nsolve)]
    for e in range(nel):
        row = [int(v) for v in bmap[e]]
        for i in range(nxt):
            a = adj[row[i]]
            for j in range(nxt):
                if i != j and row[j] not in a:
                    a.append(row[j])
    deg = [len(a) for a in adj]
    lo_hi = [(sorted(set(int(v) for v in bmap[e]))) for e in range(nel)]
    best, best_root = None, 0
    for root in range(nsolve):
        perm = _sparspak_rcm(root, adj, deg)
        if len(perm) != nsolve:
            raise ValueError("numbering graph is not connected")
        inv = np.empty(nsolve, int)
        inv[perm] = np.arange(nsolve)
        bw = max(int(inv[g].max() - inv[g].min()) for g in lo_hi) + 1
        if best is None or bw < best:
            best, best_root = bw, root
    perm = _sparspak_rcm(best_root, adj, deg)
    inv = np.empty(nsolve, int)
    inv[perm] = np.arange(nsolve)
    return inv[bmap]


# ---------------------------------------------------------------------------
# Elemental operators (src/element.cpp:521-565, 1411-1622)
# ---------------------------------------------------------------------------

def helmholtz_matrix(M: Mesh, e: int, lambda2: float, betak2: float):
    """Full np^2 x np^2 elemental Helmholtz matrix, HelmholtzRow semantics.

    H[(i,j),(m,n)] = d_im sum_q Q1[i,q] D[q,j] D[q,n]
                   + d_jn sum_p Q2[p,j] D[p,i] D[p,m]
                   + Q3[i,n] D[n,j] D[i,m] + Q3[m,j] D[j,n] D[m,i]
                   + d_im d_jn Q4[i,j] (lambda2 + betak2)
    """
    n, D = M.np, (M.Dv if lambda2 > EPSDP else M.D)
    Q1, Q2, Q3, Q4 = M.Q1[e], M.Q2[e], M.Q3[e], M.Q4[e]
    I = np.eye(n)
    T1 = np.einsum("im,iq,qj,qn->ijmn", I, Q1, D, D)
    T2 = np.einsum("jn,pj,pi,pm->ijmn", I, Q2, D, D)
    T3 = np.einsum("in,nj,im->ijmn", Q3, D, D) + np.einsum("mj,jn,mi->ijmn", Q3, D, D)
    T4 = np.einsum("im,jn,ij->ijmn", I, I, Q4 * _hcon(M, e, lambda2, betak2))
    return (T1 + T2 + T3 + T4).reshape(n * n, n * n)


def mode_constant(M: Mesh, name: str, mode: int, beta: float):
    """Field::modeConstant (src/field.cpp:1204-1227): beta k, except in
    cylindrical coordinates for the coupled v~ (beta k + 1) and w~ (beta k -
    1) fields, whose uncoupled zeroth mode takes 1."""
    if not M.cyl or name in "cpu":
        return beta * mode
    if name == "v":
        return 1.0 if mode == 0 else beta * mode + 1.0
    if name == "w":
        return 1.0 if mode == 0 else beta * mode - 1.0
    raise ValueError(f"unrecognised field name {name}")


def _hcon(M: Mesh, e, lambda2, betak2):
    """Helmholtz constant at the nodes: lambda2 + betak2, or in cylindrical
    coordinates betak2 / r^2 + lambda2 (zero where r^2 <= EPSDP), as
    Element::HelmholtzRow / HelmholtzKern form it (src/element.cpp:1450,
    1554-1575)."""
    if not M.cyl:
        return lambda2 + betak2
    r2 = (M.y if e is None else M.y[e]) ** 2
    return np.where(r2 > EPSDP, betak2 / np.where(r2 > EPSDP, r2, 1.0) + lambda2, 0.0)


def _dssum_weight(M: Mesh, e):
    """Element::bndryDsSum weights (src/element.cpp:433-463): the mass, or
    in cylindrical coordinates the r-weighted mass, 1 where it vanishes."""
    w = M.Q4[e].ravel()
    return np.where(w > EPSDP, w, 1.0) if M.cyl else w


def helmholtz_op(M: Mesh, u, lambda2, betak2):
    """Batched Element::HelmholtzOp over all elements; u: [nel, np, np]."""
    D = M.Dv if lambda2 > EPSDP else M.D
    R = u @ D.T
    S = D @ u
    R2 = M.Q1 * R + M.Q3 * S
    S2 = M.Q2 * S + M.Q3 * R
    return M.Q4 * u * _hcon(M, None, lambda2, betak2) + D.T @ S2 + R2 @ D


def lagrange_interpolants(z, x):
    """Lagrange interpolants h_j(x) of the points z and their derivatives
    (intmat_g / dermat_g as intp uses them, femlib/operators.c:250-300)."""
    n = len(z)
    h, dh = np.ones(n), np.zeros(n)
    for j in range(n):
        others = [m for m in range(n) if m != j]
        f = np.array([(x - z[m]) / (z[j] - z[m]) for m in others])
        h[j] = np.prod(f)
        dh[j] = sum(np.prod(np.delete(f, i)) / (z[j] - z[m]) for i, m in enumerate(others))
    return h, dh


def element_locate(M: Mesh, e: int, x: float, y: float, r: float = 0.0, s: float = 0.0, guess: bool = True,
                   tol: float = 1e-5, maxit: int = 20):
    """Element::locate (src/element.cpp:1061-1183) in element e: (r, s) of
    (x, y) by Newton's iteration from the nearest element node (guess) or
    from the given (r, s); None when it does not converge inside."""
    n = M.np
    X, Y = M.x[e].ravel(), M.y[e].ravel()
    if guess:
        diag = max(math.hypot(X[-1] - X[0], Y[-1] - Y[0]),
                   math.hypot(X[n * (n - 1)] - X[n - 1], Y[n * (n - 1)] - Y[n - 1]))
        d2 = (x - X) ** 2 + (y - Y) ** 2
        i = int(np.argmin(d2))
        if d2[i] - diag * diag > 0.0:
            return None
        r, s = M.z[i % n], M.z[i // n]
    Xm, Ym = M.x[e], M.y[e]
    it = 0
    while True:
        ir, dr = lagrange_interpolants(M.z, r)
        is_, ds = lagrange_interpolants(M.z, s)
        F0 = x - is_ @ Xm @ ir
        F1 = y - is_ @ Ym @ ir
        J = [dr @ Xm.T @ is_, dr @ Ym.T @ is_, ds @ Xm @ ir, ds @ Ym @ ir]
        det = J[0] * J[3] - J[1] * J[2]
        idet = 1.0 / EPSDP if abs(det) < EPSDP else 1.0 / det
        r += (F0 * J[3] - F1 * J[2]) * idet
        s += (F1 * J[0] - F0 * J[1]) * idet
        if abs(r) > 20.0 and abs(s) > 20.0:
            return None
        it += 1
        if not (it < maxit and (abs(F0) > tol or abs(F1) > tol)):
            break
    if it < maxit and abs(r) < 1.0 + tol and abs(s) < 1.0 + tol:
        return r, s
    return None


def locate(M: Mesh, x: float, y: float, tol: float = 1e-5, maxit: int = 20):
    """HistoryPoint::locate (src/history.cpp:45-63) over Element::locate:
    (element, r, s) of the first element where Newton's iteration from the
    nearest node converges inside, else None."""
    for e in range(M.nel):
        rs = element_locate(M, e, x, y, guess=True, tol=tol, maxit=maxit)
        if rs is not None:
            return e, rs[0], rs[1]
    return None


def relocate(M: Mesh, x: float, y: float, e: int, r: float, s: float, tol: float = 1e-5, maxit: int = 20):
    """FluidParticle::integrate's search (src/particle.cpp:155-175): Newton
    in element e from (r, s), else the full search; None outside."""
    if e is not None and e >= 0:
        rs = element_locate(M, e, x, y, r, s, guess=False, tol=tol, maxit=maxit)
        if rs is not None:
            return e, rs[0], rs[1]
    return locate(M, x, y, tol, maxit)


class FluidParticles:
    """Massless particles (FluidParticle, src/particle.cpp:37-281, and the
    Analyser's handling, src/analysis.cpp:63-104, 206-226, 252-272): made
    where located, moved by an Adams-Bashforth predictor and Adams-Moulton
    corrector (Integration::AdamsBashforth / AdamsMoulton,
    src/integration.cpp:37-96) of order min(steps, N_TIME) on velocities from
    `probe(e, r, s, z) -> (u, v, w)`, relocated from their element (else a
    full search); those that leave stop.  z wraps into one period in 3D."""

    AB = {1: [1.0], 2: [1.5, -0.5], 3: [23 / 12, -16 / 12, 5 / 12]}
    AM = {2: [0.5, 0.5], 3: [5 / 12, 8 / 12, -1 / 12], 4: [9 / 24, 19 / 24, -5 / 24, 1 / 24]}

    def __init__(self, M: Mesh, tok, nfields: int):
        self.M = M
        self.ncom = 3 if nfields > 3 else 2
        self.dt, self.tord = tok["D_T"], tok.ivalue("N_TIME")
        self.lz = 2 * math.pi / tok["BETA"]
        self.tol, self.maxit = tok["TOL_POS"], tok.ivalue("NR_MAX")
        self.parts, self.initial = [], []

    def _wrap(self, z):
        return self.lz - math.fmod(abs(z), self.lz) if z < 0 else math.fmod(z, self.lz)

    def make(self, pid, p, t):
        loc = locate(self.M, p[0], p[1], self.tol, self.maxit)
        if loc is None:
            return False
        z = 0.0 if self.ncom == 2 else self._wrap(p[2])
        self.parts.append(dict(id=pid, ctime=t, x=p[0], y=p[1], z=z, e=loc[0], r=loc[1], s=loc[2], step=0,
                               u=[0.0] * self.tord, v=[0.0] * self.tord, w=[0.0] * self.tord))
        return True

    def _move(self, q, x, y):
        loc = relocate(self.M, x, y, q["e"], q["r"], q["s"], self.tol, self.maxit)
        if loc is None:
            q["e"] = None
            return False
        q["e"], q["r"], q["s"] = loc
        return True

    def integrate(self, probe):
        for q in self.parts:
            if q["e"] is None:
                continue
            q["step"] += 1
            N = min(q["step"], self.tord)
            pred = [self.dt * c for c in self.AB[N]]
            corr = [self.dt * c for c in self.AM[N + 1]]
            q["u"][0], q["v"][0], q["w"][0] = probe(q["e"], q["r"], q["s"], q["z"])
            xp = q["x"] + sum(pred[i] * q["u"][i] for i in range(N))
            yp = q["y"] + sum(pred[i] * q["v"][i] for i in range(N))
            zp = q["z"] + (sum(pred[i] * q["w"][i] for i in range(N)) if self.ncom == 3 else 0.0)
            if not self._move(q, xp, yp):
                continue
            up, vp, wp = probe(q["e"], q["r"], q["s"], zp)
            q["x"] += corr[0] * up + sum(corr[i] * q["u"][i - 1] for i in range(1, N + 1))
            q["y"] += corr[0] * vp + sum(corr[i] * q["v"][i - 1] for i in range(1, N + 1))
            if self.ncom == 3:
                q["z"] += corr[0] * wp + sum(corr[i] * q["w"][i - 1] for i in range(1, N + 1))
            if not self._move(q, q["x"], q["y"]):
                continue
            if self.ncom == 3:
                q["z"] = self._wrap(q["z"])
            for c in "uvw":
                q[c] = [q[c][-1]] + q[c][:-1]


def grad(M: Mesh, u, direction):
    """Element::grad x (0) or y (1) derivative of plane data u [nel,np,np]."""
    ur = u @ M.D.T
    us = M.D @ u
    if direction == 0:
        return ur * M.drdx + us * M.dsdx
    return ur * M.drdy + us * M.dsdy


# ---------------------------------------------------------------------------
# Boundary conditions (src/condition.cpp, src/boundary.cpp, src/field.cpp)
# ---------------------------------------------------------------------------

def axis_kind(kind: str, fld: str, mclass: int) -> str:
    """An axis BC <A> (cylindrical coordinates) as the homogeneous essential
    ('D') or natural ('N') condition of its field and Fourier mode class
    (0, 1, 2 = modes 2 and up), as src/bcmgr.cpp:153-180 tabulates: u, p, c
    natural in mode 0, essential above; v~ essential; w~ essential except
    natural in mode 1.  Other kinds are returned unchanged."""
    if kind != "A":
        return kind
    if fld in "upc":
        return "N" if mclass == 0 else "D"
    if fld == "v":
        return "D"
    if fld == "w":
        return "N" if mclass == 1 else "D"
    raise ValueError(f"axis BC for unknown field {fld}")


class BoundarySystem:
    """Boundary edges (BCtriples) of one field with their kinds."""

    def __init__(self, M: Mesh, N: Numbering, fld: str, mclass: int = 0):
        self.M, self.N, self.fld = M, N, fld
        S = M.S
        self.edges = []      # (e, s, kind, expr)
        for (e, s), g in sorted(M.group.items()):
            if (e, s) in M.mate:
                continue
            bc = S.bcs.get(g, {}).get(fld)
            if bc is None:
                raise ValueError(f"no BC for field {fld} in group {g}")
            kind = axis_kind(bc[0], fld, mclass)
            if kind == "O":      # computed outflow BCs (src/bcmgr.cpp:416-431)
                if "outflow" not in S.groups.get(g, ""):
                    raise ValueError("type 'O' BC must belong to group \"outflow\"")
                kind = {"u": "OU", "v": "OV", "p": "OP"}.get(fld, "N")
            self.edges.append((e, s, kind, "0.0" if bc[0] in "AO" else bc[1]))
        n = M.np
        self.area = []
        for (e, s, _, _) in self.edges:
            idx = M.side_nodes(s)
            xs, ys = M.x[e].ravel()[idx], M.y[e].ravel()[idx]
            # straight side: |dx/dl| along the side times the GLL weight
            L = math.hypot(xs[-1] - xs[0], ys[-1] - ys[0])
            # times r in cylindrical coordinates (src/edge.cpp:75)
            self.area.append(0.5 * L * M.w * (ys if M.cyl else 1.0))
        self.nline = len(self.edges) * n
        # Mixed BCs dc/dn + K (c - C) = 0, "K;C" (Mixed::Mixed, src/condition.cpp:295-312):
        # K C <1, w> in the RHS on every plane (Mixed::sum :315-343) and K <c, w>
        # on the diagonal of the boundary system (augmentSC/Op/Dg :345-435)
        self.mix = {}
        self.mixdiag = None
        nm = n - 1
        for b, (e, s, kind, expr) in enumerate(self.edges):
            if kind != "M":
                continue
            k_s, c_s = re.split(r"[;,]", expr, maxsplit=1)
            K = float(M.S.tokens.evaluate(k_s))
            C = float(M.S.tokens.evaluate(c_s))
            self.mix[b] = (K, C)
            if self.mixdiag is None:
                self.mixdiag = np.zeros(N.nglobal)
            g = [N.btog[e, (s * nm + t) % (4 * nm)] for t in range(n)]
            np.add.at(self.mixdiag, g, K * self.area[b])

    def evaluate_physical(self, tok: Tokens, z: float, t: float):
        """BC line (values along each edge) in physical space at plane z."""
        out = np.zeros((len(self.edges), self.M.np))
        for b, (e, s, kind, expr) in enumerate(self.edges):
            if kind in ("D", "N"):       # ('M' lines are not used; 'H' computed)
                idx = self.M.side_nodes(s)
                xs, ys = self.M.x[e].ravel()[idx], self.M.y[e].ravel()[idx]
                val = tok.evaluate(expr, x=xs, y=ys, z=z, t=t)
                out[b] = np.broadcast_to(np.asarray(val, float), (self.M.np,))
        return out

    def get_essential(self, line, tgt):
        """Field::getEssential -> Essential::set (src/condition.cpp:80-101)."""
        nm = self.M.np - 1
        for b, (e, s, kind, _) in enumerate(self.edges):
            if kind in ("D", "OP"):
                g = [self.N.btog[e, (s * nm + t) % (4 * nm)] for t in range(nm + 1)]
                tgt[g] = line[b]

    def natural_sum(self, line, tgt):
        """Natural::sum (src/condition.cpp:192-219): <h, w> into tgt."""
        nm = self.M.np - 1
        for b, (e, s, kind, _) in enumerate(self.edges):
            if kind in ("N", "H", "OU", "OV"):   # the computed natural BCs sum the same way (src/condition.cpp:470-495, 573-660)
                g = [self.N.btog[e, (s * nm + t) % (4 * nm)] for t in range(nm + 1)]
                np.add.at(tgt, g, line[b] * self.area[b])
            elif kind == "M":
                K, C = self.mix[b]
                g = [self.N.btog[e, (s * nm + t) % (4 * nm)] for t in range(nm + 1)]
                np.add.at(tgt, g, K * C * self.area[b])


# ---------------------------------------------------------------------------
# Modal matrix systems and Field::solve (src/matrix.cpp, src/field.cpp)
# ---------------------------------------------------------------------------

class MatrixSys:
    """Statically condensed, banded-Cholesky Helmholtz system of one mode."""

    def __init__(self, M: Mesh, N: Numbering, lambda2: float, betak2: float,
                 method: str = "DIRECT", mixdiag=None):
        self.M, self.N = M, N
        self.lambda2, self.betak2, self.method = lambda2, betak2, method
        self.mixdiag = mixdiag
        mixed_bc = mixdiag is not None
        n = M.np
        next_ = 4 * (n - 1)
        em = M.emap()
        singular = (lambda2 + betak2) < EPSSP and (N.nglobal == N.nsolve) and not mixed_bc
        self.nsolve = N.nsolve - 1 if singular else N.nsolve
        self.nglobal = N.nglobal
        nel = M.nel
        if method == "DIRECT":
            kd = N.nband - 1
            ns = self.nsolve
            AB = np.zeros((kd + 1, ns))         # LAPACK upper band storage
            self.hbi = np.zeros((nel, next_, (n - 2) ** 2))
            self.hii = np.zeros((nel, (n - 2) ** 2, (n - 2) ** 2))
            for e in range(nel):
                H = helmholtz_matrix(M, e, lambda2, betak2)[np.ix_(em, em)]
                hbb = H[:next_, :next_]
                hbi = H[:next_, next_:]
                hii = H[next_:, next_:]
                if hii.size:
                    hii_inv = np.linalg.inv(hii)
                    hbi_c = hbi @ hii_inv
                    hbb = hbb - hbi_c @ hbi.T
                else:
                    hii_inv, hbi_c = hii, hbi
                self.hbi[e], self.hii[e] = hbi_c, hii_inv
                # band assembly (src/matrix.cpp:218-232): entries (m, n),
                # m <= n < nsolve, of the element's boundary nodes
                g = np.asarray(N.btog[e])
                gm, gn = g[:, None], g[None, :]
                sel = (gm < ns) & (gn < ns) & (gn >= gm)
                np.add.at(AB, ((kd + gm - gn)[sel], np.broadcast_to(gn, sel.shape)[sel]), hbb[sel])
            if mixdiag is not None:
                AB[kd, :ns] += mixdiag[:ns]
            self.factor = sla.cholesky_banded(AB, lower=False) if ns else AB
        else:
            npts = N.nglobal + nel * (n - 2) ** 2
            pc = np.zeros(npts)
            for e in range(nel):
                H = helmholtz_matrix(M, e, lambda2, betak2)
                dg = np.diag(H)[em]
                np.add.at(pc, N.btog[e], dg[:next_])
                pc[N.nglobal + e * (n - 2) ** 2: N.nglobal + (e + 1) * (n - 2) ** 2] = dg[next_:]
            if mixdiag is not None:
                pc[:N.nglobal] += mixdiag
            self.PC = 1.0 / pc
            self.npts = npts


def solve_plane(M: Mesh, N: Numbering, B: BoundarySystem, MS: MatrixSys,
                forcing, unknown, bcline, tol_rel=1e-8, step_max=500):
    """One plane of Field::solve (src/field.cpp:598-809).

    forcing, unknown: [nel, np, np]; returns new unknown (forcing unchanged).
    """
    n, nel = M.np, M.nel
    next_ = 4 * (n - 1)
    em = M.emap()
    lam, bk2 = MS.lambda2, MS.betak2
    nsolve, nglobal = MS.nsolve, MS.nglobal
    # -- constrain: f <- -(M f + H g)              (src/field.cpp:812-852)
    gvec = np.zeros(nglobal)
    B.get_essential(bcline, gvec)
    F = M.Q8 * forcing
    if N.emask.any():
        u = np.zeros_like(F)
        flat = u.reshape(nel, -1)
        flat[:, em[:next_]] = gvec[N.btog]
        HG = helmholtz_op(M, u, lam, bk2)
        F = F + HG * N.emask[:, None, None]
    F = -F
    Fe = F.reshape(nel, -1)[:, em]                    # emap (boundary-major)
    if MS.method == "DIRECT":
        # -- buildRHS with static condensation     (src/field.cpp:943-1009)
        RHS = np.zeros(nglobal)
        Fb = Fe[:, :next_] - np.einsum("eij,ej->ei", MS.hbi, Fe[:, next_:])
        np.add.at(RHS, N.btog, Fb)
        B.natural_sum(bcline, RHS)
        RHS[nsolve:] = 0.0
        if nsolve:
            RHS[:nsolve] = sla.cho_solve_banded((MS.factor, False), RHS[:nsolve])
        # -- global2localSC                         (src/element.cpp:368-407)
        ub = RHS[N.btog]
        ui = np.einsum("eij,ej->ei", MS.hii, Fe[:, next_:]) - np.einsum("eji,ej->ei", MS.hbi, ub)
        out = np.zeros((nel, n * n))
        out[:, em[:next_]] = ub
        out[:, em[next_:]] = ui
    else:
        out = _jacpcg(M, N, B, MS, Fe, unknown, bcline, gvec, tol_rel, step_max)
    # -- impose essential values                    (src/field.cpp:1106-1124)
    gvec = np.zeros(nglobal)
    B.get_essential(bcline, gvec)
    mask = N.bmask.astype(bool)
    bnd = out[:, em[:next_]]
    bnd[mask] = gvec[N.btog][mask]
    out[:, em[:next_]] = bnd
    return out.reshape(nel, n, n)


def _global_op(M, N, MS, xg):
    """Field::HelmholtzOperator (src/field.cpp:855-940) on global vector xg."""
    n, nel = M.np, M.nel
    next_, nint = 4 * (n - 1), (n - 2) ** 2
    em = M.emap()
    P = np.zeros((nel, n * n))
    P[:, em[:next_]] = xg[N.btog]
    P[:, em[next_:]] = xg[N.nglobal:].reshape(nel, nint)
    HP = helmholtz_op(M, P.reshape(nel, n, n), MS.lambda2, MS.betak2).reshape(nel, -1)
    y = np.zeros_like(xg)
    np.add.at(y, N.btog, HP[:, em[:next_]])
    y[N.nglobal:] = HP[:, em[next_:]].ravel()
    if MS.mixdiag is not None:
        y[:N.nglobal] += MS.mixdiag * xg[:N.nglobal]
    return y


def _jacpcg(M, N, B, MS, Fe, unknown, bcline, gvec, tol_rel, step_max):
    """Jacobi-PCG branch of Field::solve (src/field.cpp:711-805)."""
    n, nel = M.np, M.nel
    next_, nint = 4 * (n - 1), (n - 2) ** 2
    em = M.emap()
    nglobal, nsolve = MS.nglobal, MS.nsolve
    npts = MS.npts
    r = np.zeros(npts)
    np.add.at(r, N.btog, Fe[:, :next_])
    r[nglobal:] = Fe[:, next_:].ravel()
    B.natural_sum(bcline, r)
    r[nsolve:nglobal] = 0.0
    epsb2 = (tol_rel * math.sqrt(r @ r)) ** 2
    x = np.zeros(npts)
    x[:nglobal] = gvec
    uf = unknown.reshape(nel, -1)[:, em]
    xb = np.zeros(nglobal)
    xb[N.btog] = uf[:, :next_]                 # local2global (last write wins)
    x[:nglobal] = xb
    x[nglobal:] = uf[:, next_:].ravel()
    x[nsolve:nglobal] = 0.0
    p = _global_op(M, N, MS, x)
    p[nsolve:nglobal] = 0.0
    r[nsolve:nglobal] = 0.0
    r = r - p
    r2 = r @ r
    i = 0
    rho2 = 0.0
    while r2 > epsb2:
        i += 1
        if i >= step_max:
            break
        z = MS.PC * r
        rho1 = r @ z
        p = z.copy() if i == 1 else z + (rho1 / rho2) * p
        q = _global_op(M, N, MS, p)
        q[nsolve:nglobal] = 0.0
        alpha = rho1 / (p @ q)
        x = x + alpha * p
        r = r - alpha * q
        rho2 = rho1
        r2 = r @ r
    out = np.zeros((nel, n * n))
    out[:, em[:next_]] = x[N.btog]
    out[:, em[next_:]] = x[nglobal:].reshape(nel, nint)
    return out


# ---------------------------------------------------------------------------
# z-direction real DFT (femlib/fourier.c:40-165; src/auxfield.cpp:1157-1194)
# ---------------------------------------------------------------------------

def dft_forward(phys):
    """[nz, ...] physical planes -> packed Fourier planes, scaled by 1/nz."""
    nz = phys.shape[0]
    if nz == 1:
        return phys.copy()
    if nz == 2:
        out = phys.copy()
        out[1] = 0.0
        return out
    c = np.fft.rfft(phys, axis=0) / nz
    out = np.empty_like(phys)
    out[0] = c[0].real
    out[1] = c[nz // 2].real
    out[2::2] = c[1:nz // 2].real
    out[3::2] = c[1:nz // 2].imag
    return out


def dft_inverse(four):
    nz = four.shape[0]
    if nz == 1:
        return four.copy()
    if nz == 2:
        out = four.copy()
        out[1] = four[0]
        return out
    c = np.zeros((nz // 2 + 1,) + four.shape[1:], complex)
    c[0] = four[0]
    c[nz // 2] = four[1]
    c[1:nz // 2] = four[2::2] + 1j * four[3::2]
    return np.fft.irfft(c * nz, n=nz, axis=0)


# ---------------------------------------------------------------------------
# Field files (src/misc.cpp:106-180, src/auxfield.cpp:1021-1113)
# ---------------------------------------------------------------------------

def write_field(path, session_name, np_, nz, nel, step, time, dt, kinvis, beta,
                fields: dict):
    hdr = [
        f"{session_name:<25s} Session",
        f"{'Thu Jan 01 00:00:00 1970':<25s} Created",
        f"{f'{np_} {np_} {nz} {nel}':<25s} Nr, Ns, Nz, Elements",
        f"{step:<25d} Step",
        f"{time:<25.6g} Time",
        f"{dt:<25.6g} Time step",
        f"{kinvis:<25.6g} Kinvis",
        f"{beta:<25.6g} Beta",
        f"{''.join(fields.keys()):<25s} Fields written",
        f"{'binary IEEE little-endian':<25s} Format",
    ]
    with open(path, "wb") as f:
        f.write(("\n".join(hdr) + "\n").encode())
        for v in fields.values():
            f.write(np.ascontiguousarray(v, dtype="<f8").tobytes())


def read_field(path):
    with open(path, "rb") as f:
        lines = [f.readline().decode() for _ in range(10)]
        np_, _, nz, nel = (int(v) for v in lines[2].split()[:4])
        names = lines[8].split()[0]
        hdr = {"np": np_, "nz": nz, "nel": nel, "step": int(lines[3].split()[0]),
               "time": float(lines[4].split()[0])}
        out = {}
        for c in names:
            out[c] = np.frombuffer(f.read(8 * np_ * np_ * nz * nel), "<f8").reshape(
                nz, nel, np_, np_).copy()
    return hdr, out


# ---------------------------------------------------------------------------
# Drivers
# ---------------------------------------------------------------------------

class Problem:
    """Mesh + numbering + boundary systems for every field of a session."""

    def __init__(self, S: Session, rcm: bool = True, numbering: dict | None = None):
        """numbering: {field: btog} precomputed maps (see Numbering)."""
        self.S = S
        tok = S.tokens
        self.np = tok.ivalue("N_P")
        self.nz = tok.ivalue("N_Z")
        if self.nz > 1 and self.nz % 2:
            raise ValueError("N_Z must be even")
        self.M = Mesh(S, self.np)
        self.nel = self.M.nel
        self.N, self.B = {}, {}
        for c in S.fields:
            self.N[c] = Numbering(self.M, c, rcm, btog=(numbering or {}).get(c))
            self.B[c] = BoundarySystem(self.M, self.N[c], c)
        # cylindrical 3D with axis BCs: numbering and BCs per Fourier mode
        # class 0, 1, 2+ (BCmgr::getNumberSys, src/bcmgr.cpp:550-583)
        self.axis = self.M.cyl and self.nz > 1 and any(
            bc[0] == "A" for g in S.bcs.values() for bc in g.values())
        self.NB = {}
        for c in S.fields:
            for mc in range(3):
                if self.axis and mc > 0:
                    N = Numbering(self.M, c, rcm, mc)
                    self.NB[(c, mc)] = (N, BoundarySystem(self.M, N, c, mc))
                else:
                    self.NB[(c, mc)] = (self.N[c], self.B[c])
        self.dz = 2 * math.pi / tok["BETA"] / self.nz
        self.solve_seconds = 0.0   # time spent in solve(), for the CPU timings

    def nb(self, c, mode):
        """(Numbering, BoundarySystem) of field c for Fourier mode `mode`."""
        return self.NB[(c, min(mode, 2))]

    def evaluate(self, expr, t=0.0):
        """AuxField = function, physical space (src/auxfield.cpp:198-220)."""
        M = self.M
        out = np.empty((self.nz, self.nel, self.np, self.np))
        for k in range(self.nz):
            val = self.S.tokens.evaluate(expr, x=M.x, y=M.y, z=k * self.dz, t=t)
            out[k] = np.broadcast_to(np.asarray(val, float), M.x.shape)
        return out

    def bc_lines(self, c, t=0.0):
        """Fourier-transformed BC lines [nz, nedge, np] (src/field.cpp:62-160)."""
        B = self.B[c]
        phys = np.stack([B.evaluate_physical(self.S.tokens, k * self.dz, t)
                         for k in range(self.nz)])
        return dft_forward(phys)

    def modal_systems(self, c, lambda2, method="DIRECT", cache=None, modes=None):
        """ModalMatrixSys (src/matrix.cpp:33-105): one MatrixSys per mode
        (None for a mode outside `modes`, when given: a timing sample)."""
        tok = self.S.tokens
        beta = tok["BETA"]
        nmodes = (self.nz + 1) // 2
        # viscous systems: beta^2 k^2 times the SVV factor (src/matrix.cpp:78-83)
        sz = (svv_z(self.nz, nmodes, tok["SVV_EPSZ"], int(tok["SVV_MZ"]), tok["KINVIS"])
              if lambda2 > EPSDP else np.ones(nmodes))
        out = []
        for m in range(nmodes):
            if modes is not None and m not in modes:
                out.append(None)
                continue
            bk2 = mode_constant(self.M, c, m, beta) ** 2 * sz[m]
            key = (c, round(lambda2, 14), round(bk2, 14), method, min(m, 2) if self.axis else 0)
            if cache is not None and key in cache:
                out.append(cache[key])
                continue
            N, B = self.nb(c, m)
            ms = MatrixSys(self.M, N, lambda2, bk2, method, B.mixdiag)
            if cache is not None:
                cache[key] = ms
            out.append(ms)
        return out

    def solve(self, c, forcing, unknown, systems, bclines, tol_rel=1e-8, step_max=500):
        """Field::solve over all planes; forcing in Fourier space."""
        out = unknown.copy()
        t0 = time.perf_counter()
        for k in range(self.nz):
            if k == 1 or systems[k >> 1] is None:
                continue
            N, B = self.nb(c, k >> 1)
            out[k] = solve_plane(self.M, N, B, systems[k >> 1],
                                 forcing[k], unknown[k], bclines[k], tol_rel, step_max)
        self.solve_seconds += time.perf_counter() - t0
        return out


def elliptic(path: str, overrides: dict | None = None, forcing_phys=None):
    """elliptic driver (elliptic/drive.cpp:61-96, elliptic/helmholtz.cpp:29-52).

    Returns (problem, solution in physical space [nz, nel, np, np]).
    forcing_phys overrides the USER 'forcing' string (the `.frc` path).
    """
    S = read_session(path, overrides)
    P = Problem(S)
    c = S.fields[0]
    tok = S.tokens
    if forcing_phys is None:
        fstr = None
        for ln in S.user:
            parts = ln.split(None, 1)
            if parts and parts[0].upper() == "FORCING":
                fstr = parts[1].split()[0]
        forcing_phys = P.evaluate(fstr) if fstr else np.zeros((P.nz, P.nel, P.np, P.np))
    F = dft_forward(forcing_phys)
    if P.nz > 1:
        F[1] = 0.0
    systems = P.modal_systems(c, tok["LAMBDA2"], "JACPCG" if tok.ivalue("ITERATIVE") else "DIRECT")
    u0 = np.zeros_like(F)
    U = P.solve(c, F, u0, systems, P.bc_lines(c), tok["TOL_REL"], tok.ivalue("STEP_MAX"))
    if P.nz > 1:
        U[1] = 0.0
    return P, dft_inverse(U)


def exact_field(P: Problem, which: str = "EXACT", t: float = 0.0):
    for ln in P.S.user:
        parts = ln.split(None, 1)
        if parts and parts[0].upper() == which:
            return P.evaluate(parts[1].split()[0], t)
    raise KeyError(which)


# ---------------------------------------------------------------------------
# DNS time step (dns/integrate.cpp:66-289, dns/nonlinear.cpp:198-381)
# ---------------------------------------------------------------------------

SS_COEFF = {1: [1.0, -1.0], 2: [1.5, -2.0, 0.5],
            3: [11.0 / 6.0, -3.0, 1.5, -1.0 / 3.0]}      # src/integration.cpp:99-133
EX_COEFF = {1: [1.0], 2: [2.0, -1.0], 3: [3.0, -3.0, 1.0]}  # src/integration.cpp:136-164


def fourier_grad_z(P: Problem, u):
    """AuxField::gradient(2) on Fourier data (src/auxfield.cpp:651-672)."""
    beta = P.S.tokens["BETA"]
    out = np.empty_like(u)
    out[0] = 0.0
    out[1] = 0.0
    for m in range(1, P.nz // 2):
        out[2 * m] = -beta * m * u[2 * m + 1]
        out[2 * m + 1] = beta * m * u[2 * m]
    return out


def plane_grad(P: Problem, u, d):
    if d == 2:
        return fourier_grad_z(P, u)
    return grad(P.M, u, d)


def smooth(P: Problem, c: str, u):
    """Field::smooth (src/field.cpp:282-327), per plane."""
    M, N = P.M, P.N[c]
    next_ = 4 * (P.np - 1)
    em = M.emap()[:next_]
    out = u.copy()
    wq = np.stack([_dssum_weight(M, e) for e in range(P.nel)])[:, em]
    for k in range(u.shape[0]):
        flat = out[k].reshape(P.nel, -1)
        ds = np.zeros(N.nglobal)
        np.add.at(ds, N.btog, wq * flat[:, em])
        ds *= N.imass
        flat[:, em] = ds[N.btog]
    return out


class DNS:
    """Velocity-correction DNS on a Problem (Cartesian, periodic / Dirichlet).

    State is kept in Fourier space as [nz, nel, np, np] arrays per field,
    with the reference's multi-level storage Us/Uf (dns/integrate.cpp:94-136).
    """

    def __init__(self, P: Problem, ic: dict | None = None, t0: float = 0.0,
                 dealias: bool | None = None, advection: int = 1, modes=None):
        if dealias is None:   # the session token (the reference's build-time DEALIAS)
            dealias = float(P.S.tokens.get("DEALIAS", 0)) > 0
        self.dealias = bool(dealias) and P.nz > 2
        self.P = P
        S = P.S
        tok = S.tokens
        self.ncom = len(S.fields) - 1
        self.ndim = 3 if P.nz > 1 else 2
        self.nord = tok.ivalue("N_TIME")
        self.dt = tok["D_T"]
        self.nu = tok["KINVIS"]
        self.vel = S.fields[:self.ncom]
        self.pname = S.fields[self.ncom]
        shape = (P.nz, P.nel, P.np, P.np)
        self.u = {}
        for c in S.fields:
            if ic and c in ic:
                phys = ic[c]
            else:
                phys = np.zeros(shape)
            f = dft_forward(phys)
            if P.nz > 1:
                f[1] = 0.0
            self.u[c] = f
        self.Us = [[np.zeros(shape) for _ in range(self.ncom)] for _ in range(self.nord)]
        self.Uf = [[np.zeros(shape) for _ in range(self.ncom)] for _ in range(self.nord)]
        self.step, self.time = 0, t0
        self.toggle = 1
        self.advection = advection          # dns -S/-C/-N (dns/drive.cpp:86-91)
        self.cache = {}
        lam = SS_COEFF[self.nord][0] / (self.dt * self.nu)
        # preSolve (dns/integrate.cpp:292-325): ITERATIVE selects Jacobi-PCG velocity systems
        vmethod = "JACPCG" if tok.ivalue("ITERATIVE") else "DIRECT"
        # modes: build and solve only these Fourier modes (a CPU timing sample)
        self.modes = modes
        self.vsys = {c: P.modal_systems(c, lam, vmethod, self.cache, modes) for c in self.vel}
        self.psys = P.modal_systems(self.pname, 0.0, "DIRECT", self.cache, modes)
        self._hopbc_setup()
        self._force_setup()

    # -- Body forcing (FieldForce, dns/fieldforce.cpp:31-137, and the
    #    VirtualForce classes :240-822), on the grid of the products.
    def _force_grid(self, expr, t):
        P, M = self.P, self.P.M
        nzl = 3 * P.nz // 2 if self.dealias else P.nz
        dz = 2 * math.pi / P.S.tokens["BETA"] / nzl
        out = np.empty((nzl,) + M.x.shape)
        for k in range(nzl):
            val = P.S.tokens.evaluate(expr, x=M.x, y=M.y, z=k * dz, t=t)
            out[k] = np.broadcast_to(np.asarray(val, float), M.x.shape)
        return out

    def _force_file(self, fname):
        hdr, flds = read_field(fname.strip())
        P = self.P
        shape = (P.nz, P.nel, P.np, P.np)
        return [np.asarray(flds[c], float).reshape(shape) if c in flds else np.zeros(shape)
                for c in "uvw"[:self.ncom]]

    def _force_setup(self):
        S, tok = self.P.S, self.P.S.tokens
        self.force = None
        if S.force is None:
            return
        t0 = tok["t"]
        xyz = "XYZ"

        def val(name):
            v = force_value(S, name)
            return None if v is None else float(tok.evaluate(v))

        F = {"const": [val("CONST_" + xyz[i]) or 0.0 for i in range(self.ncom)]}
        for i in range(self.ncom):
            if abs(val("WHITE_EPS_" + xyz[i]) or 0.0) > EPSDP:
                raise NotImplementedError("white-noise forcing")
        fname = force_value(S, "STEADY_FILE")
        if fname is not None:
            F["steady"] = self._force_file(fname)
        else:
            F["steady"] = [None if force_value(S, "STEADY_" + xyz[i]) is None
                           else self._force_grid(force_value(S, "STEADY_" + xyz[i]), t0)
                           for i in range(self.ncom)]
        alpha = [force_value(S, "MOD_ALPHA_" + xyz[i]) for i in range(self.ncom)]
        F["alpha"] = [a if a is not None else "0" for a in alpha]
        F["moda"] = [None] * self.ncom
        if any(a is not None for a in alpha):
            fname = force_value(S, "MOD_A_FILE")
            if fname is not None:
                F["moda"] = self._force_file(fname)
            else:
                F["moda"] = [None if force_value(S, "MOD_A_" + xyz[i]) is None
                             else self._force_grid(force_value(S, "MOD_A_" + xyz[i]), t0)
                             for i in range(self.ncom)]
        F["st"] = [force_value(S, "SPATIOTEMP_ALPHA_" + xyz[i]) for i in range(self.ncom)]
        F["mask"] = None
        m = force_value(S, "SPONGE_M")
        if m is not None:
            F["mask"] = self._force_grid(m, t0)
            F["mask_expr"] = m
            upd = force_value(S, "SPONGE_UPDATE")
            F["update"] = 0 if upd is None else int(round(float(tok.evaluate(upd))))
            F["uref"] = [self._force_grid(force_value(S, "SPONGE_" + "UVW"[i]) or "0", t0)
                         for i in range(self.ncom)]
        d = force_value(S, "DRAG_M")
        F["drag"] = None if d is None else self._force_grid(d, t0)
        uns = force_value(S, "CORIOLIS_UNSTEADY")
        uns = 0 if uns is None else int(round(float(tok.evaluate(uns))))
        omega, domega, on = ["0"] * 3, ["0"] * 3, False
        for i in range(3):
            if self.ncom == 3 or i == 2:
                v = force_value(S, "CORIOLIS_OMEGA_" + xyz[i])
                if v is not None:
                    omega[i], on = v, True
                v = force_value(S, f"CORIOLIS_DOMEGA_{xyz[i]}_DT")
                if uns and v is not None:
                    domega[i] = v
        F["coriolis"] = (2 if uns else 1) if on else 0
        if F["coriolis"] and self.P.M.cyl:
            raise NotImplementedError("Coriolis forcing in cylindrical coordinates")
        F["omega"], F["domega"] = omega, domega
        F["m2o"] = [-2.0 * float(tok.evaluate(o)) for o in omega]
        F["o"], F["mo"], F["dodt"] = [0.0] * 3, [0.0] * 3, [0.0] * 3
        dl, ch = val("SFD_DELTA"), val("SFD_CHI")
        F["qbar"] = None
        if dl is not None or ch is not None:
            if dl is None or ch is None:
                raise ValueError("SFD_DELTA and SFD_CHI must be paired.")
            F["chi"], F["rate"] = ch, self.dt / dl
            F["qbar"] = [None] * self.ncom
        self.force = F

    def _force_physical(self, i, n, Uphys):
        """FieldForce::addPhysical (dns/fieldforce.cpp:75-107) for component i."""
        F = self.force
        if F is None:
            return n
        P, M, tok = self.P, self.P.M, self.P.S.tokens
        t = self.time
        nzl = n.shape[0]
        dz = 2 * math.pi / tok["BETA"] / nzl
        X, Y = M.x[None], M.y[None]
        Z = (np.arange(nzl) * dz)[:, None, None, None]
        f = np.zeros_like(n)
        if F["mask"] is not None:                        # SpongeForce (:563-578)
            if F["update"] and self.step % F["update"] == 0:
                F["mask"] = self._force_grid(F["mask_expr"], t)
            f = (F["uref"][i] - Uphys[i]) * F["mask"]
        if F["coriolis"]:                                # CoriolisForce (:726-756)
            def cross_x(c, a):                           # (a x X)_c, src/element.cpp:1752-1785
                if c == 0:
                    return a[1] * Z - a[2] * Y
                if c == 1:
                    return a[2] * X - a[0] * Z
                return a[0] * Y - a[1] * X

            def cross(c, a, b):                          # src/auxfield.cpp:325-383
                if self.ncom == 2:
                    return -2.0 * a[2] * b[1] if c == 0 else 2.0 * a[2] * b[0]
                c0, c1 = (1, 2, 0)[c], (2, 0, 1)[c]
                return a[c0] * b[c1] - a[c1] * b[c0]

            if F["coriolis"] == 2:
                if i == 0:
                    for c in ((2,) if self.ncom == 2 else range(3)):
                        F["o"][c] = float(tok.evaluate(F["omega"][c], t=t))
                        F["mo"][c] = -F["o"][c]
                        F["m2o"][c] = -2.0 * F["o"][c]
                        F["dodt"][c] = -float(tok.evaluate(F["domega"][c], t=t))
                f = f + cross_x(i, F["dodt"])
                w = [cross_x(c, F["mo"]) for c in range(self.ncom)]
                f = f + cross(i, F["o"], w)
            f = f + cross(i, F["m2o"], Uphys)
        if F["steady"][i] is not None:                   # SteadyForce (:335-344)
            f = f + F["steady"][i]
        if F["moda"][i] is not None:                     # ModulatedForce (:449-460)
            alpha = float(tok.evaluate(F["alpha"][i], t=t))
            if abs(alpha) > EPSDP:
                f = f + alpha * F["moda"][i]
        if F["st"][i] is not None:                       # SpatioTemporalForce (:499-514)
            f = f + self._force_grid(F["st"][i], t)
        if F["drag"] is not None:                        # DragForce (:614-628)
            mag = np.sqrt(sum(u * u for u in Uphys))
            f = f - mag * F["drag"] * Uphys[i]
        if F["qbar"] is not None:                        # SFDForce (:792-822)
            if F["qbar"][i] is None:
                F["qbar"][i] = Uphys[i].copy()
            q = F["qbar"][i]
            f = f - F["chi"] * Uphys[i] + F["chi"] * q
            F["qbar"][i] = q * (1.0 - F["rate"]) + F["rate"] * Uphys[i]
        if M.cyl and i < 2:                              # radius-premultiplied x, r components (:100)
            f = f * M.y[None]
        return n + f

    def _force_fourier(self, i, N):
        """FieldForce::addFourier (dns/fieldforce.cpp:110-137): ConstForce."""
        if self.force is not None and abs(self.force["const"][i]) > EPSDP:
            add = self.force["const"][i]
            # radius-premultiplied x, r components (dns/fieldforce.cpp:131)
            N[0] += add * self.P.M.y if (self.P.M.cyl and i < 2) else add
        return N

    # -- High-order pressure BCs (BCmgr::buildComputedBCs / maintainFourier /
    #    evaluateCNBCp, src/bcmgr.cpp:937-996, 1036-1296, 1299-1331;
    #    Edge::curlCurl, src/edge.cpp:110-256).
    def _hopbc_setup(self):
        P, M = self.P, self.P.M
        B = P.B[self.pname]
        self.hedges = [b for b, (_, _, kind, _) in enumerate(B.edges) if kind == "H"]
        nedge = len(B.edges)
        self.eidx, self.nx, self.ny = [], np.zeros((nedge, P.np)), np.zeros((nedge, P.np))
        for b, (e, s, _, _) in enumerate(B.edges):
            idx = M.side_nodes(s)
            self.eidx.append((e, idx))
            # Element::sideGeom (src/element.cpp:1625-1747): outward normal
            # from the mapping partials at the side's nodes, normalised
            sgn, (a, c) = {0: (-1, ("dsdx", "dsdy")), 1: (1, ("drdx", "drdy")),
                           2: (1, ("dsdx", "dsdy")), 3: (-1, ("drdx", "drdy"))}[s]
            nx = sgn * getattr(M, a)[e].ravel()[idx]
            ny = sgn * getattr(M, c)[e].ravel()[idx]
            ln = np.hypot(nx, ny)
            self.nx[b], self.ny[b] = nx / ln, ny / ln
        ey = np.stack([M.y[e].ravel()[idx] for (e, idx) in self.eidx]) if self.eidx else np.zeros((0, P.np))
        self._edge_divy = np.where(ey > EPSDP, 1.0 / np.where(ey > EPSDP, ey, 1.0), 0.0)
        shape = (P.nz, nedge, P.np)
        self.un = [np.zeros(shape) for _ in range(self.nord)]
        self.hop = [np.zeros(shape) for _ in range(self.nord)]
        # computed outflow BCs (BCmgr::buildComputedBCs, src/bcmgr.cpp:937-996):
        # edge velocities in physical space, div u and n.grad(u).n per level
        self.oedges = [b for b, (_, _, kind, _) in enumerate(B.edges) if kind == "OP"]
        self.ouvw = [[np.zeros(shape) for _ in range(3)] for _ in range(self.nord)]
        self.odivu = [np.zeros(shape) for _ in range(self.nord)]
        self.ogradu = [np.zeros(shape) for _ in range(self.nord)]
        self.otoggle = False
        self.ofbuf = np.zeros(shape)

    def _edges(self, f):
        """Values of plane data f [nel, np, np] along every boundary edge."""
        return np.stack([f[e].ravel()[idx] for (e, idx) in self.eidx])

    def _maintain_fourier(self, U, N):
        """BCmgr::maintainFourier (src/bcmgr.cpp:1036-1296), the terms the
        high-order pressure BC uses: -d(u.n)/dt, n.N and -nu n.curlcurl u,
        and the gradient terms of the computed outflow BCs."""
        if self.oedges:
            self._outflow_fourier(U)
        if not self.hedges:
            return
        P, M = self.P, self.P.M
        nz = P.nz
        Je = min(self.step - 1, self.nord)
        invdt = 1.0 / self.dt
        self.hop = [np.zeros_like(self.hop[0])] + self.hop[:-1]
        h = self.hop[0]
        un = np.zeros_like(h)
        for k in range(nz):
            if k == 1:
                continue
            un[k] = self._edges(U[0][k]) * self.nx + self._edges(U[1][k]) * self.ny
            if Je:
                a = SS_COEFF[Je]
                w = a[0] * un[k]
                for q in range(Je):
                    w = w + a[q + 1] * self.un[q][k]
                h[k] = -invdt * w
            nN = self._edges(N[0][k]) * self.nx + self._edges(N[1][k]) * self.ny
            if M.cyl:        # N_x, N_y are radius-premultiplied (src/bcmgr.cpp:1141-1143)
                nN = nN * self._edge_divy
            h[k] += nN
        self.un = [un] + self.un[:-1]
        beta = P.S.tokens["BETA"]
        nu = self.nu

        dy = self._edge_divy if M.cyl else 1.0       # Element::sideDivY (src/element.cpp:965-1010)
        dy2 = dy * dy if M.cyl else 1.0

        def curl_terms(Ur, Vr):
            w = grad(M, Vr, 0) - grad(M, Ur, 1)
            x = self._edges(grad(M, w, 1))
            if M.cyl:                                  # + w / r (src/edge.cpp:160-167)
                x = x + self._edges(w) * dy
            return x, -self._edges(grad(M, w, 0))

        xr, yr = curl_terms(U[0][0], U[1][0])
        h[0] += -nu * xr * self.nx
        h[0] += -nu * yr * self.ny
        for m in range(1, nz // 2):
            bk = m * beta
            kr, ki = 2 * m, 2 * m + 1
            xr, yr = curl_terms(U[0][kr], U[1][kr])
            xi, yi = curl_terms(U[0][ki], U[1][ki])
            xi = xi + bk * self._edges(grad(M, U[2][kr], 0)) * dy
            yi = yi + bk * self._edges(grad(M, U[2][kr], 1)) * dy
            xr = xr - bk * self._edges(grad(M, U[2][ki], 0)) * dy
            yr = yr - bk * self._edges(grad(M, U[2][ki], 1)) * dy
            if M.cyl:                                  # src/edge.cpp:203-204, 221-222
                yi = yi + bk * self._edges(U[2][kr]) * dy2
                yr = yr - bk * self._edges(U[2][ki]) * dy2
            xr = xr + bk * bk * self._edges(U[0][kr]) * dy2
            xi = xi + bk * bk * self._edges(U[0][ki]) * dy2
            yr = yr + bk * bk * self._edges(U[1][kr]) * dy2
            yi = yi + bk * bk * self._edges(U[1][ki]) * dy2
            h[kr] += -nu * xr * self.nx
            h[ki] += -nu * xi * self.nx
            h[kr] += -nu * yr * self.ny
            h[ki] += -nu * yi * self.ny

    # -- Computed outflow BCs (Dong, Karniadakis & Chryssostomidis 2014;
    #    BCmgr::maintainFourier :1203-1293, evaluateCEBCp :1361-1465,
    #    evaluateCNBCu :1516-1633)
    def _outflow_fourier(self, U):
        """nu div u and nu n.grad(u).n along every edge, newest level first."""
        P, M = self.P, self.P.M
        nu, beta = self.nu, P.S.tokens["BETA"]
        self.odivu = [np.zeros_like(self.odivu[0])] + self.odivu[:-1]
        self.ogradu = [np.zeros_like(self.ogradu[0])] + self.ogradu[:-1]
        dv, gr = self.odivu[0], self.ogradu[0]
        dy = self._edge_divy

        def side_grad(f):
            return self._edges(grad(M, f, 0)), self._edges(grad(M, f, 1))

        # The reference's loop over the higher modes (src/bcmgr.cpp:1231-1238)
        # never sets UxIm: its imaginary planes take du/dx from the plane the
        # curl curl loop before it left there, the highest mode's imaginary
        # plane; restated as computed.
        last_im = 2 * (P.nz // 2 - 1) + 1

        def planes(k, kz, sgn):
            xr, yr = side_grad(U[0][last_im if k > 1 and k % 2 else k])
            dv[k] += xr
            gr[k] += (xr * self.nx + yr * self.ny) * self.nx
            xr, yr = side_grad(U[1][k])
            dv[k] += yr
            gr[k] += (xr * self.nx + yr * self.ny) * self.ny
            if M.cyl:
                dv[k] += self._edges(U[1][k]) * dy
            if kz is not None:
                wz = self._edges(U[2][kz])
                dv[k] += sgn * (wz * dy if M.cyl else wz)

        planes(0, None, 0.0)
        for m in range(1, P.nz // 2):
            bk = m * beta
            planes(2 * m, 2 * m + 1, -bk)
            planes(2 * m + 1, 2 * m, bk)
        dv *= nu
        gr *= nu

    def _outflow_p_lines(self, lines):
        """Essential outflow pressure: extrapolated nu n.grad(u).n minus the
        transform of KE* S0, KE* = |u*|^2 / 2 and S0 = (1 - tanh(u*.n /
        U0Delta)) / 2 from the extrapolated edge velocities."""
        if not self.oedges:
            return lines
        P, tok = self.P, self.P.S.tokens
        Je = min(self.step, self.nord)
        b = EX_COEFF[Je]
        if self.otoggle:
            u, v, w = (sum(b[q] * self.ouvw[q][c] for q in range(Je)) for c in range(3))
            unp = self.nx * u + self.ny * v
            ke = 0.5 * (w * w + (v * v + u * u))
            with np.errstate(divide="ignore"):
                iuzd = 1.0 / float(tok.get("U0Delta", 0.0))
            s0 = 0.5 * (1.0 - np.tanh(unp * iuzd))
            fb = ke * s0
            if P.nz > 2:
                fb = dft_forward(fb)
            elif P.nz == 2:
                fb = fb.copy()
                fb[1] = 0.0
            self.ofbuf = fb
            self.otoggle = False
        for k in range(P.nz):
            for e in self.oedges:
                if P.nz > 1 and k == 1:
                    lines[k, e] = 0.0
                    continue
                lines[k, e] = sum(b[q] * self.ogradu[q][k, e] for q in range(Je)) - self.ofbuf[k, e]
        return lines

    def _outflow_u_lines(self, c, lines):
        """Natural outflow velocity (u or v): (p - extrapolated nu div u +
        KE* S0 / nu) times n_x or n_y, p the new pressure."""
        if not self.oedges or c not in self.vel[:2]:
            return lines
        P = self.P
        Je = min(self.step, self.nord)
        b = EX_COEFF[Je]
        pc = self.pname
        nrm = self.nx if c == self.vel[0] else self.ny
        for k in range(P.nz):
            if P.nz > 1 and k == 1:
                lines[k, self.oedges] = 0.0
                continue
            pe = self._edges(self.u[pc][k])
            for e in self.oedges:
                work = sum(b[q] * self.odivu[q][k, e] for q in range(Je))
                lines[k, e] = ((1.0 / self.nu) * self.ofbuf[k, e] + (pe[e] - work)) * nrm[e]
        return lines

    def _hopbc_lines(self, lines):
        """BCmgr::evaluateCNBCp (src/bcmgr.cpp:1299-1331): extrapolated
        dp/dn on the high-order pressure edges of the Fourier BC lines."""
        if not self.hedges:
            return lines
        Je = min(self.step, self.nord)
        b = EX_COEFF[Je]
        for k in range(self.P.nz):
            for e in self.hedges:
                v = np.zeros(self.P.np)
                if k != 1:
                    for q in range(Je):
                        v = v + b[q] * self.hop[q][k, e]
                lines[k, e] = v
        return lines

    # -- 3/2-rule transforms (AuxField::transform32, src/auxfield.cpp:1197-1258,
    #    as compiled with DEALIAS): the nz Fourier planes zero-padded to
    #    3 nz / 2 planes before the inverse transform; the first nz planes of
    #    the 3 nz / 2 forward transform kept.
    def _inverse32(self, F):
        nz = self.P.nz
        if not self.dealias:
            return dft_inverse(F)
        pad = np.zeros((3 * nz // 2,) + F.shape[1:])
        pad[:nz] = F
        return dft_inverse(pad)

    def _forward32(self, phys):
        if not self.dealias:
            return dft_forward(phys)
        return dft_forward(phys)[:self.P.nz]

    def nonlinear(self):
        """Cartesian nonlinear terms (dns/nonlinear.cpp): advection 0 skew-symmetric
        (:38-190), 1 alternating skew (:198-381), 2 convective (:384-480), 3 Stokes.
        With dealias, every product is formed on the 3/2-padded z grid."""
        P = self.P
        U = [self.u[c].copy() for c in self.vel]
        Uphys = [self._inverse32(self.u[c]) for c in self.vel]
        if self.oedges:                  # BCmgr::maintainPhysical (src/bcmgr.cpp:998-1034)
            if self.dealias:
                raise NotImplementedError("outflow BCs with DEALIAS")
            lv = [np.stack([self._edges(Uphys[i][k]) for k in range(P.nz)]) for i in range(self.ncom)]
            if self.ncom < 3:
                lv.append(np.zeros_like(lv[0]))
            self.ouvw = [lv] + self.ouvw[:-1]
            self.otoggle = True
        if self.advection == 1:
            forms = ("conv",) if self.toggle else ("cons",)
        elif self.advection == 0:
            forms = ("conv", "cons")
        elif self.advection == 2:
            forms = ("conv",)
        else:
            forms = ()
        N = []
        if P.M.cyl:
            return self._nonlinear_cyl(U, Uphys, forms)
        for i in range(self.ncom):
            n = np.zeros_like(Uphys[0])
            for j in range(self.ndim):
                if "conv" in forms:
                    if j == 2:
                        tmp = self._inverse32(fourier_grad_z(P, U[i]))
                    else:
                        tmp = grad(P.M, Uphys[i], j)
                    n -= Uphys[j] * tmp
                if "cons" in forms:
                    tmp = Uphys[i] * Uphys[j]
                    if j == 2:
                        tmp = self._inverse32(fourier_grad_z(P, self._forward32(tmp)))
                    else:
                        tmp = grad(P.M, tmp, j)
                    n -= tmp
            if len(forms) == 2:
                n *= 0.5
            n = self._force_physical(i, n, Uphys)
            n = self._forward32(n)
            n = self._force_fourier(i, n)
            N.append(smooth(P, self.vel[0], n))
        if self.advection == 1:
            self.toggle = 1 - self.toggle
        return U, N

    def _nonlinear_cyl(self, U, Uphys, forms):
        """Cylindrical nonlinear terms (dns/nonlinear.cpp:97-160, 258-334,
        398-440): radius-premultiplied x and r components, frame terms of
        the azimuthal velocity, z the azimuthal Fourier direction."""
        P = self.P
        y = P.M.y[None]
        nz3 = P.nz > 2
        divy = np.where(y > EPSDP, 1.0 / np.where(y > EPSDP, y, 1.0), 0.0)
        N = []
        for i in range(self.ncom):
            n = np.zeros_like(Uphys[0])
            if forms == ("conv", "cons"):                 # skewSymmetric (:97-160)
                if i == 0:
                    n -= Uphys[0] * Uphys[1]
                if i == 1:
                    n -= Uphys[1] * Uphys[1]
                if self.ncom == 3:
                    if i == 1:
                        n += 2.0 * (Uphys[2] * Uphys[2])
                    if i == 2:
                        n += -3.0 * (Uphys[2] * Uphys[1])
                    if nz3:
                        n -= Uphys[2] * self._inverse32(fourier_grad_z(P, U[i]))
                        n -= self._inverse32(fourier_grad_z(P, self._forward32(Uphys[i] * Uphys[2])))
            elif forms == ("conv",):                       # u.grad(u) (:264-292, 398-430)
                if self.ncom == 3:
                    if i == 1:
                        n = Uphys[2] * Uphys[2]
                    if i == 2:
                        n = -(Uphys[2] * Uphys[1])
                    if nz3:
                        n -= Uphys[2] * self._inverse32(fourier_grad_z(P, U[i]))
            elif forms == ("cons",):                       # div(uu) (:298-334)
                if i == 0:
                    n -= Uphys[0] * Uphys[1]
                if i == 1:
                    n -= Uphys[1] * Uphys[1]
                if self.ncom == 3:
                    if i == 1:
                        n += Uphys[2] * Uphys[2]
                    if i == 2:
                        n += -2.0 * (Uphys[2] * Uphys[1])
                    if nz3:
                        n -= self._inverse32(fourier_grad_z(P, self._forward32(Uphys[i] * Uphys[2])))
            if forms and i == 2:
                n = n * divy
            if "conv" in forms:
                for j in range(2):
                    tmp = grad(P.M, Uphys[i], j)
                    if i < 2:
                        tmp = tmp * y
                    n -= Uphys[j] * tmp
            if "cons" in forms:
                for j in range(2):
                    tmp = grad(P.M, Uphys[j] * Uphys[i], j)
                    if i < 2:
                        tmp = tmp * y
                    n -= tmp
            if len(forms) == 2:
                n *= 0.5
            n = self._force_physical(i, n, Uphys)
            n = self._forward32(n)
            n = self._force_fourier(i, n)
            N.append(smooth(P, self.vel[0], n))
        if self.advection == 1:
            self.toggle = 1 - self.toggle
        return U, N

    def _couple(self, v, w, sign):
        """AuxField::couple (src/auxfield.cpp:1376-1451) on modes k >= 1:
        forward v~ = v + i w, w~ = v - i w; inverse back."""
        v, w = v.copy(), w.copy()
        for m in range(1, (self.P.nz + 1) // 2):
            kr, ki = 2 * m, 2 * m + 1
            Vr, Vi, Wr, Wi = v[kr].copy(), v[ki].copy(), w[kr].copy(), w[ki].copy()
            if sign > 0:
                v[kr], v[ki] = Vr - Wi, Vi + Wr
                w[kr], w[ki] = Vr + Wi, Vi - Wr
            else:
                v[kr], v[ki] = 0.5 * (Vr + Wr), 0.5 * (Vi + Wi)
                w[kr], w[ki] = 0.5 * (Vi - Wi), 0.5 * (Wr - Vr)
        return v, w

    def advance(self, nsteps: int = 1):
        P = self.P
        tok = P.S.tokens
        for _ in range(nsteps):
            U, N = self.nonlinear()
            self.Us[0] = U
            self.Uf[0] = N
            self.step += 1
            self.time += self.dt
            self._maintain_fourier(U, N)
            cyl = P.M.cyl
            if cyl:                                   # dns/integrate.cpp:160
                y = P.M.y[None]
                U[0], U[1] = U[0] * y, U[1] * y
                self.Us[0] = U
            # -- waveProp (dns/integrate.cpp:204-239)
            Je = min(self.step, self.nord)
            alpha = SS_COEFF[Je]
            beta = [b * self.dt for b in EX_COEFF[Je]]
            uhat = []
            for i in range(self.ncom):
                h = np.zeros_like(U[0])
                for q in range(Je):
                    h += -alpha[q + 1] * self.Us[q][i]
                    h += beta[q] * self.Uf[q][i]
                uhat.append(h)
            self.Uf = [self.Uf[-1]] + self.Uf[:-1]          # rollm(Uf)
            # -- setPForce (dns/integrate.cpp:242-257)
            div = np.zeros_like(U[0])
            for i in range(self.ndim):
                div += plane_grad(P, uhat[i], i)
            div /= self.dt
            pc = self.pname
            self.u[pc] = P.solve(pc, div, self.u[pc], self.psys,
                                 self._outflow_p_lines(self._hopbc_lines(P.bc_lines(pc, self.time))),
                                 tok["TOL_REL"])
            # -- project (dns/integrate.cpp:260-289)
            a = -1.0 / (self.dt * self.nu)
            b = 1.0 / self.nu
            forc = []
            for i in range(self.ncom):
                f = a * (uhat[i] * y if cyl and i == 2 else uhat[i])
                if i < self.ndim:
                    g = plane_grad(P, self.u[pc], i)
                    f = f + b * (g * y if cyl and i < 2 else g)
                forc.append(f)
            # the velocity level stored is the step's old velocity as the
            # nonlinear step copied it (radius-weighted in cylindrical
            # coordinates: D->u holds it after waveProp's swap)
            self.Us[0] = U
            self.Us = [self.Us[-1]] + self.Us[:-1]          # rollm(Us)
            # -- viscous substep (dns/integrate.cpp:177-193, 328-356); in
            #    cylindrical 3D v and w are solved coupled as v~, w~
            c3d = cyl and self.ncom == 3
            lines = {c: self._outflow_u_lines(c, P.bc_lines(c, self.time)) for c in self.vel}
            if c3d:
                forc[1], forc[2] = self._couple(forc[1], forc[2], 1)
                self.u[self.vel[1]], self.u[self.vel[2]] = self._couple(self.u[self.vel[1]],
                                                                        self.u[self.vel[2]], 1)
                lines[self.vel[1]], lines[self.vel[2]] = self._couple(lines[self.vel[1]], lines[self.vel[2]], 1)
            for i, c in enumerate(self.vel):
                if self.step < self.nord:
                    lam = SS_COEFF[Je][0] / (self.dt * self.nu)
                    sysi = P.modal_systems(c, lam, "JACPCG", self.cache, self.modes)
                else:
                    sysi = self.vsys[c]
                self.u[c] = P.solve(c, forc[i], self.u[c], sysi,
                                    lines[c], tok["TOL_REL"],
                                    tok.ivalue("STEP_MAX"))
            if c3d:
                self.u[self.vel[1]], self.u[self.vel[2]] = self._couple(self.u[self.vel[1]],
                                                                        self.u[self.vel[2]], -1)

    # -- Statistics (src/statistics.cpp:94-405), AVERAGE 1 or 2
    def stats_init(self, level):
        names = list(self.P.S.fields)
        if level > 1:
            names += [chr(ord("A") + i) for i in range(self.ncom * (self.ncom + 1) // 2)]
        if level > 2:      # energy-equation correlations (src/statistics.cpp:128-175)
            names += list("qdmnortsabcGHIJKL" if self.ncom == 3 else "qdmnrsabGHI")
        shape = (self.P.nz, self.P.nel, self.P.np, self.P.np)
        self.avg = {c: np.zeros(shape) for c in sorted(names)}
        self.avg_level, self.navg = level, 0

    def stats_update(self):
        """Statistics::update: weight, add the raw fields (Fourier) and the
        velocity products (physical), smooth with the first field's
        numbering, normalise."""
        n = self.navg
        for c in self.avg:
            self.avg[c] = self.avg[c] * n
        for c in self.P.S.fields:
            self.avg[c] = self.avg[c] + self.u[c]
        if self.avg_level > 1:
            ph = [dft_inverse(self.u[c]) for c in self.vel]
            pairs = [(0, 0), (0, 1), (1, 1), (0, 2), (1, 2), (2, 2)]
            for k in range(self.ncom * (self.ncom + 1) // 2):
                i, j = pairs[k]
                c = chr(ord("A") + k)
                self.avg[c] = self.avg[c] + ph[i] * ph[j]
        if self.avg_level > 2:
            self._stats_energy(ph)
        for c in self.avg:
            self.avg[c] = smooth(self.P, self.vel[0], self.avg[c]) / (n + 1)
        self.navg += 1

    def _stats_energy(self, ph):
        """AVERAGE 3 (Statistics::update, src/statistics.cpp:247-391,
        Cartesian): p u_i, q = |u|^2 / 2, q u_i, the rate-of-strain tensor
        from gradients of the Fourier fields (then to physical space), S_ij
        u_j and S_ij S_ij."""
        P, nv, A = self.P, self.ncom, self.avg
        pp = dft_inverse(self.u[self.pname])
        for i, c in enumerate("mno"[:nv]):
            A[c] = A[c] + pp * ph[i]
        q = 0.5 * sum(ph[i] * ph[i] for i in range(nv))
        A["q"] = A["q"] + q
        for i, c in enumerate("rst"[:nv]):
            A[c] = A[c] + ph[i] * q
        off = {}
        for i in range(nv):
            for j in range(nv):
                if j == i:
                    continue
                gij = plane_grad(P, self.u[self.vel[i]], j)
                off[i + j - 1] = gij if j > i else off[i + j - 1] + gij
        So = [dft_inverse(0.5 * off[k]) for k in range(nv * (nv - 1) // 2)]
        Sd = [dft_inverse(plane_grad(P, self.u[self.vel[i]], i)) for i in range(nv)]
        A["G"], A["H"], A["I"] = A["G"] + Sd[0], A["H"] + So[0], A["I"] + Sd[1]
        A["a"] = A["a"] + Sd[0] * ph[0] + So[0] * ph[1]
        A["b"] = A["b"] + So[0] * ph[0] + Sd[1] * ph[1]
        A["d"] = A["d"] + Sd[0] ** 2 + 2 * So[0] ** 2 + Sd[1] ** 2
        if nv == 3:
            A["J"], A["K"], A["L"] = A["J"] + So[1], A["K"] + So[2], A["L"] + Sd[2]
            A["a"] = A["a"] + So[1] * ph[2]
            A["b"] = A["b"] + So[2] * ph[2]
            A["c"] = A["c"] + So[1] * ph[0] + So[2] * ph[1] + Sd[2] * ph[2]
            A["d"] = A["d"] + 2 * So[1] ** 2 + 2 * So[2] ** 2 + Sd[2] ** 2

    def stats_physical(self):
        out = {}
        for c, v in self.avg.items():
            if c in self.P.S.fields:
                f = v.copy()
                if self.P.nz > 1:
                    f[1] = 0.0
                out[c] = dft_inverse(f)
            else:
                out[c] = v.copy()
        return out

    # -- Analyser (src/analysis.cpp:329-443)
    def _mode_l2(self, F, m):
        """AuxField::mode_L2 (src/auxfield.cpp:919-947): sum over elements of
        Q4-weighted Re^2 + Im^2 of mode m, over twice the area."""
        Q4 = self.P.M.Q4
        re = F[2 * m] if self.P.nz > 1 else F[0]
        ek = (Q4 * re * re).sum()
        if self.P.nz > 1:
            ek += (Q4 * F[2 * m + 1] ** 2).sum()
        return ek / (2.0 * Q4.sum())

    def modal_energy(self):
        nm = (self.P.nz + 1) // 2
        return np.array([sum(self._mode_l2(self.u[c], m) for c in self.vel[:self.ndim]) for m in range(nm)])

    def divergence_energy(self):
        P = self.P
        div = sum(plane_grad(P, self.u[c], i) for i, c in enumerate(self.vel[:self.ndim]))
        L2 = sum(self._mode_l2(div, m) for m in range((P.nz + 1) // 2))
        return L2 / (2 * math.pi / P.S.tokens["BETA"])

    def cfl(self):
        """Analyser::estimateCFL's inverse time scale (Element::CFL,
        src/element.cpp:1207-1250; AuxField::CFL, src/auxfield.cpp:1719-1762)."""
        M, P = self.P.M, self.P
        d = M.z[1] - M.z[0]
        out = 0.0
        for i, (a, b) in enumerate((("drdx", "dsdx"), ("drdy", "dsdy"))):
            u = self.u[self.vel[i]][0]
            w = d * np.abs(getattr(M, a)) + d * np.abs(getattr(M, b))
            out = max(out, np.abs(u / w).max())
        if self.ncom == 3:
            out = max(out, np.abs(self.u[self.vel[2]][0]).max() / (2 * math.pi / P.S.tokens["BETA"] / P.nz))
        return out

    def probe(self, points):
        """History-point values (HistoryPoint::extract, src/history.cpp:66-78;
        AuxField::probe, src/auxfield.cpp:1621-1700): [n, nfields] in FIELDS
        order at physical (x, y, z), the Fourier series of the held half
        spectrum summed at z (non-zero modes doubled)."""
        P, M = self.P, self.P.M
        tok = P.S.tokens
        out = np.zeros((len(points), len(P.S.fields)))
        for i, (x, y, z) in enumerate(points):
            loc = locate(M, x, y, tok["TOL_POS"], tok.ivalue("NR_MAX"))
            if loc is None:
                raise ValueError("history point not in mesh")
            e, r, s = loc
            ir, _ = lagrange_interpolants(M.z, r)
            is_, _ = lagrange_interpolants(M.z, s)
            for f, c in enumerate(P.S.fields):
                vals = np.array([is_ @ self.u[c][k, e] @ ir for k in range(P.nz)])
                if P.nz < 3:
                    out[i, f] = vals[0]
                    continue
                bz = z * tok["BETA"]
                nzh = P.nz // 2
                v = vals[0] + vals[1] * math.cos(nzh * bz)
                for k in range(1, nzh):
                    v += 2.0 * vals[2 * k] * math.cos(k * bz) - 2.0 * vals[2 * k + 1] * math.sin(k * bz)
                out[i, f] = v
        return out

    def wall_forces(self):
        """DNSAnalyser::analyse's forces (dns/dnsanalysis.cpp:97-113):
        Field::normTraction / tangTraction (src/field.cpp:392-458) over the
        edges of the group named "wall" (Edge::normTraction / tangTraction /
        scalarFlux, src/edge.cpp:259-378), on the mean (plane 0) data.
        Returns (pressure[3], viscous[3])."""
        P, M = self.P, self.P.M
        S, tok = P.S, P.S.tokens
        names = S.fields
        B = P.B[names[0]]
        mu = tok["RHO"] * tok["KINVIS"]
        pf, vf = np.zeros(3), np.zeros(3)
        pres = self.u[names[self.ndim]][0]          # field DIM: p, or w for 2D "uvwp"
        u, v = self.u[names[0]][0], self.u[names[1]][0]
        w = self.u[names[2]][0] if self.ndim == 3 else None
        grads = {id(a): (grad(M, a, 0), grad(M, a, 1)) for a in [u, v] + ([w] if w is not None else [])}
        for b, (e, s, _, _) in enumerate(B.edges):
            if S.groups.get(M.group[(e, s)], "") != "wall":
                continue
            idx = M.side_nodes(s)
            sgn, (a, c) = {0: (-1, ("dsdx", "dsdy")), 1: (1, ("drdx", "drdy")),
                           2: (1, ("dsdx", "dsdy")), 3: (-1, ("drdx", "drdy"))}[s]
            nx = sgn * getattr(M, a)[e].ravel()[idx]
            ny = sgn * getattr(M, c)[e].ravel()[idx]
            ln = np.hypot(nx, ny)
            nx, ny = nx / ln, ny / ln
            area = B.area[b]
            pv = pres[e].ravel()[idx]
            pf[0] += np.sum(nx * pv * area)
            pf[1] += np.sum(ny * pv * area)
            ux, uy = (t[e].ravel()[idx] for t in grads[id(u)])
            vx, vy = (t[e].ravel()[idx] for t in grads[id(v)])
            sx = np.sum((2.0 * ux * nx + uy * ny) * area) + np.sum(vx * ny * area)
            sy = np.sum(uy * nx * area) + np.sum((2.0 * vy * ny + vx * nx) * area)
            vf[0] -= mu * sx
            vf[1] -= mu * sy
            if w is not None:
                wx, wy = (t[e].ravel()[idx] for t in grads[id(w)])
                vf[2] -= mu * np.sum((wx * nx + wy * ny) * area)
        return pf, vf

    def wall_traction(self):
        """Field::traction (src/field.cpp:533-593; Edge::traction,
        src/edge.cpp:381-540) per Fourier mode over the edges of the group
        named "wall" in SURFACES order, then the inverse z transform (plane 0
        copied when N_Z = 2): [3, nz, np * nwall] normal, in-plane and
        out-of-plane tractions in physical space."""
        P, M = self.P, self.P.M
        S, tok = P.S, P.S.tokens
        names = S.fields
        mu = tok["RHO"] * tok["KINVIS"]
        beta = tok["BETA"]
        nz = P.nz
        pres, u, v = self.u[names[self.ncom]], self.u[names[0]], self.u[names[1]]
        w = self.u[names[2]] if self.ncom == 3 else None
        walls = [(e, s) for (e, s, kind, g) in S.surfaces if kind == "B" and S.groups.get(g, "") == "wall"]
        npn = P.np
        out = np.zeros((3, nz, npn * len(walls)))
        for b, (e, s) in enumerate(walls):
            idx = M.side_nodes(s)
            sgn, (a, c) = {0: (-1, ("dsdx", "dsdy")), 1: (1, ("drdx", "drdy")),
                           2: (1, ("dsdx", "dsdy")), 3: (-1, ("drdx", "drdy"))}[s]
            nx = sgn * getattr(M, a)[e].ravel()[idx]
            ny = sgn * getattr(M, c)[e].ravel()[idx]
            ln = np.hypot(nx, ny)
            nx, ny = nx / ln, ny / ln
            sl = slice(b * npn, (b + 1) * npn)

            def gr(f):
                return grad(M, f, 0)[e].ravel()[idx], grad(M, f, 1)[e].ravel()[idx]

            def tang(U, V):
                ux, uy = gr(U)
                vx, vy = gr(V)
                return (-2 * ux * nx * ny - uy * ny * ny + uy * nx * nx) + (2 * vy * nx * ny - vx * ny * ny + vx * nx * nx)

            out[0, 0, sl] = pres[0][e].ravel()[idx]
            out[1, 0, sl] = -mu * tang(u[0], v[0])
            if w is not None:
                wx, wy = gr(w[0])
                out[2, 0, sl] = -mu * (wx * nx + wy * ny)
            for m in range(1, nz // 2 if nz > 2 else 1):
                bk, re, im = m * beta, 2 * m, 2 * m + 1
                side = lambda f: f[e].ravel()[idx]
                out[0, re, sl], out[0, im, sl] = side(pres[re]), side(pres[im])
                out[1, re, sl] = -mu * tang(u[re], v[re])
                out[1, im, sl] = -mu * tang(u[im], v[im])
                wx, wy = gr(w[re])
                out[2, re, sl] = -mu * ((wx - bk * side(u[im])) * nx + (wy - bk * side(v[im])) * ny)
                wx, wy = gr(w[im])
                out[2, im, sl] = -mu * ((wx + bk * side(u[re])) * nx + (wy + bk * side(v[re])) * ny)
        if nz == 2:
            out[:, 1] = out[:, 0]
        elif nz > 2:
            out = np.stack([dft_inverse(out[c]) for c in range(3)])
        return out

    def physical(self):
        out = {}
        for c, v in self.u.items():
            f = v.copy()
            if self.P.nz > 1:
                f[1] = 0.0
            out[c] = dft_inverse(f)
        return out


def user_functions(S: Session):
    """USER-section 'name = expr' lines (as `compare` reads them)."""
    out = {}
    for ln in S.user:
        if "=" in ln:
            name, expr = ln.split("=", 1)
            out[name.strip()] = expr.strip()
    return out


def dns_session(path: str, overrides: dict | None = None, nsteps: int | None = None,
                advection: int = 1):
    """Run `dns` with the USER solution at t=0 as restart (test/testregress)."""
    S = read_session(path, overrides)
    P = Problem(S)
    funcs = user_functions(S)
    ic = {c: P.evaluate(funcs[c], 0.0) for c in S.fields if c in funcs}
    D = DNS(P, ic, advection=advection)
    D.advance(S.tokens.ivalue("N_STEP") if nsteps is None else nsteps)
    return D


def compare_errors(D: DNS, noise: float = 1e-12):
    """`compare -n` ∞-norm errors vs the USER solution (utility/compare.cpp:197-232)."""
    P = D.P
    funcs = user_functions(P.S)
    t = float(f"{D.time:.6g}")
    out = {}
    for c, ph in D.physical().items():
        ex = P.evaluate(funcs[c], t) if c in funcs else np.zeros_like(ph)
        err = np.abs(ex - ph).max()
        out[c] = "noise-level" if err < noise else f"{err:.4e}"
    return out
