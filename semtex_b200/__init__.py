"""semtex_b200: B200-native spectral-element--Fourier Helmholtz solve and DNS step.

Python mirror of the reference's C++ API for the hot path, over the C ABI of
``libsemtex_b200.so`` (include/semtex_b200.h):

* :class:`Context`  -- FEML session + mesh + numbering on one GPU
  (the FEML/Mesh/Element/BCmgr/Domain construction, elliptic/drive.cpp:145-216)
* :class:`ModalMatrixSys` -- per-mode condensed systems (src/matrix.h:55-71)
* :class:`Field`    -- device field data in the reference plane layout with
  ``solve`` (src/field.h:27) and ``transform`` (src/auxfield.h:61)
* :func:`elliptic`  -- the `elliptic` driver (elliptic/drive.cpp:61-96)

Device memory is held in torch tensors (plumbing only); every numerical
operation runs in the library's CUDA kernels.  There is no CPU fallback.
"""

from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import _lib
from ._lib import FORWARD, INVERSE, STX_DIRECT, STX_JACPCG, STX_MIXED, StxError, check, lib
from .fieldfile import read_field, write_field

DIRECT, JACPCG, MIXED = STX_DIRECT, STX_JACPCG, STX_MIXED

__all__ = ["Context", "ModalMatrixSys", "Field", "DNS", "DNSAdjoint", "Batch", "expression", "svv", "numbering", "element_matrix", "solve_multi", "solve_host_batch", "elliptic", "dns", "read_field",
           "write_field", "FORWARD", "INVERSE", "DIRECT", "JACPCG", "MIXED", "StxError"]


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("semtex_b200 needs a CUDA device (no CPU fallback)")
    return torch


class Context:
    """A session on one GPU: mesh, geometry, numbering and BC storage."""

    def __init__(self, session: str, overrides: dict | str | None = None, device: int = 0,
                 stream: int | None = None):
        if isinstance(overrides, dict):
            overrides = ";".join(f"{k}={v}" for k, v in overrides.items())
        self._h = C.c_void_p()
        check(lib().stx_context_create(session.encode(), overrides.encode() if overrides else None,
                                       device, C.c_void_p(stream) if stream else None,
                                       C.byref(self._h)))
        self.session = session
        self.device = device
        np_, nz, nel, ps = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        check(lib().stx_context_geometry(self._h, C.byref(np_), C.byref(nz), C.byref(nel), C.byref(ps)))
        self.np, self.nz, self.nel, self.plane_size = np_.value, nz.value, nel.value, ps.value
        buf = C.create_string_buffer(64)
        check(lib().stx_context_fields(self._h, buf, 64))
        self.fields = buf.value.decode()

    @property
    def handle(self):
        return self._h

    @property
    def stream(self) -> int:
        """cudaStream_t (as an int) all of this context's device work runs on."""
        s = C.c_void_p()
        check(lib().stx_context_stream(self._h, C.byref(s)))
        return s.value or 0

    def torch_stream(self):
        return _torch().cuda.ExternalStream(self.stream, device=f"cuda:{self.device}")

    def close(self):
        if self._h:
            check(lib().stx_context_destroy(self._h))
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def token(self, expr: str) -> float:
        v = C.c_double()
        check(lib().stx_token(self._h, expr.encode(), C.byref(v)))
        return v.value

    def numbering(self, field: str):
        a, b, c = C.c_int(), C.c_int(), C.c_int()
        check(lib().stx_numbering(self._h, field.encode(), C.byref(a), C.byref(b), C.byref(c)))
        return {"nglobal": a.value, "nsolve": b.value, "nband": c.value}

    def families(self) -> int:
        v = C.c_int()
        check(lib().stx_mesh_families(self._h, C.byref(v)))
        return v.value

    def mesh_coords(self):
        n = self.nel * self.np * self.np
        x, y = np.empty(n), np.empty(n)
        check(lib().stx_mesh_coords(self._h, x.ctypes.data, y.ctypes.data))
        s = (self.nel, self.np, self.np)
        return x.reshape(s), y.reshape(s)

    def locate(self, xy) -> tuple[np.ndarray, np.ndarray]:
        """Elements (-1 outside the mesh) and canonical (r, s) of points
        [n, 2] (HistoryPoint::locate / Element::locate)."""
        pts = np.ascontiguousarray(np.asarray(xy, dtype=np.float64).reshape(-1, 2))
        n = pts.shape[0]
        el = np.empty(n, dtype=np.int32)
        rs = np.empty((n, 2))
        check(lib().stx_mesh_locate(self._h, n, pts.ctypes.data, el.ctypes.data, rs.ctypes.data))
        return el, rs

    def evaluate(self, expr: str, t: float = 0.0) -> np.ndarray:
        """AuxField = "function" in physical space, [nz, nel, np, np]."""
        out = np.empty((self.nz, self.nel, self.np, self.np))
        check(lib().stx_field_evaluate(self._h, expr.encode(), t, out.ctypes.data))
        return out

    def bc_evaluate(self, field: str, t: float = 0.0):
        check(lib().stx_field_bc_evaluate(self._h, field.encode(), t))

    def sync(self):
        check(lib().stx_sync(self._h))

    # -- device field storage in the reference layout
    def new_field(self, name: str = "f"):
        return Field(self, name)


class Field:
    """Device data of one field, [nz, plane_size] doubles (AuxField storage)."""

    def __init__(self, ctx: Context, name: str):
        torch = _torch()
        self.ctx, self.name = ctx, name
        self.data = torch.zeros((ctx.nz, ctx.plane_size), dtype=torch.float64,
                                device=f"cuda:{ctx.device}")
        torch.cuda.synchronize(self.data.device)

    def ptr(self):
        return C.c_void_p(self.data.data_ptr())

    def load_physical(self, a: np.ndarray):
        """Set from physical-space [nz, nel, np, np] host data (no transform)."""
        torch = _torch()
        n = self.ctx.nel * self.ctx.np ** 2
        self.data.zero_()
        self.data[:, :n] = torch.from_numpy(np.ascontiguousarray(a).reshape(self.ctx.nz, n)).to(self.data.device)
        torch.cuda.synchronize(self.data.device)   # library work runs on the context stream
        return self

    def to_numpy(self) -> np.ndarray:
        n = self.ctx.nel * self.ctx.np ** 2
        self.ctx.sync()
        return self.data[:, :n].cpu().numpy().reshape(self.ctx.nz, self.ctx.nel, self.ctx.np, self.ctx.np)

    def transform(self, sign: int):
        """AuxField::transform (src/auxfield.cpp:1157)."""
        check(lib().stx_transform(self.ctx.handle, self.ptr(), sign))
        return self

    def zero_nyquist(self):
        if self.ctx.nz > 1:
            self.ctx.sync()
            self.data[1].zero_()
            _torch().cuda.synchronize(self.data.device)
        return self

    def solve(self, forcing: "Field", system: "ModalMatrixSys", tol_rel: float | None = None,
              step_max: int | None = None):
        """Field::solve(f, MMS) (src/field.cpp:598-809); forcing in Fourier space."""
        ctx = self.ctx
        tol = ctx.token("TOL_REL") if tol_rel is None else tol_rel
        smax = int(ctx.token("STEP_MAX")) if step_max is None else step_max
        iters = (C.c_int * ctx.nz)()
        rc = lib().stx_field_solve(system.handle, forcing.ptr(), self.ptr(), tol, smax, iters)
        if rc == _lib.STX_ENOCONV:
            import warnings
            warnings.warn("Field::solve: step limit exceeded")
        else:
            check(rc)
        self.iterations = list(iters)
        return self


class ModalMatrixSys:
    """ModalMatrixSys(lambda2, beta, base, nmodes, ..., method) for one field."""

    def __init__(self, ctx: Context, field: str, lambda2: float, beta: float | None = None,
                 base_mode: int = 0, num_modes: int | None = None, method: int = DIRECT):
        self.ctx = ctx
        beta = ctx.token("BETA") if beta is None else beta
        num_modes = (ctx.nz + 1) // 2 if num_modes is None else num_modes
        self._h = C.c_void_p()
        check(lib().stx_modal_create(ctx.handle, field.encode(), lambda2, beta, base_mode, num_modes,
                                     method, C.byref(self._h)))
        self.field, self.lambda2, self.beta, self.method = field, lambda2, beta, method
        self.num_modes = num_modes

    @property
    def handle(self):
        return self._h

    def status(self) -> int:
        """Device status word (stx_modal_status): 0 when every bounded wait met its copy."""
        v = C.c_int()
        check(lib().stx_modal_status(self._h, C.byref(v)))
        return v.value

    def info(self, mode: int):
        a, b = C.c_int(), C.c_int()
        check(lib().stx_modal_info(self._h, mode, C.byref(a), C.byref(b)))
        return {"nsolve": a.value, "nband": b.value}

    def close(self):
        if self._h and self.ctx._h:
            check(lib().stx_modal_destroy(self._h))
        self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def solve_host(self, forcing_phys: np.ndarray, out: np.ndarray | None = None) -> np.ndarray:
        """Whole elliptic solve from/to host memory (stx_elliptic_solve_host)."""
        ctx = self.ctx
        shape = (ctx.nz, ctx.nel, ctx.np, ctx.np)
        f = np.ascontiguousarray(forcing_phys, dtype=np.float64)
        if f.shape != shape:
            raise ValueError(f"forcing shape {f.shape} != {shape}")
        if out is None:
            out = np.empty(shape)
        check(lib().stx_elliptic_solve_host(self._h, C.c_void_p(f.ctypes.data),
                                            C.c_void_p(out.ctypes.data)))
        return out


def solve_host_batch(system: "ModalMatrixSys", forcings, solutions):
    """Whole elliptic solves of several host forcings, copies overlapped with
    the solves (stx_elliptic_solve_host_batch).  forcings / solutions are
    sequences of [nz, nel, np, np] float64 arrays (pinned host memory, e.g.
    torch tensors from pin_memory(), lets the copies overlap) or raw host
    addresses (int)."""
    n = len(forcings)
    if len(solutions) != n:
        raise ValueError("as many solutions as forcings")

    def addr(a):
        if isinstance(a, int):
            return a
        if hasattr(a, "data_ptr"):
            return a.data_ptr()
        if not (isinstance(a, np.ndarray) and a.dtype == np.float64 and a.flags.c_contiguous):
            raise ValueError("forcings and solutions must be C-contiguous float64 arrays")
        return a.ctypes.data

    fin = (C.c_void_p * n)(*[addr(a) for a in forcings])
    fout = (C.c_void_p * n)(*[addr(a) for a in solutions])
    check(lib().stx_elliptic_solve_host_batch(system.handle, n, fin, fout))
    return solutions


def solve_multi(systems, forcings, unknowns):
    """Field::solve of several fields at once (stx_field_solve_multi): systems
    sharing their matrices read every skeleton matrix tile once for all."""
    n = len(systems)
    sy = (C.c_void_p * n)(*[s.handle.value for s in systems])
    fr = (C.c_void_p * n)(*[f.ptr().value for f in forcings])
    un = (C.c_void_p * n)(*[u.ptr().value for u in unknowns])
    check(lib().stx_field_solve_multi(sy, n, fr, un))


class Batch:
    """Independent DIRECT solves replayed as one CUDA graph (stx_batch_*).

    ``items`` is a list of (ModalMatrixSys, forcing Field, solution Field);
    the fields' device storage is fixed in the graph.  ``launch()`` replays
    every solve with one graph launch on ``stream``."""

    def __init__(self, items, stream: int | None = None):
        n = len(items)
        self.items = list(items)   # keep systems and buffers alive
        sys_ = (C.c_void_p * n)(*[s.handle.value for s, _, _ in items])
        frc = (C.c_void_p * n)(*[f.ptr().value for _, f, _ in items])
        unk = (C.c_void_p * n)(*[u.ptr().value for _, _, u in items])
        self._h = C.c_void_p()
        check(lib().stx_batch_create(sys_, frc, unk, n, C.c_void_p(stream) if stream else None,
                                     C.byref(self._h)))
        a, b, st = C.c_int(), C.c_int(), C.c_void_p()
        check(lib().stx_batch_info(self._h, C.byref(a), C.byref(b), C.byref(st)))
        self.nsystems, self.kernel_nodes, self.stream = a.value, b.value, st.value

    def launch(self):
        check(lib().stx_batch_launch(self._h))

    def close(self):
        if self._h:
            check(lib().stx_batch_destroy(self._h))
        self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def expression(expr: str, x, y, z, t: float = 0.0, assignments: str | None = None, compiled: bool = True):
    """The session-expression evaluator on the host (no device): `expr` at the
    points (x, y, z) and time t.  compiled=True runs the postfix program the
    device runs for forcing fields; False the interpreter.  Returns (values,
    program length)."""
    x, y, z = (np.ascontiguousarray(np.broadcast_to(np.asarray(v, float), np.broadcast(x, y, z).shape)).ravel()
               for v in (x, y, z))
    out = np.empty_like(x)
    nops = C.c_int(0)
    check(lib().stx_expression_eval(expr.encode(), assignments.encode() if assignments else None, int(compiled),
                                     x.size, x.ctypes.data, y.ctypes.data, z.ctypes.data, float(t),
                                     out.ctypes.data, C.byref(nops)))
    return out, nops.value


def svv(np_: int, eps_n: float, m_n: int, nz: int = 1, eps_z: float = 0.0, m_z: int = -1, kinvis: float = 1.0):
    """Spectral vanishing viscosity operators (host): the derivative matrix of
    the viscous systems [np, np] and the factors of beta^2 k^2 of their
    (nz+1)/2 Fourier modes."""
    D = np.empty((np_, np_))
    Z = np.empty((nz + 1) // 2)
    check(lib().stx_svv(int(np_), float(eps_n), int(m_n), int(nz), float(eps_z), int(m_z), float(kinvis),
                        D.ctypes.data, Z.ctypes.data))
    return D, Z


def numbering(session: str, field: str, overrides=None, mode: int = 0):
    """The `enumerate` utility (utility/enumerate.cpp:110-199) on the host, no
    GPU needed: one field's global numbering for Fourier mode `mode` (they
    differ only in cylindrical sessions with axis BCs) as a dict of nglobal,
    nsolve, nband and the per-element boundary-major arrays btog / bmask."""
    if isinstance(overrides, dict):
        overrides = ";".join(f"{k}={v}" for k, v in overrides.items())
    ov = overrides.encode() if overrides else None
    v = [C.c_int() for _ in range(5)]
    check(lib().stx_numbering_host_mode(session.encode(), ov, field.encode(), int(mode),
                                        *[C.byref(x) for x in v], None, None))
    nel, next_, nglobal, nsolve, nband = (x.value for x in v)
    btog = np.zeros((nel, next_), np.int32)
    bmask = np.zeros((nel, next_), np.int32)
    check(lib().stx_numbering_host_mode(session.encode(), ov, field.encode(), int(mode), None, None, None, None,
                                        None, C.c_void_p(btog.ctypes.data), C.c_void_p(bmask.ctypes.data)))
    return {"nglobal": nglobal, "nsolve": nsolve, "nband": nband, "btog": btog, "bmask": bmask}


def element_matrix(session: str, elmt: int, lambda2: float, betak2: float, overrides=None):
    """Elemental Helmholtz matrix (np^2 x np^2, row-major nodes) on the host."""
    if isinstance(overrides, dict):
        overrides = ";".join(f"{k}={v}" for k, v in overrides.items())
    ov = overrides.encode() if overrides else None
    n = C.c_int()
    check(lib().stx_element_matrix_host(session.encode(), ov, int(elmt), float(lambda2), float(betak2),
                                        C.byref(n), None))
    H = np.empty((n.value ** 2, n.value ** 2))
    check(lib().stx_element_matrix_host(session.encode(), ov, int(elmt), float(lambda2), float(betak2), None,
                                        H.ctypes.data))
    return H


def _user_value(session: str, key: str):
    txt = open(session).read()
    import re
    m = re.search(r"<USER>(.*?)</USER>", txt, re.S | re.I)
    if not m:
        return None
    for ln in m.group(1).splitlines():
        parts = ln.split(None, 1)
        if parts and parts[0].upper() == key.upper():
            return parts[1].split()[0]
    return None


def elliptic(session: str, overrides=None, iterative: bool = False, device: int = 0,
             write: bool = False):
    """The `elliptic` driver: solve the session's Helmholtz problem on the GPU.

    Forcing comes from ``session.frc`` if present, else the USER ``forcing``
    string, else zero (elliptic/drive.cpp:258-354).  Returns the physical
    solution [nz, nel, np, np]; with ``write`` also writes ``session.fld``.
    """
    ctx = Context(session, overrides, device)
    c = ctx.fields[0]
    frc = session + ".frc"
    if os.path.exists(frc):
        _, flds = read_field(frc)
        forcing = next(iter(flds.values()))
    else:
        fs = _user_value(session, "forcing")
        forcing = ctx.evaluate(fs) if fs else np.zeros((ctx.nz, ctx.nel, ctx.np, ctx.np))
    sys_ = ModalMatrixSys(ctx, c, ctx.token("LAMBDA2"), method=JACPCG if iterative else DIRECT)
    u = sys_.solve_host(forcing)
    if write:
        write_field(session + ".fld", os.path.basename(session), ctx.np, ctx.nz, ctx.nel, 1, 0.0,
                    ctx.token("D_T"), ctx.token("KINVIS"), ctx.token("BETA"), {c: u})
    sys_.close()
    ctx.close()
    return u


class DNS:
    """integrate() on the device (dns/integrate.cpp:66-200).

    advection: 0 skew-symmetric, 1 alternating skew-symmetric (default),
    2 convective, 3 Stokes -- the dns -S / default / -C / -N forms.
    """

    def __init__(self, ctx: Context, advection: int = 1):
        self.ctx = ctx
        self._h = C.c_void_p()
        check(lib().stx_dns_create(ctx.handle, advection, C.byref(self._h)))

    def close(self):
        if self._h and self.ctx._h:
            check(lib().stx_dns_destroy(self._h))
        self._h = C.c_void_p()

    def checkpoint(self) -> np.ndarray:
        """Full state (fields, multistep history, pressure-BC levels, forcing
        state, averages, step, time) as a host array (stx_dns_checkpoint_save)."""
        n = C.c_ulonglong()
        check(lib().stx_dns_checkpoint_size(self._h, C.byref(n)))
        buf = np.empty(n.value // 8, dtype=np.float64)
        check(lib().stx_dns_checkpoint_save(self._h, C.c_void_p(buf.ctypes.data), n.value))
        return buf

    def restore(self, buf: np.ndarray):
        """Continue from a checkpoint of the same session (stx_dns_checkpoint_load)."""
        buf = np.ascontiguousarray(buf, dtype=np.float64)
        check(lib().stx_dns_checkpoint_load(self._h, C.c_void_p(buf.ctypes.data), buf.nbytes))

    def system_bytes(self, field: str):
        """Algorithmic bytes of one direct solve of `field`'s steady-step
        system, per phase (stx_dns_system + stx_modal_bytes)."""
        h = C.c_void_p()
        check(lib().stx_dns_system(self._h, field.encode(), C.byref(h)))
        b = (C.c_double * 4)()
        check(lib().stx_modal_bytes(h, b))
        return list(b)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def restart(self, fields: dict, t0: float = 0.0):
        """Set physical-space initial fields {name: [nz, nel, np, np]}."""
        check(lib().stx_dns_restart(self._h, t0))
        for c, a in fields.items():
            a = np.ascontiguousarray(a, dtype=np.float64)
            check(lib().stx_dns_set_field(self._h, c.encode(), C.c_void_p(a.ctypes.data)))

    def advance(self, nsteps: int):
        check(lib().stx_dns_advance(self._h, nsteps))

    def field(self, c: str) -> np.ndarray:
        ctx = self.ctx
        out = np.empty((ctx.nz, ctx.nel, ctx.np, ctx.np))
        check(lib().stx_dns_get_field(self._h, c.encode(), C.c_void_p(out.ctypes.data)))
        return out

    def state(self):
        s, t = C.c_int(), C.c_double()
        check(lib().stx_dns_state(self._h, C.byref(s), C.byref(t)))
        return s.value, t.value

    def status(self) -> int:
        """Device status of every system (0: every bounded wait met its copy)."""
        v = C.c_int()
        check(lib().stx_dns_status(self._h, C.byref(v)))
        return v.value

    # -- Statistics (src/statistics.cpp), token AVERAGE 1 or 2
    def stats_update(self):
        check(lib().stx_dns_stats_update(self._h))

    def stats(self):
        """(number of updates, {name: physical average [nz, nel, np, np]})."""
        buf = C.create_string_buffer(64)
        n = C.c_int()
        check(lib().stx_dns_stats_info(self._h, buf, 64, C.byref(n), -1))
        ctx = self.ctx
        out = {}
        for c in buf.value.decode():
            a = np.empty((ctx.nz, ctx.nel, ctx.np, ctx.np))
            check(lib().stx_dns_stats_get(self._h, c.encode(), C.c_void_p(a.ctypes.data)))
            out[c] = a
        return n.value, out

    def graph_info(self):
        """(cycle length of the captured step graph, graph launches so far)."""
        a, b = C.c_int(), C.c_longlong()
        check(lib().stx_dns_graph_info(self._h, C.byref(a), C.byref(b)))
        return a.value, b.value

    # -- Analyser (src/analysis.cpp:329-443) on the device
    def modal_energy(self) -> np.ndarray:
        out = np.zeros((self.ctx.nz + 1) // 2)
        check(lib().stx_dns_modal_energy(self._h, C.c_void_p(out.ctypes.data)))
        return out

    def divergence_energy(self) -> float:
        v = C.c_double()
        check(lib().stx_dns_divergence_energy(self._h, C.byref(v)))
        return v.value

    def cfl(self) -> float:
        """Inverse CFL time scale (Analyser::estimateCFL); CFL number = cfl() * D_T."""
        v = C.c_double()
        check(lib().stx_dns_cfl(self._h, C.byref(v)))
        return v.value

    def probe(self, points) -> np.ndarray:
        """Field values at history points [n, 3] (x, y, z), [n, nfields] in
        FIELDS order (HistoryPoint::extract); points outside the mesh are
        rejected."""
        pts = np.asarray(points, dtype=np.float64).reshape(-1, 3)
        el, rs = self.ctx.locate(pts[:, :2])
        if (el < 0).any():
            raise ValueError(f"history point {pts[int(np.argmin(el))]} not in mesh")
        z = np.ascontiguousarray(pts[:, 2])
        out = np.empty((pts.shape[0], len(self.ctx.fields)))
        check(lib().stx_dns_probe(self._h, pts.shape[0], el.ctypes.data, rs.ctypes.data, z.ctypes.data,
                                  out.ctypes.data))
        return out

    def wall_forces(self) -> tuple[np.ndarray, np.ndarray]:
        """(pressure, viscous) forces [3] on the "wall" group
        (Field::normTraction / tangTraction)."""
        p, v = np.zeros(3), np.zeros(3)
        check(lib().stx_dns_wall_forces(self._h, p.ctypes.data, v.ctypes.data))
        return p, v

    def wall_traction(self) -> np.ndarray:
        """Normal, in-plane and out-of-plane tractions along the "wall"
        group in physical space, [3, nz, N_P x wall edges] (Field::traction,
        the data of session.wss)."""
        n = C.c_int()
        check(lib().stx_dns_wall_traction(self._h, C.byref(n), None))
        out = np.zeros((3, self.ctx.nz, n.value))
        if n.value:
            check(lib().stx_dns_wall_traction(self._h, C.byref(n), out.ctypes.data))
        return out


class DNSAdjoint:
    """Discrete adjoint and tangent-linear model of a DNS's time steps over
    the C ABI (stx_dns_adjoint_*): :meth:`record` runs steps keeping
    full-state checkpoints on the device every ``checkpoint_every`` steps;
    :meth:`backward` maps d(objective)/d(final velocity) to
    d(objective)/d(initial velocity) (segments recomputed from their
    checkpoints, steps transposed last to first); :meth:`tangent` maps an
    initial-velocity direction to the final velocity's derivative along it.
    Velocities are dicts {component: [nz, nel, np, np]} in physical space,
    as :meth:`DNS.restart` and :meth:`DNS.field` use them."""

    def __init__(self, dns: DNS, checkpoint_every: int = 10):
        self.dns = dns
        self._h = C.c_void_p()
        check(lib().stx_dns_adjoint_create(dns._h, checkpoint_every, C.byref(self._h)))
        names = dns.ctx.fields
        self.components = names[:-1]

    def close(self):
        if self._h and self.dns._h:
            check(lib().stx_dns_adjoint_destroy(self._h))
        self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def record(self, nsteps: int):
        check(lib().stx_dns_adjoint_record(self._h, nsteps))

    def info(self):
        """(first step, last step, checkpoint bytes on the device)."""
        a, b, n = C.c_int(), C.c_int(), C.c_ulonglong()
        check(lib().stx_dns_adjoint_info(self._h, C.byref(a), C.byref(b), C.byref(n)))
        return a.value, b.value, n.value

    def _pack(self, fields: dict) -> np.ndarray:
        ctx = self.dns.ctx
        shape = (ctx.nz, ctx.nel, ctx.np, ctx.np)
        return np.ascontiguousarray(np.stack([np.broadcast_to(np.asarray(fields[c], dtype=np.float64), shape)
                                              for c in self.components]))

    def _unpack(self, a: np.ndarray) -> dict:
        return {c: a[i] for i, c in enumerate(self.components)}

    def backward(self, seed: dict) -> dict:
        x = self._pack(seed)
        out = np.empty_like(x)
        check(lib().stx_dns_adjoint_backward(self._h, C.c_void_p(x.ctypes.data), C.c_void_p(out.ctypes.data)))
        return self._unpack(out)

    def tangent(self, direction: dict) -> dict:
        x = self._pack(direction)
        out = np.empty_like(x)
        check(lib().stx_dns_adjoint_tangent(self._h, C.c_void_p(x.ctypes.data), C.c_void_p(out.ctypes.data)))
        return self._unpack(out)


def _user_functions(session: str):
    import re
    txt = open(session).read()
    m = re.search(r"<USER>(.*?)</USER>", txt, re.S | re.I)
    out = {}
    if m:
        for ln in m.group(1).splitlines():
            if "=" in ln:
                k, v = ln.split("=", 1)
                out[k.strip()] = v.strip()
    return out


def dns(session: str, overrides=None, nsteps: int | None = None, advection: int = 1, device: int = 0,
        write: bool = False):
    """The `dns` driver: restart from ``session.rst`` if present, else from the
    USER section at t=0 (as `compare` writes it), integrate N_STEP steps and
    return the physical fields; with ``write`` also write ``session.fld``."""
    ctx = Context(session, overrides, device)
    D = DNS(ctx, advection)
    rst = session + ".rst"
    t0 = 0.0
    if os.path.exists(rst):
        hdr, flds = read_field(rst)
        t0 = hdr["time"]
    else:
        funcs = _user_functions(session)
        flds = {c: ctx.evaluate(funcs[c], 0.0) for c in ctx.fields if c in funcs}
    D.restart(flds, t0)
    D.advance(int(ctx.token("N_STEP")) if nsteps is None else nsteps)
    out = {c: D.field(c) for c in ctx.fields}
    step, t = D.state()
    if write:
        write_field(session + ".fld", os.path.basename(session), ctx.np, ctx.nz, ctx.nel, step, t,
                    ctx.token("D_T"), ctx.token("KINVIS"), ctx.token("BETA"), out)
    D.close()
    ctx.close()
    return out, t
