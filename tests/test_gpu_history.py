"""History points, wall forces, wall tractions and the analyser's files on
the device (stx_mesh_locate, stx_dns_probe, stx_dns_wall_forces,
stx_dns_wall_traction; the `dns` program's session.his, session.mdl,
session.flx and session.wss).

- Probes and forces against the oracle's restatement (HistoryPoint::extract
  over AuxField::probe, src/auxfield.cpp:1621-1700; Field::normTraction /
  tangTraction, src/field.cpp:392-458) evaluated on the DNS's own Fourier
  fields after a few steps: the plane channel in 3D (N_Z = 8) and 2D, and
  the periodic Taylor-Green box (no wall: zero forces).
- Wall tractions (Field::traction, src/field.cpp:533-593) against the
  oracle on the channel with 8, 2 and 1 planes: every mode's normal,
  in-plane and out-of-plane traction, then the inverse z transform.
- Phase averages (N_PHASE, STEPS_P: Statistics::phaseUpdate) in
  session.<phase>.phs and the running averages beside them, against the
  oracle's statistics on the device DNS's fields.
- The `dns` program's particle tracks (session.par in, session.trk out,
  FluidParticle, src/particle.cpp) against the oracle's particle integrator
  moving on the device DNS's own fields, step by step, with new particles
  every SPAWN steps.
- The `dns` program's files against the same values through the Python
  API, line for line in the reference's formats (src/analysis.cpp:275-375,
  dns/dnsanalysis.cpp:44-127).
"""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

import semtex_b200 as S
import semtex_oracle as O
from semtex_b200 import _lib, sessions
from semtex_b200.fieldfile import write_field

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "semtex_b200", "bin")


def _fourier(D, c):
    """The DNS's Fourier-space storage of field c, [nz, nel, np, np]."""
    from cuda.bindings import runtime as rt
    ctx = D.ctx
    ctx.sync()   # the DNS runs on the context's own stream: its step must be done before the copy
    p = C.c_void_p()
    _lib.check(_lib.lib().stx_dns_field_ptr(D._h, c.encode(), C.byref(p)))
    buf = np.empty((ctx.nz, ctx.plane_size))
    err, = rt.cudaMemcpy(buf.ctypes.data, p.value, buf.nbytes, rt.cudaMemcpyKind.cudaMemcpyDeviceToHost)
    assert err == rt.cudaError_t.cudaSuccess
    n = ctx.nel * ctx.np * ctx.np
    return buf[:, :n].reshape(ctx.nz, ctx.nel, ctx.np, ctx.np).copy()


def _oracle_on(D, path):
    """The oracle's DNS holding the device DNS's current Fourier fields."""
    OD = O.DNS(O.Problem(O.read_session(path)))
    for c in D.ctx.fields:
        OD.u[c] = _fourier(D, c)
    return OD


def _channel(tmp_path, name, nz, history=None, extra=None):
    path = sessions.channel_session(str(tmp_path / name), 4, 2, 6, nz, re=200.0, dt=5e-3, ntime=3,
                                    history=history, extra=extra)
    ctx = S.Context(path)
    x, y = ctx.mesh_coords()
    ic = sessions.channel_initial(x, y, np.arange(ctx.nz) * 2 * np.pi / ctx.nz, amplitude=0.05)
    return path, ctx, {c: ic[c] for c in ctx.fields[:-1]}


POINTS = [(0.3, -0.95, 0.0), (1.7, 0.2, 1.1), (3.14159, 0.0, 2.5), (5.9, 0.81, 4.0), (2.2, -0.4, 7.5),
          (4.0, 1.0, 3.3)]


@pytest.mark.parametrize("nz", [8, 1])
def test_channel_probe_and_wall_forces_match_oracle(tmp_path, nz):
    path, ctx, ic = _channel(tmp_path, f"ch{nz}", nz)
    D = S.DNS(ctx, 1)
    D.restart(ic, 0.0)
    D.advance(7)
    got = D.probe(POINTS)
    pf, vf = D.wall_forces()
    OD = _oracle_on(D, path)
    want = OD.probe(POINTS)
    assert got.shape == (len(POINTS), len(ctx.fields))
    assert np.abs(got - want).max() <= 1e-12 * max(1.0, np.abs(want).max())
    opf, ovf = OD.wall_forces()
    scale = max(np.abs(opf).max(), np.abs(ovf).max())
    assert scale > 1e-3
    assert np.abs(pf - opf).max() <= 1e-12 * scale and np.abs(vf - ovf).max() <= 1e-12 * scale
    if nz == 1:
        assert pf[2] == 0.0 and vf[2] == 0.0
    D.close()


@pytest.mark.parametrize("nz", [8, 2, 1])
def test_channel_wall_traction_matches_oracle(tmp_path, nz):
    path, ctx, ic = _channel(tmp_path, f"wt{nz}", nz)
    D = S.DNS(ctx, 1)
    D.restart(ic, 0.0)
    D.advance(6)
    got = D.wall_traction()
    want = _oracle_on(D, path).wall_traction()
    assert got.shape == want.shape == (3, ctx.nz, 2 * 4 * ctx.np)   # 4 wall edges top and bottom
    for c in range(3):
        scale = max(np.abs(want[c]).max(), 1e-300)
        assert np.abs(got[c] - want[c]).max() <= 1e-11 * scale, c
    assert np.abs(got[1]).max() > 1e-4
    if nz == 1:
        assert not got[2].any()
    D.close()


def test_taylor_green_probe_and_no_wall(tmp_path):
    path = sessions.taylor_green_session(str(tmp_path / "tg"), 3, 6, 8, re=100.0, dt=2e-3)
    ctx = S.Context(path)
    x, y = ctx.mesh_coords()
    z = (np.arange(ctx.nz) * 2 * np.pi / ctx.nz)[:, None, None, None]
    ic = {"u": np.sin(x) * np.cos(y) * np.cos(z), "v": -np.cos(x) * np.sin(y) * np.cos(z), "w": 0 * z + 0 * x}
    D = S.DNS(ctx, 1)
    D.restart({c: np.broadcast_to(v, (ctx.nz, ctx.nel, ctx.np, ctx.np)).copy() for c, v in ic.items()}, 0.0)
    D.advance(4)
    pts = [(0.5, 0.5, 0.3), (6.0, 3.0, 5.0), (2 * np.pi, 0.0, 0.0)]
    got = D.probe(pts)
    want = _oracle_on(D, path).probe(pts)
    assert np.abs(got - want).max() <= 1e-12 * max(1.0, np.abs(want).max())
    # the Taylor-Green velocity at t ~ 0 at the first point, z-dependence included
    x0, y0, z0 = pts[0]
    assert abs(got[0, 0] - np.sin(x0) * np.cos(y0) * np.cos(z0)) < 1e-2
    pf, vf = D.wall_forces()
    assert not pf.any() and not vf.any()
    with pytest.raises(ValueError, match="not in mesh"):
        D.probe([(7.0, 1.0, 0.0)])
    D.close()


def test_dns_program_writes_history_modal_and_flux_files(tmp_path):
    hist = [(1, 0.3, -0.95, 0.0), (2, 3.0, 0.5, 1.5), (7, 9.0, 0.0, 0.0)]   # the last is outside
    nstep = 6
    path, ctx, ic = _channel(tmp_path, "chf", 8, history=hist,
                             extra={"N_STEP": nstep, "IO_HIS": 2, "IO_MDL": 3, "IO_FLD": nstep, "IO_WSS": 3})
    write_field(path + ".rst", "chf", ctx.np, ctx.nz, ctx.nel, 0, 0.0, 5e-3, 1.0 / 200.0, 1.0,
                {**ic, "p": np.zeros_like(ic["u"])})
    r = subprocess.run([os.path.join(BIN, "dns"), path], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    assert "History point at (9.000000, 0.000000, 0.000000) not in mesh" in r.stderr
    # the same run through the Python API, formatted as the reference formats
    D = S.DNS(ctx, 1)
    D.restart(ic, 0.0)
    his, mdl, flx, wss = [], [], [], []
    for step in range(1, nstep + 1):
        D.advance(1)
        t = D.state()[1]
        if step % 3 == 0:
            wss.append((step, D.wall_traction()))
        if step % 2 == 0 or step == nstep:
            vals = D.probe([h[1:] for h in hist[:2]])
            for (i, *_), v in zip(hist[:2], vals):
                his.append(f"{i:4d}{t:15.8e}" + "".join(f"{a:14.6e}" for a in v[:-1]) + f"{v[-1]:19.11e}")
            pf, vf = D.wall_forces()
            tf = pf + vf
            flx.append("%6d %#10.6g " % (step, t) + " ".join(
                "%#10.6g %#10.6g %#10.6g" % (pf[k], vf[k], tf[k]) for k in range(3)))
        if step % 3 == 0:
            mdl += [f"{t:10g}{m:5d}{e:15g}" for m, e in enumerate(D.modal_energy())]
    D.close()
    _same_lines(open(path + ".his").read().splitlines(), his)
    _same_lines(open(path + ".mdl").read().splitlines(),
                ["#     Time Mode         Energy", "# ----------------------------"] + mdl)
    _same_lines(open(path + ".flx").read().splitlines(),
                ["# DNS state information file", "# Step Time [Fpre Fvis Ftot]-axis",
                 "# -------------------------------"] + flx)
    assert len(his) == 2 * 3 and len(mdl) == 2 * 4 and len(flx) == 3
    # session.wss: per output step a ten-line header and 3 x N_Z planes of
    # the wall lines
    raw = open(path + ".wss", "rb").read()
    pos = 0
    for step, want in wss:
        hdr = []
        for _ in range(10):
            end = raw.index(b"\n", pos)
            hdr.append(raw[pos:end].decode())
            pos = end + 1
        assert hdr[0].split()[0] == "chf" and hdr[8].split()[0] == "nts"
        assert hdr[2].split()[:4] == [str(ctx.np), "1", str(ctx.nz), "8"]
        assert int(hdr[3].split()[0]) == step and "binary IEEE" in hdr[9]
        got = np.frombuffer(raw[pos:pos + want.nbytes], dtype=np.float64).reshape(want.shape)
        pos += want.nbytes
        for c in range(3):
            assert np.abs(got[c] - want[c]).max() <= 1e-9 * max(np.abs(want[c]).max(), 1e-300)
    assert pos == len(raw)


def _same_lines(got, want):
    """The same tokens, and the same numbers up to the printed precision:
    the two runs differ in round-off (the element condensation sums with
    atomic adds), which may move a last digit."""
    assert len(got) == len(want)
    for g, w in zip(got, want):
        if g.startswith("#"):
            assert g == w
            continue
        tg, tw = g.split(), w.split()
        assert len(tg) == len(tw)
        # values at round-off level (a force on a periodic direction) are
        # compared against the line's scale
        scale = max(abs(float(b)) for b in tw[1:])
        for a, b in zip(tg, tw):
            if "." not in b and "e" not in b:
                assert a == b
            else:
                assert abs(float(a) - float(b)) <= 2e-6 * abs(float(b)) + 1e-12 * scale, (g, w)


def _probe_at(F, M, e, r, s, z, beta):
    """Physical velocity of Fourier fields F [ncom][nz, nel, np, np] at
    (element e, r, s, z) (AuxField::probe)."""
    ir, _ = O.lagrange_interpolants(M.z, r)
    is_, _ = O.lagrange_interpolants(M.z, s)
    out = []
    for f in F:
        vals = np.array([is_ @ f[k, e] @ ir for k in range(f.shape[0])])
        if f.shape[0] < 3:
            out.append(vals[0])
            continue
        nzh, bz = f.shape[0] // 2, z * beta
        v = vals[0] + vals[1] * np.cos(nzh * bz)
        for k in range(1, nzh):
            v += 2 * vals[2 * k] * np.cos(k * bz) - 2 * vals[2 * k + 1] * np.sin(k * bz)
        out.append(v)
    return out + [0.0] * (3 - len(out))


def test_dns_program_tracks_particles(tmp_path):
    nstep = 6
    path, ctx, ic = _channel(tmp_path, "chp", 8, extra={"N_STEP": nstep, "IO_HIS": 2, "IO_FLD": nstep,
                                                       "SPAWN": 3, "D_T": 0.05})
    write_field(path + ".rst", "chp", ctx.np, ctx.nz, ctx.nel, 0, 0.0, 0.05, 1.0 / 200.0, 1.0,
                {**ic, "p": np.zeros_like(ic["u"])})
    places = [(0.4, -0.5, 0.3), (3.0, 0.2, 6.0), (5.8, 0.9, -1.0), (9.0, 0.0, 0.0)]   # the last is outside
    with open(path + ".par", "w") as f:
        for i, (x, y, z) in enumerate(places):
            f.write(f"{i + 1} 0.0 0.0 {x} {y} {z}\n")
    r = subprocess.run([os.path.join(BIN, "dns"), path], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    assert "Particle at (9.000000, 0.000000, 0.000000) not in mesh" in r.stderr
    # the same particles on the device DNS's fields, through the oracle
    Sn = O.read_session(path)
    M = O.Problem(Sn).M
    T = O.FluidParticles(M, Sn.tokens, 4)
    for i, pl in enumerate(places):
        if T.make(i + 1, pl, 0.0):
            T.initial.append(pl)
    D = S.DNS(ctx, 1)
    D.restart(ic, 0.0)
    want = []
    for step in range(1, nstep + 1):
        D.advance(1)
        t = D.state()[1]
        if step % 3 == 0:
            for i, pl in enumerate(T.initial):
                T.make(i + 1, pl, t)
        F = [_fourier(D, c) for c in "uvw"]
        T.integrate(lambda e, r_, s_, z: _probe_at(F, M, e, r_, s_, z, 1.0))
        if step % 2 == 0:
            want += [(q["id"], t, q["ctime"], q["x"], q["y"], q["z"]) for q in T.parts if q["e"] is not None]
    D.close()
    got = [ln.split() for ln in open(path + ".trk").read().splitlines()]
    assert len(got) == len(want) == 3 + 6 + 9   # three particles, three more every 3 steps
    for g, w in zip(got, want):
        assert int(g[0]) == w[0]
        for a, b in zip(g[1:], w[1:]):
            assert abs(float(a) - b) <= 2e-6 * abs(b) + 1e-9, (g, w)


def test_dns_program_phase_averages(tmp_path):
    from semtex_b200.fieldfile import read_field
    nstep = 8
    path = sessions.taylor_green_session(str(tmp_path / "tgp"), 3, 6, 8, re=100.0, dt=2e-3, nstep=nstep,
                                         extra={"TOL_REL": 1e-14, "AVERAGE": 2, "N_PHASE": 2, "STEPS_P": 4,
                                                "IO_FLD": 2, "IO_HIS": 4})
    ctx = S.Context(path)
    funcs = S._user_functions(path)
    ic = {c: ctx.evaluate(funcs[c], 0.0) for c in ctx.fields if c in funcs}
    write_field(path + ".rst", "tgp", ctx.np, ctx.nz, ctx.nel, 0, 0.0, 2e-3, 1.0 / 100.0, 1.0,
                {c: ic.get(c, np.zeros_like(ic["u"])) for c in ctx.fields})
    r = subprocess.run([os.path.join(BIN, "dns"), path], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    # the oracle's statistics, two phase sets and the running set, on the
    # device DNS's fields of the same steps
    P = O.Problem(O.read_session(path))
    sets = {}
    for key in ("0", "1", "avg"):
        sets[key] = O.DNS(P)
        sets[key].stats_init(2)
    D = S.DNS(ctx, 1)
    D.restart(ic, 0.0)
    for step in range(1, nstep + 1):
        D.advance(1)
        upd = []
        if step % 2 == 0:
            upd.append(str((step % 4) // 2))
        if step % 4 == 0:
            upd.append("avg")
        for key in upd:
            for c in ctx.fields:
                sets[key].u[c] = _fourier(D, c)
            sets[key].stats_update()
    D.close()
    for key, fn in (("0", path + ".0.phs"), ("1", path + ".1.phs"), ("avg", path + ".avg")):
        hdr, got = read_field(fn)
        ref = sets[key].stats_physical()
        assert hdr["step"] == 2 and sorted(got) == sorted(ref), (key, hdr["step"], sorted(got))
        for c in ref:
            scale = max(np.linalg.norm(ref[c]), 1e-300)
            assert np.linalg.norm(got[c] - ref[c]) / scale < (1e-9 if c == "p" else 1e-10), (key, c)
