"""The `elliptic` and `dns` programs (semtex_b200/bin), built over the C ABI.

CPU: they exist and print their usage.  GPU: the reference's own regression
workflow (test/testregress:14-30) -- a restart file holding the USER-section
solution at t = 0, `dns -chk session`, then the errors of session.fld -- and
`elliptic` on the test sessions, against the oracle.
"""
import json
import os
import shutil
import subprocess

import numpy as np
import pytest

import semtex_oracle as O
from semtex_b200.fieldfile import read_field, write_field

from conftest import GOLDEN, SESSIONS

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "semtex_b200", "bin")
GOLD = json.load(open(os.path.join(GOLDEN, "regress_ok.json")))["goldens"]


@pytest.mark.parametrize("prog", ["dns", "elliptic"])
def test_programs_print_usage(prog):
    r = subprocess.run([os.path.join(BIN, prog), "-h"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0 and "Usage" in r.stdout


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["helmholtz1", "mixed1"])
def test_elliptic_program(tmp_path, name):
    path = str(tmp_path / name)
    shutil.copy(os.path.join(SESSIONS, name), path)
    r = subprocess.run([os.path.join(BIN, "elliptic"), path], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    hdr, flds = read_field(path + ".fld")
    P, U = O.elliptic(path)
    u = flds[P.S.fields[0]]
    assert np.linalg.norm(u - U) / np.linalg.norm(U) < 1e-10
    assert "norm_inf" in r.stdout


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["kovas1", "taylor2"])
def test_dns_program_regression_workflow(tmp_path, name):
    path = str(tmp_path / name)
    shutil.copy(os.path.join(SESSIONS, name), path)
    S = O.read_session(path)
    P = O.Problem(S)
    funcs = O.user_functions(S)
    ic = {c: P.evaluate(funcs[c], 0.0) for c in S.fields if c in funcs}   # what `compare` writes
    write_field(path + ".rst", name, P.np, P.nz, P.nel, 0, 0.0, S.tokens["D_T"], S.tokens["KINVIS"],
                S.tokens["BETA"], ic)
    r = subprocess.run([os.path.join(BIN, "dns"), "-chk", path], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    hdr, flds = read_field(path + ".fld")
    assert hdr["step"] == S.tokens.ivalue("N_STEP")
    t = float(f"{hdr['time']:.6g}")
    for c in S.fields:
        err = np.abs(P.evaluate(funcs[c], t) - flds[c]).max()
        got = "noise-level" if err < 1e-12 else f"{err:.4e}"
        assert got == GOLD[name][c], (name, c, got)


@pytest.mark.gpu
def test_dns_program_writes_averages(tmp_path):
    # AVERAGE = 2: running averages updated every IO_HIS steps, written to
    # session.avg with the dumps (step = number of updates), names in the
    # reference's order.
    from semtex_b200 import sessions
    path = sessions.taylor_green_session(str(tmp_path / "tgavg"), 3, 6, 8, re=100.0, dt=2e-3, nstep=12,
                                         extra={"TOL_REL": 1e-14, "AVERAGE": 2, "IO_HIS": 3, "IO_FLD": 6})
    S = O.read_session(path)
    P = O.Problem(S)
    funcs = O.user_functions(S)
    ic = {c: P.evaluate(funcs[c], 0.0) for c in S.fields if c in funcs}
    write_field(path + ".rst", "tgavg", P.np, P.nz, P.nel, 0, 0.0, S.tokens["D_T"], S.tokens["KINVIS"],
                S.tokens["BETA"], ic)
    r = subprocess.run([os.path.join(BIN, "dns"), path], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    hdr, avg = read_field(path + ".avg")
    assert hdr["fields"] == "ABCDEFpuvw" and hdr["step"] == 4
    hdr, chk = read_field(path + ".chk")
    assert hdr["step"] == 6
    hdr, fld = read_field(path + ".fld")
    assert hdr["step"] == 12
    assert np.all(np.isfinite(avg["A"])) and np.abs(avg["A"]).max() > 0.1


@pytest.mark.gpu
def test_dns_program_iterative_option(tmp_path):
    # -i: Jacobi-PCG viscous steps (token ITERATIVE = 1), as the library
    # runs them with the token set
    import semtex_b200 as S
    from semtex_b200 import sessions
    path = sessions.channel_session(str(tmp_path / "chi"), 4, 2, 6, 4, re=200.0, dt=5e-3, nstep=6,
                                    extra={"TOL_REL": 1e-12})
    ctx = S.Context(path, overrides={"ITERATIVE": 1})
    x, y = ctx.mesh_coords()
    ic = sessions.channel_initial(x, y, np.arange(ctx.nz) * 2 * np.pi / ctx.nz, amplitude=0.05)
    ic = {c: ic[c] for c in ctx.fields[:-1]}
    write_field(path + ".rst", "chi", ctx.np, ctx.nz, ctx.nel, 0, 0.0, 5e-3, 1.0 / 200.0, 1.0,
                {**ic, "p": np.zeros_like(ic["u"])})
    r = subprocess.run([os.path.join(BIN, "dns"), "-i", "-chk", path], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    hdr, flds = read_field(path + ".fld")
    D = S.DNS(ctx, 1)
    D.restart(ic, 0.0)
    D.advance(6)
    for c in ctx.fields:
        want = D.field(c)
        tol = 1e-8 if c == "p" else 1e-10
        assert np.linalg.norm(flds[c] - want) <= tol * np.linalg.norm(want), c
    D.close()
