"""Body forcing (<FORCE>, dns/fieldforce.cpp) on the CPU: the FORCE-section
token lookup (FEML::valueFromSection, src/feml.cpp:430-560), the compiled
expression programs the device runs for forcing fields against the
interpreter, and the oracle's forced DNS on an exact steady solution."""
import numpy as np
import pytest

import semtex_oracle as O
import semtex_b200 as S
from semtex_b200 import sessions


def _session(lines):
    return O.Session("s", O.Tokens(), "uvp", {}, {}, None, None, [], [], lines)


def test_force_section_lookup():
    S_ = _session(["CONST_X = 1.5", "# a comment hides the next line", "CONST_Y = 2", "\tSPONGE_M=0.5*x",
                   "A =x= 3", "MOD_ALPHA_X"])
    assert O.force_value(S_, "CONST_X") == " 1.5"
    assert O.force_value(S_, "CONST_Y") is None          # skipped with the comment line
    assert O.force_value(S_, "SPONGE_M") == "0.5*x"
    assert O.force_value(S_, "A") == "x"                 # the value ends at the next '='
    assert O.force_value(S_, "MOD_ALPHA_X") is None      # a token without a value
    assert O.force_value(S_, "CONST") is None            # whole words only
    assert O.force_value(_session(None), "CONST_X") is None


EXPRESSIONS = [
    "sin(x)*cos(y)*cos(z)+t", "-x^2", "2^-1^2", "x&y", "y~x", "x%0.7", "1/(x-x)", "heav(x-1)+sgn(y)",
    "jn(2,x)+yn(1,x+1)+j0(x)+y1(x+2)+j1(x)+y0(x+1)", "rad(x,y)+ang(x,y)+step(x,1)", "gamma(x+1)+lgamma(x+1)",
    "2*KINVIS+PI", "a*x", "erf(x)+erfc(y)+int(x)+floor(y)+ceil(y)+abs(y)",
    "acosh(x+1)+asinh(y)+atanh(y/2)+log(x+1)+log10(x+1)+sqrt(x)", "tan(y)+exp(-x)+sinh(y)+cosh(y)+tanh(z)",
    "acos(y/2)+asin(y/2)+atan(x)", "0.5*(1+tanh((x-5)/0.5))*(1-y*y)^2*cos(2*PI*t/4)",
]


@pytest.mark.parametrize("expr", EXPRESSIONS)
def test_compiled_programs_match_interpreter(expr):
    rng = np.random.default_rng(7)
    x, y, z = rng.uniform(0.1, 3, 64), rng.uniform(-1, 1, 64), rng.uniform(0, 6, 64)
    a, nops = S.expression(expr, x, y, z, 0.3, "a=3;KINVIS=0.01", compiled=True)
    b, _ = S.expression(expr, x, y, z, 0.3, "a=3;KINVIS=0.01", compiled=False)
    assert nops >= 1
    np.testing.assert_array_equal(a, b)


def test_constant_folding():
    _, n = S.expression("2*KINVIS+PI^2-sin(PI/2)", [0.0], [0.0], [0.0])
    assert n == 1
    _, n = S.expression("x*(2+3)", [0.0], [0.0], [0.0])
    assert n == 3


@pytest.mark.parametrize("bad", ["a=3", "foo(x)", "sin(x,y)", "(x+1", "x+"])
def test_compile_errors(bad):
    with pytest.raises(S.StxError):
        S.expression(bad, [0.0], [0.0], [0.0])


def test_oracle_poiseuille_stays_steady(tmp_path):
    # u = 1 - y^2 driven by CONST_X = 2 KINVIS is an exact steady solution
    # (nu u'' + f = 0) that the polynomial basis represents exactly.
    p = sessions.rect_session(str(tmp_path / "pois"), 4, 3, x=(0.0, 2.0), y=(-1.0, 1.0),
                              tokens={"N_P": 6, "N_TIME": 2, "D_T": 0.01, "KINVIS": 0.1, "N_STEP": 5,
                                      "TOL_REL": 1e-14},
                              fields="uvp", periodic_x=True,
                              bcs={"w": {"u": "<D> 0", "v": "<D> 0", "p": "<H> 0"}},
                              user=["u = 1-y*y", "v = 0", "p = 0"], force=["CONST_X = 2*KINVIS"])
    D = O.dns_session(p)
    ph = D.physical()
    assert np.abs(ph["u"] - (1 - D.P.M.y ** 2)).max() < 1e-13
    assert np.abs(ph["v"]).max() < 1e-13
    # without the force the same flow decays
    D0 = O.dns_session(p)
    D0.force = None
    D0.advance(5)
    assert np.abs(D0.physical()["u"] - ph["u"]).max() > 1e-3


def test_force_section_lookup_matches_oracle(tmp_path):
    # the library's FORCE-section reader (host, no device) against the
    # oracle's restatement of FEML::valueFromSection, quirks included
    import ctypes as C
    from semtex_b200._lib import lib
    lines = ["CONST_X = 1.5", "# a comment hides the next line", "CONST_Y = 2", "\tSPONGE_M=0.5*x",
             "A =x= 3", "MOD_ALPHA_X", "STEADY_FILE =forcing.fld", "  SFD_CHI  =  0.25  "]
    p = sessions.rect_session(str(tmp_path / "fs"), 2, 2, tokens={"N_P": 3}, fields="uvp", force=lines)
    txt = open(p).read().replace("\t# a comment", "# a comment")   # a '#' in the first column
    open(p, "w").write(txt)
    S_ = O.read_session(p)
    assert O.force_value(S_, "CONST_Y") is None
    for tok in ("CONST_X", "CONST_Y", "SPONGE_M", "A", "MOD_ALPHA_X", "STEADY_FILE", "SFD_CHI", "CONST",
                "NOT_THERE"):
        buf = C.create_string_buffer(256)
        found = C.c_int()
        assert lib().stx_session_force_value(p.encode(), tok.encode(), buf, 256, C.byref(found)) == 0
        want = O.force_value(S_, tok)
        got = buf.value.decode() if found.value else None
        assert got == want, (tok, got, want)
