"""Corrupt or inconsistent sessions are reported as status codes, on the host.

The reference prints the message and exits (message(..., ERROR),
veclib/util.c:24-46); the library returns STX_ESESSION (or STX_EINVAL for a
bad argument) with the message in stx_last_error, and the process carries
on.  These run through stx_numbering_host, which needs no GPU.
"""
import pytest

import semtex_b200 as S
from semtex_b200 import _lib, sessions


def _ok(tmp_path, name="ok", **kw):
    return sessions.helmholtz_session(str(tmp_path / name), 3, 5, nz=1, lambda2=1.0, beta=1.0, **kw)


def _code(path, field="c"):
    with pytest.raises(_lib.StxError) as e:
        S.numbering(path, field)
    return e.value.code, str(e.value)


def test_missing_session_file(tmp_path):
    code, msg = _code(str(tmp_path / "does_not_exist"))
    assert code == _lib.STX_ESESSION


def test_field_not_in_session(tmp_path):
    code, _ = _code(_ok(tmp_path), field="q")
    assert code in (_lib.STX_ESESSION, _lib.STX_EINVAL)


def test_element_with_unknown_node(tmp_path):
    # an element naming a vertex past the end of <NODES>
    p = _ok(tmp_path)
    txt = open(p).read()
    head, _, rest = txt.partition("<ELEMENTS")
    body, _, tail = rest.partition("</ELEMENTS>")
    lines = body.split("\n")
    for i, ln in enumerate(lines):
        if "<Q>" in ln:
            parts = ln.split()
            k = parts.index("<Q>")
            parts[k + 1] = "9999"
            lines[i] = "\t" + "\t".join(parts)
            break
    open(p, "w").write(head + "<ELEMENTS" + "\n".join(lines) + "</ELEMENTS>" + tail)
    code, _ = _code(p)
    assert code == _lib.STX_ESESSION


def test_bad_token_expression(tmp_path):
    p = _ok(tmp_path)
    txt = open(p).read().replace("N_P = 5", "N_P = 5 * (", 1)
    open(p, "w").write(txt)
    code, _ = _code(p)
    assert code == _lib.STX_ESESSION


def test_unknown_bc_kind(tmp_path):
    p = _ok(tmp_path)
    txt = open(p).read().replace("<D>", "<Z>").replace("</D>", "</Z>")
    open(p, "w").write(txt)
    code, msg = _code(p)
    assert code in (_lib.STX_ESESSION, _lib.STX_EUNSUPPORTED)


def test_library_usable_after_errors(tmp_path):
    with pytest.raises(_lib.StxError):
        S.numbering(str(tmp_path / "nope"), "c")
    n = S.numbering(_ok(tmp_path, "fine"), "c")
    assert n["nglobal"] > n["nsolve"] > 0
    assert _lib.lib().stx_last_error() == b""
