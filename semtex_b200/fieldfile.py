"""Semtex binary field files (.fld / .rst / .chk / .frc).

Format of writeField / readField (src/misc.cpp:106-222) and the AuxField
binary stream operators (src/auxfield.cpp:1021-1113): ten text header lines
(25-character value column followed by a label), then each field's nz planes
of nel*np*np doubles in the writer's byte order.
"""

from __future__ import annotations

import sys
import time as _time

import numpy as np


def _fmt_g(v):
    return f"{v:<25.6g}"


def write_field(path, session, np_, nz, nel, step, time, dt, kinvis, beta, fields: dict):
    """Write physical-space fields {name: [nz, nel, np, np]}."""
    order = "little" if sys.byteorder == "little" else "big"
    created = _time.strftime("%a %b %d %H:%M:%S %Y", _time.localtime())[:24]
    hdr = [
        f"{session:<25s} Session",
        f"{created:<25s} Created",
        f"{f'{np_} {np_} {nz} {nel}':<25s} Nr, Ns, Nz, Elements",
        f"{step:<25d} Step",
        _fmt_g(time) + " Time",
        _fmt_g(dt) + " Time step",
        _fmt_g(kinvis) + " Kinvis",
        _fmt_g(beta) + " Beta",
        f"{''.join(fields.keys()):<25s} Fields written",
        f"{'binary IEEE ' + order + '-endian':<25s} Format",
    ]
    with open(path, "wb") as f:
        f.write(("\n".join(hdr) + "\n").encode())
        for v in fields.values():
            a = np.ascontiguousarray(v, dtype=np.float64)
            if a.size != np_ * np_ * nz * nel:
                raise ValueError("field size does not match header")
            f.write(a.tobytes())


def read_field(path):
    """Return (header dict, {name: [nz, nel, np, np]})."""
    with open(path, "rb") as f:
        lines = [f.readline().decode(errors="replace") for _ in range(10)]
        np_, _, nz, nel = (int(v) for v in lines[2].split()[:4])
        names = lines[8].split()[0]
        fmt = lines[9]
        dt = np.dtype("<f8")
        if "big" in fmt:
            dt = np.dtype(">f8")
        hdr = {"session": lines[0].split()[0], "np": np_, "nz": nz, "nel": nel,
               "step": int(lines[3].split()[0]), "time": float(lines[4].split()[0]),
               "dt": float(lines[5].split()[0]), "kinvis": float(lines[6].split()[0]),
               "beta": float(lines[7].split()[0]), "fields": names}
        n = np_ * np_ * nz * nel
        out = {}
        for c in names:
            buf = f.read(8 * n)
            if len(buf) != 8 * n:
                raise ValueError(f"{path}: truncated field '{c}'")
            out[c] = np.frombuffer(buf, dt).astype(np.float64).reshape(nz, nel, np_, np_)
    return hdr, out
