"""ctypes binding of ``libsemtex_b200.so`` (declarations of include/semtex_b200.h).

The library is loaded from the package directory; a missing library is an
ImportError-grade failure, never a silent fallback.
"""

from __future__ import annotations

import ctypes as C
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsemtex_b200.so")
HEADER = os.path.join(HERE, "..", "include", "semtex_b200.h")

STX_OK, STX_EINVAL, STX_ESESSION, STX_ENUMERIC, STX_ECUDA, STX_ENOCONV, STX_EUNSUPPORTED = range(7)
STX_DIRECT, STX_JACPCG, STX_MIXED = 0, 1, 2
FORWARD, INVERSE = 1, -1

_p = C.c_void_p
_i = C.c_int
_d = C.c_double
_pd = C.POINTER(C.c_double)
_pi = C.POINTER(C.c_int)
_s = C.c_char_p

SIGNATURES = {
    "stx_last_error": (_s, []),
    "stx_context_create": (_i, [_s, _s, _i, _p, C.POINTER(_p)]),
    "stx_context_destroy": (_i, [_p]),
    "stx_context_geometry": (_i, [_p, _pi, _pi, _pi, _pi]),
    "stx_context_fields": (_i, [_p, _s, _i]),
    "stx_token": (_i, [_p, _s, _pd]),
    "stx_numbering": (_i, [_p, C.c_char, _pi, _pi, _pi]),
    "stx_numbering_host": (_i, [_s, _s, C.c_char, _pi, _pi, _pi, _pi, _pi, _p, _p]),
    "stx_numbering_host_mode": (_i, [_s, _s, C.c_char, _i, _pi, _pi, _pi, _pi, _pi, _p, _p]),
    "stx_element_matrix_host": (_i, [_s, _s, _i, _d, _d, _pi, _p]),
    "stx_mesh_coords": (_i, [_p, _p, _p]),
    "stx_mesh_families": (_i, [_p, _pi]),
    "stx_mesh_mass": (_i, [_p, _p]),
    "stx_mesh_locate": (_i, [_p, _i, _p, _p, _p]),
    "stx_mesh_locate_host": (_i, [_s, _s, _i, _p, _p, _p]),
    "stx_mesh_relocate": (_i, [_p, _i, _p, _p, _p]),
    "stx_mesh_relocate_host": (_i, [_s, _s, _i, _p, _p, _p]),
    "stx_field_evaluate": (_i, [_p, _s, _d, _p]),
    "stx_expression_eval": (_i, [_s, _s, _i, _i, _p, _p, _p, _d, _p, _pi]),
    "stx_svv": (_i, [_i, _d, _i, _i, _d, _i, _d, _p, _p]),
    "stx_session_force_value": (_i, [_s, _s, _p, _i, _pi]),
    "stx_field_bc_evaluate": (_i, [_p, C.c_char, _d]),
    "stx_modal_create": (_i, [_p, C.c_char, _d, _d, _i, _i, _i, C.POINTER(_p)]),
    "stx_modal_destroy": (_i, [_p]),
    "stx_modal_info": (_i, [_p, _i, _pi, _pi]),
    "stx_field_solve": (_i, [_p, _p, _p, _d, _i, _pi]),
    "stx_transform": (_i, [_p, _p, _i]),
    "stx_field_solve_profiled": (_i, [_p, _p, _p, C.POINTER(C.c_float), _pi]),
    "stx_field_solve_noalloc": (_i, [_p, _p, _p]),
    "stx_field_solve_multi": (_i, [_p, _i, _p, _p]),
    "stx_modal_bytes": (_i, [_p, _pd]),
    "stx_modal_launches": (_i, [_p, _pi]),
    "stx_modal_status": (_i, [_p, _pi]),
    "stx_dns_create": (_i, [_p, _i, C.POINTER(_p)]),
    "stx_dns_destroy": (_i, [_p]),
    "stx_dns_restart": (_i, [_p, _d]),
    "stx_dns_set_field": (_i, [_p, C.c_char, _p]),
    "stx_dns_get_field": (_i, [_p, C.c_char, _p]),
    "stx_dns_advance": (_i, [_p, _i]),
    "stx_dns_state": (_i, [_p, _pi, _pd]),
    "stx_dns_field_ptr": (_i, [_p, C.c_char, C.POINTER(_p)]),
    "stx_dns_system": (_i, [_p, C.c_char, C.POINTER(_p)]),
    "stx_elliptic_solve_host_batch": (_i, [_p, _i, C.POINTER(_p), C.POINTER(_p)]),
    "stx_dns_checkpoint_size": (_i, [_p, C.POINTER(C.c_ulonglong)]),
    "stx_dns_checkpoint_save": (_i, [_p, _p, C.c_ulonglong]),
    "stx_dns_checkpoint_load": (_i, [_p, _p, C.c_ulonglong]),
    "stx_dns_modal_energy": (_i, [_p, _p]),
    "stx_dns_divergence_energy": (_i, [_p, _pd]),
    "stx_dns_cfl": (_i, [_p, _pd]),
    "stx_dns_probe": (_i, [_p, _i, _p, _p, _p, _p]),
    "stx_dns_wall_forces": (_i, [_p, _p, _p]),
    "stx_dns_wall_traction": (_i, [_p, _pi, _p]),
    "stx_dns_graph_info": (_i, [_p, _pi, C.POINTER(C.c_longlong)]),
    "stx_dns_status": (_i, [_p, _pi]),
    "stx_dns_stats_update": (_i, [_p]),
    "stx_dns_stats_info": (_i, [_p, _s, _i, _pi, _i]),
    "stx_dns_stats_get": (_i, [_p, C.c_char, _p]),
    "stx_dns_stats_set": (_i, [_p, C.c_char, _p]),
    "stx_dns_stats_swap": (_i, [_p]),
    "stx_dns_adjoint_create": (_i, [_p, _i, C.POINTER(_p)]),
    "stx_dns_adjoint_destroy": (_i, [_p]),
    "stx_dns_adjoint_record": (_i, [_p, _i]),
    "stx_dns_adjoint_backward": (_i, [_p, _p, _p]),
    "stx_dns_adjoint_tangent": (_i, [_p, _p, _p]),
    "stx_dns_adjoint_info": (_i, [_p, _pi, _pi, C.POINTER(C.c_ulonglong)]),
    "stx_elliptic_solve_host": (_i, [_p, _p, _p]),
    "stx_sync": (_i, [_p]),
    "stx_context_stream": (_i, [_p, C.POINTER(_p)]),
    "stx_context_scratch": (_i, [_p, C.c_ulonglong, C.POINTER(_p)]),
    "stx_batch_create": (_i, [_p, _p, _p, _i, _p, C.POINTER(_p)]),
    "stx_batch_launch": (_i, [_p]),
    "stx_batch_info": (_i, [_p, _pi, _pi, C.POINTER(_p)]),
    "stx_batch_destroy": (_i, [_p]),
}


class StxError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"[stx error {code}] {msg}")
        self.code = code


_LIB = None


def header_symbols():
    """Names of the functions include/semtex_b200.h declares."""
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"\b(stx_[a-z0-9_]+)\s*\(", txt)))


def lib():
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"semtex_b200 native library missing: {LIB_PATH} "
                              "(run semtex_b200/build.py)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _LIB = L
    return _LIB


def check(rc):
    if rc != STX_OK:
        raise StxError(rc, lib().stx_last_error().decode())
    return rc
