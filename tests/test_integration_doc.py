"""The Fortran binding include/msg123_gpu.f90 agrees with the C ABI.

No Fortran compiler exists here, so the `bind(C)` module a maintainer would add is checked
as text: each derived type must have the C struct's fields, in order, at the offsets C
gives them (interoperable types follow the companion C compiler's layout), and each bound
procedure must be declared in include/msg123_gpu.h with the same number of arguments.
"""
import ctypes as C
import os
import re

import pytest

from msg123_b200 import abi

ROOT = os.path.join(os.path.dirname(__file__), "..")
KINDS = {"integer(c_int32_t)": 4, "integer(c_int)": 4, "real(c_double)": 8, "real(c_float)": 4, "type(c_ptr)": 8}
STRUCTS = {"msg_grid_t": abi.MsgGrid, "msg_params_t": abi.MsgParams, "msg_stats_t": abi.MsgStats,
           "msg_run_stats_t": abi.MsgRunStats, "msg_convrec_t": abi.MsgConvRec}


def _module():
    """The module source with comments dropped and continuation lines joined."""
    text = open(os.path.join(ROOT, "include", "msg123_gpu.f90")).read()
    lines = [ln.split("!")[0].rstrip() for ln in text.splitlines()]
    return re.sub(r"&\s*\n\s*", " ", "\n".join(ln for ln in lines if ln.strip()))


def _types(src):
    out = {}
    for name, body in re.findall(r"type, bind\(C\) :: (\w+)\n(.*?)\n\s*end type", src, re.S):
        fields = []
        for line in body.splitlines():
            kind, names = line.split("::")
            size = KINDS[kind.strip()]
            fields += [(n.strip(), size) for n in names.split(",")]
        out[name] = fields
    return out


def _c_layout(fields):
    off, layout = 0, []
    for name, size in fields:
        off = (off + size - 1) // size * size
        layout.append((name, off))
        off += size
    align = max(s for _, s in fields)
    return layout, (off + align - 1) // align * align


@pytest.mark.parametrize("name", sorted(STRUCTS))
def test_fortran_types_match_c_structs(name):
    types = _types(_module())
    assert name in types, f"{name} missing from the Fortran module"
    layout, size = _c_layout(types[name])
    cls = STRUCTS[name]
    want = [(f, getattr(cls, f).offset) for f, _ in cls._fields_]
    assert layout == want
    assert size == C.sizeof(cls)


def test_bound_procedures_exist_in_header():
    src = _module()
    header = open(os.path.join(ROOT, "include", "msg123_gpu.h")).read()
    procs = re.findall(r"(?:function|subroutine) (msg_gpu_\w+)\(([^)]*)\)\s+bind\(C\)", src)
    assert len(procs) >= 20
    for name, args in procs:
        m = re.search(r"MSG_API [^;]*?\b" + name + r"\(([^)]*)\);", header, re.S)
        assert m, f"{name} is not declared in the header"
        nf = len([a for a in args.split(",") if a.strip()])
        nc = len([a for a in m.group(1).split(",") if a.strip() and a.strip() != "void"])
        assert nf == nc, (name, nf, nc)
