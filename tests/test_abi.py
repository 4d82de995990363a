"""The C-ABI library loads, exports every entry point of include/msg123_gpu.h, and the
ctypes struct layouts match the C header (checked with a compiled probe)."""
import ctypes as C
import os
import re
import subprocess

import pytest

from msg123_b200 import abi
from msg123_b200.solver import LIB_PATH

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "msg123_gpu.h")


def declared_symbols():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"\b(msg_gpu_\w+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    lib = C.CDLL(LIB_PATH)
    syms = declared_symbols()
    assert len(syms) >= 20
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing


def test_nm_exports_match_header():
    out = subprocess.run(["nm", "-D", "--defined-only", LIB_PATH], capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r" T (msg_gpu_\w+)", out))
    assert set(declared_symbols()) <= exported


@pytest.mark.parametrize("name,cls", [("msg_grid_t", abi.MsgGrid), ("msg_params_t", abi.MsgParams),
                                      ("msg_stats_t", abi.MsgStats), ("msg_run_stats_t", abi.MsgRunStats),
                                      ("msg_convrec_t", abi.MsgConvRec)])
def test_struct_layout_matches_header(tmp_path, name, cls):
    fields = [f for f, _ in cls._fields_]
    src = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"', 'int main(void){',
           f'printf("%zu\\n", sizeof({name}));']
    src += [f'printf("%zu\\n", offsetof({name}, {f}));' for f in fields]
    src += ['return 0;}']
    c = tmp_path / "probe.c"
    c.write_text("\n".join(src))
    exe = tmp_path / "probe"
    subprocess.run(["gcc", str(c), "-o", str(exe)], check=True)
    vals = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True).stdout.split()]
    assert vals[0] == C.sizeof(cls)
    assert vals[1:] == [getattr(cls, f).offset for f in fields]
