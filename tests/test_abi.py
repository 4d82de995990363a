"""The C-ABI library loads, exports every entry point of include/msg123_gpu.h, the ctypes
struct layouts match the C header (checked with a compiled probe), and the argument checks
that precede any device work return their status and message without a GPU."""
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


def _lib():
    L = C.CDLL(LIB_PATH)
    L.msg_gpu_last_error.restype = C.c_char_p
    L.msg_gpu_create.argtypes = [C.POINTER(abi.MsgGrid), C.POINTER(abi.MsgParams), C.POINTER(C.c_void_p)]
    return L


@pytest.mark.parametrize("change,code,words", [
    (dict(vg_form=3), abi.MSG_ERR_ARG, "vg_form"),
    (dict(precision=2), abi.MSG_ERR_ARG, "precision"),
    (dict(maxout_iter=0), abi.MSG_ERR_ARG, "iteration caps"),
    (dict(len_scal=0.0), abi.MSG_ERR_ARG, "len_scal"),
])
def test_create_rejects_bad_parameters(change, code, words):
    """Argument checks come before any device work, so they run here without a GPU: a bad
    knob is a negative status with a message, never a crash or a half-built context."""
    from msg123_b200.config import make_config
    L = _lib()
    p = make_config("box", shape=(3, 3, 3))
    prm = dict(p.params, **change)
    g, q, ctx = abi.fill_grid(p), abi.fill_params(prm), C.c_void_p()
    rc = L.msg_gpu_create(C.byref(g), C.byref(q), C.byref(ctx))
    assert rc == code and ctx.value is None
    assert words in L.msg_gpu_last_error().decode()


def test_create_rejects_empty_grid_and_null_arrays():
    from msg123_b200.config import make_config
    L = _lib()
    p = make_config("box", shape=(3, 3, 3))
    g, q, ctx = abi.fill_grid(p), abi.fill_params(p.params), C.c_void_p()
    g.nz = 0
    assert L.msg_gpu_create(C.byref(g), C.byref(q), C.byref(ctx)) == abi.MSG_ERR_SIZE
    g = abi.fill_grid(p)
    g.ksz = None
    assert L.msg_gpu_create(C.byref(g), C.byref(q), C.byref(ctx)) == abi.MSG_ERR_ARG
    assert "NULL" in L.msg_gpu_last_error().decode()
    assert L.msg_gpu_create(None, C.byref(q), C.byref(ctx)) == abi.MSG_ERR_ARG


def test_null_context_is_an_argument_error():
    L = _lib()
    buf = (abi.MsgConvRec * 4)()
    out = (C.c_double * 4)()
    assert L.msg_gpu_convlog(None, buf, 4) == abi.MSG_ERR_ARG
    assert L.msg_gpu_set_convlog(None, 1) == abi.MSG_ERR_ARG
    assert L.msg_gpu_water_table(None, out) == abi.MSG_ERR_ARG
    assert L.msg_gpu_calc_mass(None, out) == abi.MSG_ERR_ARG
    L.msg_gpu_destroy(None)                   # a no-op


def test_missing_library_fails_loudly(monkeypatch):
    """No CPU fallback: without the CUDA library every entry into the solver raises."""
    from msg123_b200 import solver
    monkeypatch.setattr(solver, "_lib", None)
    monkeypatch.setattr(solver, "LIB_PATH", "/nonexistent/libmsg123gpu.so")
    with pytest.raises(solver.MsgError, match="missing"):
        solver.load_library()


def test_smoke_fails_loudly_without_a_gpu():
    """On a machine without a GPU the smoke check raises the library's CUDA error instead of
    passing on some host path."""
    from conftest import has_gpu
    if has_gpu():
        pytest.skip("a GPU is present")
    import __graft_entry__ as entry
    from msg123_b200.solver import MsgError
    with pytest.raises(MsgError, match="err_cuda"):
        entry.smoke()
