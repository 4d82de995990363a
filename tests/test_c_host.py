"""The C ABI from a C host: tests/c_host/abi_host.c is compiled with gcc against
include/msg123_gpu.h, linked with the in-tree libmsg123gpu.so and run; it reads a restart
file written here in gfortran's record layout and exercises the argument checks (no GPU
needed for either)."""
import os
import struct
import subprocess

import numpy as np

from msg123_b200.solver import LIB_PATH

ROOT = os.path.join(os.path.dirname(__file__), "..")


def test_c_host_links_and_calls_the_abi(tmp_path):
    exe = tmp_path / "abi_host"
    libdir = os.path.dirname(LIB_PATH)
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "c_host", "abi_host.c"), "-L", libdir, "-lmsg123gpu",
                    "-Wl,-rpath," + libdir, "-o", str(exe)], check=True)
    vals = np.arange(1.0, 11.0)
    f = tmp_path / "rest.bin"
    b = vals.astype("<f8").tobytes()
    f.write_bytes(struct.pack("<i", 8) + struct.pack("<d", 7200.0) + struct.pack("<i", 8)
                  + struct.pack("<i", len(b)) + b + struct.pack("<i", len(b)))
    out = subprocess.run([str(exe), str(f), "10"], check=True, capture_output=True, text=True).stdout.splitlines()
    inv = float(np.float32(1.0) / np.float32(10.0))
    assert out[0] == f"read_restart rc=0 time=7200.0 sum={sum(v * inv for v in vals):.17g}"
    assert out[1].startswith("read_restart(wrong n) rc=-3") and "not a restart file of 11 cells" in out[1]
    assert out[2].startswith("create(vg_form=7) rc=-1 ctx=null") and "vg_form" in out[2]
    assert out[3].startswith("create(null arrays) rc=-1") and "NULL" in out[3]
