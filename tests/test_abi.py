"""The C ABI without a GPU: the built library loads and exports every entry point include/mose_b200.h
declares, the ctypes mirror matches the C struct layouts, and the host-side checks of mb_init reject bad
input before any device work (no compute call is made here)."""
import ctypes as C
import os
import re
import subprocess

import pytest

from mosegpu import abi
from mosegpu import engine

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "mose_b200.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    inline = set(re.findall(r"static\s+inline\s+\w+\s+(mb_[a-z_]+)\s*\(", src))   # header-only helpers
    return sorted(set(re.findall(r"\b(mb_[a-z_]+)\s*\(", src)) - inline)


def test_library_loads_and_exports_every_declared_symbol():
    if not os.path.exists(engine.LIB_PATH):
        import build  # noqa: F401  (mose-gpu_b200/build.py)
        build.build()
    L = engine.load_library()
    names = declared_functions()
    assert len(names) >= 12
    for n in names:
        assert hasattr(L, n), n
    assert L.mb_version().startswith(b"mose_b200")


def test_struct_layouts_match_the_header(tmp_path):
    prog = tmp_path / "sizes.c"
    prog.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "mose_b200.h"\nint main(void){\n'
                    'printf("%zu %zu %zu %zu %zu %zu %zu\\n", sizeof(mb_block), sizeof(mb_bc), sizeof(mb_conn),'
                    ' sizeof(mb_mesh), sizeof(mb_thermo), sizeof(mb_scheme), sizeof(mb_status));\n'
                    'printf("%zu %zu %zu\\n", offsetof(mb_scheme, cfl), offsetof(mb_bc, q), offsetof(mb_mesh, blk));\n'
                    'return 0;}\n')
    exe = tmp_path / "sizes"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(prog), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()
    got = [int(x) for x in out]
    want = [C.sizeof(abi.MBBlock), C.sizeof(abi.MBBc), C.sizeof(abi.MBConn), C.sizeof(abi.MBMesh),
            C.sizeof(abi.MBThermo), C.sizeof(abi.MBScheme), C.sizeof(abi.MBStatus),
            abi.MBScheme.cfl.offset, abi.MBBc.q.offset, abi.MBMesh.blk.offset]
    assert got == want


def test_init_rejects_bad_arguments_without_a_device():
    L = engine.load_library()
    h = C.c_void_p()
    assert L.mb_init(None, None, None, 0, C.byref(h)) == abi.MB_E_ARG
    mesh = abi.MBMesh()
    mesh.nblk = 1
    mesh.ncell_total = 10
    sc = abi.MBScheme()
    sc.riemann = 14   # HLLC-PC (preconditioned integration variables): not served
    sc.limiter = 1
    sc.n_rk = 3
    sc.ndir = 3
    th = abi.MBThermo()
    assert L.mb_init(C.byref(mesh), C.byref(sc), C.byref(th), 0, C.byref(h)) == abi.MB_E_UNSUPPORTED
    sc.riemann = abi.RS_HLLC
    sc.n_rk = 7
    assert L.mb_init(C.byref(mesh), C.byref(sc), C.byref(th), 0, C.byref(h)) == abi.MB_E_UNSUPPORTED


def test_engine_refuses_to_run_without_cuda():
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    from mosegpu import case as cs
    with pytest.raises(RuntimeError):
        engine.Engine(cs.riemann_1d(n=16))
