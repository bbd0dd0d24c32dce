"""The C ABI without a GPU: the built library loads and exports every entry point include/mose_b200.h
declares, the ctypes mirror matches the C struct layouts, and the host-side checks of mb_init reject bad
input before any device work (no compute call is made here)."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
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


def _noalloc_shape(L, n1, n2, n3):
    n = (C.c_int32 * 3)(n1, n2, n3)
    kc, nt = C.c_int32(), C.c_int32()
    rc = L.mb_dt_block_noalloc_tiles(n, C.byref(kc), C.byref(nt))
    return rc, kc.value, nt.value


def test_noalloc_tile_shape_at_the_partials_boundary():
    """mb_dt_block_noalloc keeps one partial minimum per tile in a static array of 65536: its k chunk starts at 16
    planes and doubles until the tiles fit. At 4096 (i, j) tiles, 256 planes fit in 16-plane chunks exactly; one
    plane more needs 32-plane chunks, and the chunks of the kernel's decomposition cover every plane once."""
    L = engine.load_library()
    ti, tj = 64, 64
    assert _noalloc_shape(L, 32 * ti, 8 * tj, 256) == (abi.MB_OK, 16, 65536)
    rc, kc, nt = _noalloc_shape(L, 32 * ti, 8 * tj, 257)
    assert (rc, kc, nt) == (abi.MB_OK, 32, ti * tj * 9)
    # the decomposition of the kernel (k_dt_partials): tile t -> i-tile t % ti, j-tile (t / ti) % tj, planes
    # 1 + kc * (t / (ti tj)) .. min(that + kc, n3 + 1) - 1
    t = np.arange(nt)
    kt = t // (ti * tj)
    k0 = 1 + kc * kt
    k1 = np.minimum(k0 + kc, 257 + 1)
    cover = np.zeros((ti * tj, 257 + 2), dtype=np.int64)
    ij = t % (ti * tj)
    for q in range(kc):                      # plane k0 + q of every tile, where it is below k1
        k = k0 + q
        ok = k < k1
        np.add.at(cover, (ij[ok], k[ok]), 1)
    assert (cover[:, 1:258] == 1).all() and cover[:, 0].sum() == 0 and cover[:, 258].sum() == 0
    # a single plane of more than 65536 tiles is refused
    assert _noalloc_shape(L, 32 * 65537, 8, 1)[0] == abi.MB_E_ARG
    assert _noalloc_shape(L, 32 * 256, 8 * 256, 1) == (abi.MB_OK, 16, 65536)


def test_noalloc_refuses_preconditioning_before_any_device_work():
    """integration-variables = prec takes its steps from a context's Ur field: mb_dt_block_noalloc refuses it
    (host check, no launch, so it runs without a GPU)."""
    L = engine.load_library()
    sc = abi.MBScheme()
    sc.ndir = 3
    sc.cfl = 0.5
    sc.intvar = 2
    n = (C.c_int32 * 3)(8, 8, 8)
    dummy = C.c_void_p(1)                    # never dereferenced: the scheme check comes first
    f = L.mb_dt_block_noalloc
    f.argtypes = [C.c_void_p, C.c_int64, C.c_int64, C.POINTER(C.c_int32)] + [C.c_void_p] * 5 + \
                 [C.c_int32, C.c_int32, C.c_double, C.POINTER(abi.MBScheme), C.c_void_p, C.c_void_p]
    f.restype = C.c_int
    rc = f(dummy, 1 << 20, 0, n, dummy, dummy, dummy, dummy, dummy, 0, 10000, 28.97, C.byref(sc), dummy, None)
    assert rc == abi.MB_E_UNSUPPORTED
