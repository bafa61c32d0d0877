"""The C ABI library loads and exports every symbol include/v3dm.h declares (no GPU needed)."""
import ctypes as C
import re

import pytest


def _declared(header):
    return sorted(set(re.findall(r"V3DM_API\s+(?:const\s+char\s*\*|int)\s+(v3dm_\w+)\s*\(", header.read_text())))


def test_exports_every_declared_symbol(v3dm_mod):
    names = _declared(v3dm_mod.HEADER_PATH)
    assert len(names) >= 25
    lib = C.CDLL(str(v3dm_mod.LIB_PATH))
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_status_strings(v3dm_mod):
    lib = v3dm_mod.lib()
    for s in range(0, 11):
        assert lib.v3dm_status_string(s) and lib.v3dm_status_string(s) != b"unknown status"


def test_no_cpu_fallback_without_gpu(v3dm_mod):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(v3dm_mod.V3DMError) as e:
        v3dm_mod.SIFTMatching()
    assert e.value.status == v3dm_mod.ERR_NO_DEVICE
    with pytest.raises(v3dm_mod.V3DMError) as e:
        v3dm_mod.VocabularyTreeTraversal(10, 3)
    assert e.value.status == v3dm_mod.ERR_NO_DEVICE
    for make in (v3dm_mod.BatchMatching, v3dm_mod.Loader, v3dm_mod.Retrieval, v3dm_mod.Ransac):
        with pytest.raises(v3dm_mod.V3DMError) as e:
            make()
        assert e.value.status == v3dm_mod.ERR_NO_DEVICE, make.__name__


def test_null_arguments_are_rejected(v3dm_mod):
    lib = v3dm_mod.lib()
    assert lib.v3dm_matcher_create(None, 0, 0) == v3dm_mod.ERR_ARG
    assert lib.v3dm_allocate(None, 10, 10, 0) == v3dm_mod.ERR_ARG
    assert lib.v3dm_putative(None, 0.7, 0.8, None, 0, None) == v3dm_mod.ERR_ARG
    assert lib.v3dm_voctree_counts(0, 3, None, None) == v3dm_mod.ERR_ARG
    assert v3dm_mod.voctree_counts(10, 6) == (1111110, 1000000)
    assert v3dm_mod.voctree_counts(50, 3) == (127550, 125000)
    assert lib.v3dm_retrieval_create(None, 0) == v3dm_mod.ERR_ARG
    assert lib.v3dm_ransac_create(None, 0) == v3dm_mod.ERR_ARG
    assert lib.v3dm_retrieval_binomial(None, 10, 1, None, None, 0.1, 1, None, None) == v3dm_mod.ERR_ARG
    assert lib.v3dm_ransac_essential(None, 1, None, None, None, 2.0, 10, 11, None, 0, None, None, None) == \
        v3dm_mod.ERR_ARG
    assert lib.v3dm_retrieval_wait(None) == v3dm_mod.ERR_ARG and lib.v3dm_ransac_wait(None) == v3dm_mod.ERR_ARG


def test_header_is_plain_c_and_links(v3dm_mod, tmp_path):
    """include/v3dm.h compiles as C99 (-Wall -Werror -pedantic) and every declared entry point links
    against libv3dm.so from a C program, as a cgo / JNI / FFI binding would see it."""
    import shutil
    import subprocess
    if shutil.which("gcc") is None:
        pytest.skip("no gcc")
    names = _declared(v3dm_mod.HEADER_PATH)
    src = tmp_path / "abi_check.c"
    body = "\n".join(f"  p[{i}] = (void (*)(void))&{n};" for i, n in enumerate(names))
    src.write_text('#include "v3dm.h"\n#include <stdio.h>\n\nint main(void) {\n'
                   f"  void (*p[{len(names)}])(void);\n{body}\n"
                   '  printf("%d\\n", (int)(sizeof(p) / sizeof(p[0])));\n  return 0;\n}\n')
    out = tmp_path / "abi_check"
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-pedantic", "-I",
                    str(v3dm_mod.HEADER_PATH.parent), str(src), "-o", str(out), "-L", str(v3dm_mod.LIB_PATH.parent),
                    "-lv3dm", f"-Wl,-rpath,{v3dm_mod.LIB_PATH.parent}"], check=True, capture_output=True, text=True)
    r = subprocess.run([str(out)], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0 and int(r.stdout) == len(names)


def test_misaligned_device_buffers_are_rejected(v3dm_mod):
    """Device buffers that the kernels access as vectors must be aligned for them; a misaligned
    one is an argument error before any device work (checked here without a GPU; the tree's
    device calls are checked in tests/test_gpu_voctree.py)."""
    import ctypes as C
    lib = v3dm_mod.lib()
    fn = lib.v3dm_putative_u8_noalloc
    fn.argtypes = [C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_float, C.c_float, C.c_void_p,
                   C.c_void_p, C.c_void_p]
    ok, odd4, odd8 = 4096, 4096 + 2, 4096 + 4  # fake device addresses: aligned, off by 2, 4-aligned only
    for left, right, pairs, count in ((odd4, ok, ok, ok), (ok, odd4, ok, ok), (ok, ok, odd8, ok), (ok, ok, ok, odd4)):
        st = fn(0, C.c_void_p(left), 10, C.c_void_p(right), 10, 0.7, 0.8, C.c_void_p(pairs), C.c_void_p(count), None)
        assert st == v3dm_mod.ERR_ARG, (left, right, pairs, count)
    q = lib.v3dm_quantize_u8_device
    q.argtypes = [C.c_void_p, C.c_longlong, C.c_void_p, C.c_void_p]
    assert q(C.c_void_p(odd8), 8, C.c_void_p(ok), None) == v3dm_mod.ERR_ARG      # floats read as float4
    assert q(C.c_void_p(ok), 8, C.c_void_p(odd4), None) == v3dm_mod.ERR_ARG      # bytes written as uchar4
