"""CPU-side checks of the drop-in boundary: the C-ABI library loads, exports every
symbol include/*.h declares, and fails loudly (no CPU fallback) without a GPU."""
import ctypes
import glob
import os
import re

import pytest

import fastpoly_b200 as F
from conftest import ROOT


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names.update(re.findall(r"\b(fpx_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(F.LIB_PATH)
    names = declared_symbols()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_ntt_max_log_without_device():
    assert F.ntt_max_log(998244353) == 23
    assert F.ntt_max_log(167772161) == 25
    assert F.ntt_max_log(469762049) == 26
    assert F.ntt_max_log(754974721) == 24
    assert F.ntt_max_log(1000000007) == 1


def test_context_fails_loudly_without_gpu():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    with pytest.raises(F.FpxError) as e:
        F.Context(0)
    assert e.value.code == F.EUNSUPPORTED


def test_null_context_rejected():
    lib = F.load_library()
    assert lib.fpx_ctx_destroy(None) == F.EINVAL
    assert lib.fpx_conv(None, 998244353, None, 0, None, 0, 0, None, None, 0) == F.EINVAL


@pytest.mark.parametrize("cls,ctype", [("Job", "fpx_job"), ("ServeConfig", "fpx_serve_config"),
                                       ("ServeStats", "fpx_serve_stats"), ("PoolStats", "fpx_pool_stats_t"),
                                       ("ColShape", "fpx_col_shape")])
def test_struct_layout_matches_header(tmp_path, cls, ctype):
    """Each ctypes structure of fastpoly_b200 has the layout of its struct in include/fpx_b200.h."""
    import shutil
    import subprocess
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    S = getattr(F, cls)
    fields = [f for f, _ in S._fields_]
    src = tmp_path / "layout.c"
    src.write_text("#include <stdio.h>\n#include <stddef.h>\n#include \"fpx_b200.h\"\nint main(void) {\n"
                   f"  printf(\"%zu\\n\", sizeof({ctype}));\n"
                   + "".join(f"  printf(\"%zu\\n\", offsetof({ctype}, {f}));\n" for f in fields)
                   + "  return 0;\n}\n")
    exe = tmp_path / "layout"
    subprocess.run([cc, "-I" + os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()]
    assert got[0] == ctypes.sizeof(S)
    assert got[1:] == [getattr(S, f).offset for f in fields]


def test_batch_output_buffer_reuse():
    """Context.batch hands a large output buffer out again only once no result
    view of the call that had it is alive."""
    import numpy as np
    ctx = F.Context.__new__(F.Context)  # the buffer logic needs no device
    ctx._outbufs = []
    words = 3 << 20
    first = ctx._out_buffer(words)
    result = first[5:10]
    result[:] = 7
    del first
    second = ctx._out_buffer(words)
    assert not np.shares_memory(second, result), "a buffer with a live result was handed out again"
    assert (result == 7).all()
    addr = second.__array_interface__["data"][0]
    del second
    third = ctx._out_buffer(words - 100)
    assert third.__array_interface__["data"][0] == addr
    del third
    larger = ctx._out_buffer(2 * words)  # fits no kept buffer: a new one
    assert larger.size == 2 * words and not np.shares_memory(larger, result)
    assert len(ctx._outbufs) <= 2
    small = ctx._out_buffer(100)
    assert small.size == 100 and all(b.size >= F._OUT_KEEP_WORDS for b in ctx._outbufs)


def test_batch_rejects_null_context():
    lib = F.load_library()
    assert lib.fpx_batch_run(None, None, 0, 0) == F.EINVAL
    assert lib.fpx_batch_submit(None, None, 0) == F.EINVAL


def test_serve_plan_bytes_without_device():
    """The admission measure needs no GPU: native products plan two N-word
    buffers, CRT products three primes' worth plus their residues."""
    import numpy as np
    keep = []
    a = np.ones(1 << 16, np.uint32)
    native, _, _ = F.make_job(("conv", 998244353, a, a), keep)
    crt, _, _ = F.make_job(("conv", 1000000007, a, a), keep)
    lib = F.load_library()
    nb = lib.fpx_serve_plan_bytes(ctypes.byref(native))
    cb = lib.fpx_serve_plan_bytes(ctypes.byref(crt))
    N = 1 << 17
    assert nb >= 4 * (2 * N) and nb < 4 * (6 * N)
    assert cb > 2.5 * nb
    assert lib.fpx_serve_plan_bytes(None) == 0
