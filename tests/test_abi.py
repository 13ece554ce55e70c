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


def test_job_struct_layout_matches_header(tmp_path):
    """fastpoly_b200.Job (ctypes) has the layout of struct fpx_job in include/fpx_b200.h."""
    import shutil
    import subprocess
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    fields = [f for f, _ in F.Job._fields_]
    src = tmp_path / "layout.c"
    src.write_text("#include <stdio.h>\n#include <stddef.h>\n#include \"fpx_b200.h\"\nint main(void) {\n"
                   "  printf(\"%zu\\n\", sizeof(fpx_job));\n"
                   + "".join(f"  printf(\"%zu\\n\", offsetof(fpx_job, {f}));\n" for f in fields)
                   + "  return 0;\n}\n")
    exe = tmp_path / "layout"
    subprocess.run([cc, "-I" + os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()]
    assert got[0] == ctypes.sizeof(F.Job)
    assert got[1:] == [getattr(F.Job, f).offset for f in fields]


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
