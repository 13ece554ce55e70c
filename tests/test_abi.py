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
    ctx._L = F.load_library()  # no GPU: page-locked memory is refused, ordinary buffers kept instead
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


def _records_in_python(jobs):
    """The job records Context.batch builds, restated in Python: (op, p, la, lb,
    k, n, cap1, cap2) per job."""
    import numpy as np
    rows = []
    for jb in jobs:
        op, p = F._OPS[jb[0]], int(jb[1])
        na = np.asarray(jb[2]).size
        nb = np.asarray(jb[3]).size if op in (F.OP_CONV, F.OP_DIVMOD) else 0
        k, n, cap2 = 0, 0, 0
        if op == F.OP_CONV:
            n = F.SIZE_MAX if len(jb) < 5 or jb[4] is None else int(jb[4])
            cap = min(na, n) + min(nb, n) - 1 if na and nb and n else 0
            cap1 = max(min(cap, n), 1)
        elif op == F.OP_POW:
            k, n = int(jb[3]), int(jb[4])
            cap1 = max(n, 1)
        elif op == F.OP_DIVMOD:
            cap1, cap2 = max(na, 1), max(nb, 1)
        else:
            n = int(jb[3])
            cap1 = max(n, 1)
        rows.append((op, p, na, nb, k, n, cap1, cap2))
    return rows


def test_batch_records_from_job_tuples():
    """The C helper behind Context.batch writes the records the job tuples
    describe, for every operation, argument form and array kind (uint32,
    other dtypes, lists, read-only and non-contiguous arrays, empty operands)."""
    import numpy as np
    rng = np.random.default_rng(3)
    a = rng.integers(0, 97, 50, dtype=np.uint32)
    ro = a.copy()
    ro.setflags(write=False)
    jobs = [("conv", 97, a, a), ("conv", 97, a, a[:7], None), ("conv", 97, a, a, 30), ("conv", 97, a, [], None),
            ("conv", 97, [1, 2, 3], a.astype(np.int64), 0), ("conv", 97, a[::2], ro),
            ("inv", 998244353, a, 100), ("log", 998244353, ro, np.int64(9)), ("exp", 7340033, [0, 1], 5),
            ("sqrt", 97, a.astype(np.int32), 3), ("pow", 97, a, (1 << 64) - 1, 40), ("pow", 97, a, 0, 0),
            ("divmod", 97, a, a[:9]), ("divmod", 97, a[:3], a), ("inv", np.uint32(97), np.zeros(0, np.uint32), 4)]
    m = len(jobs)
    arr = np.zeros(m, dtype=F._JOB_DTYPE)
    caps = np.empty(2 * m, np.int64)
    keep = F._jobs_ext().fill(jobs, arr.ctypes.data, caps.ctypes.data, F._OPS, F._arr)
    want = _records_in_python(jobs)
    for i, (op, p, la, lb, k, n, c1, c2) in enumerate(want):
        r = arr[i]
        assert (int(r["op"]), int(r["p"]), int(r["la"]), int(r["lb"]), int(r["k"]), int(r["n"])) == \
            (op, p, la, lb, k, n), (i, jobs[i][0])
        assert (int(caps[i]), int(caps[m + i])) == (c1, c2), i
        assert (int(r["a"]) == 0) == (la == 0) and (int(r["b"]) == 0) == (lb == 0), i
    # uint32 C-contiguous inputs are read in place, everything else converted (and kept)
    assert int(arr[0]["a"]) == a.ctypes.data and int(arr[7]["a"]) == ro.ctypes.data
    assert len(keep) == 6 and all(k.dtype == np.uint32 and k.flags.c_contiguous for k in keep)
    for bad, exc in [(("conv", 97, a), ValueError), (("nope", 97, a, 1), KeyError), (("inv", -1, a, 4), OverflowError),
                     (("inv", 1 << 32, a, 4), OverflowError), (("pow", 97, a, 3), ValueError)]:
        with pytest.raises(exc):
            F._jobs_ext().fill([bad], arr.ctypes.data, caps.ctypes.data, F._OPS, F._arr)


def test_host_alloc_arguments_without_gpu():
    """fpx_host_alloc / fpx_host_free reject bad arguments; without a GPU the
    page-locked allocation itself is refused (no host fallback is made up)."""
    lib = F.load_library()
    p = ctypes.c_void_p(123)
    assert lib.fpx_host_alloc(0, ctypes.byref(p)) == F.EINVAL and not p.value
    assert lib.fpx_host_alloc(16, None) == F.EINVAL
    assert lib.fpx_host_free(None) == F.EINVAL
    try:
        import torch
        if torch.cuda.is_available():
            return  # with a GPU the allocation is made (the batch tests use it)
    except ImportError:
        pass
    assert lib.fpx_host_alloc(1 << 20, ctypes.byref(p)) == F.ENOMEM and not p.value
