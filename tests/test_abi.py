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
