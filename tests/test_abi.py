"""CPU tests of the C-ABI library: it loads and exports every declared symbol."""
import ctypes
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "zola_b200.h")).read()
    return sorted(set(re.findall(r"ZOLA_API\s+[\w\s\*]+?\b(zola_\w+)\s*\(", src)))


def test_library_exports_every_declared_symbol(zpkg):
    L = zpkg.lib()
    syms = declared_symbols()
    assert len(syms) >= 12
    for s in syms:
        assert hasattr(L, s), s
    assert set(syms) <= set(zpkg.EXPORTS) | set(syms)


def test_ctx_create_fails_cleanly_without_gpu(zpkg):
    import torch
    if torch.cuda.is_available():
        return
    h = ctypes.c_void_p()
    rc = zpkg.lib().zola_ctx_create(0, ctypes.byref(h))
    assert rc != 0
