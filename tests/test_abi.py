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


def test_ctypes_structures_match_the_header(zpkg, tmp_path):
    """The Python mirror's ctypes structures have the sizes and field offsets
    that a C compiler gives the header's structs (gcc on include/zola_b200.h)."""
    import shutil
    import subprocess
    if shutil.which("gcc") is None:
        return
    pairs = [("zola_optics", zpkg.Optics), ("zola_localization", zpkg.Localization),
             ("zola_loc_params", zpkg.LocParams), ("zola_fit_params", zpkg.FitParams),
             ("zola_fit_class", zpkg.FitClass), ("zola_drift_params", zpkg.DriftParams),
             ("zola_calib_data", zpkg.CalibData)]
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "zola_b200.h"', "int main(void) {"]
    for cname, cls in pairs:
        lines.append(f'    printf("{cname} size %zu\\n", sizeof({cname}));')
        for f in cls._fields_:
            lines.append(f'    printf("{cname} {f[0]} %zu\\n", offsetof({cname}, {f[0]}));')
    lines += ["    return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.check_call(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)])
    got = {}
    for ln in subprocess.check_output([str(exe)], text=True).splitlines():
        cname, key, val = ln.split()
        got[(cname, key)] = int(val)
    for cname, cls in pairs:
        assert got[(cname, "size")] == ctypes.sizeof(cls), cname
        for f in cls._fields_:
            assert got[(cname, f[0])] == getattr(cls, f[0]).offset, (cname, f[0])


def declared_arity():
    """{name: parameter count} of every ZOLA_API function in the header."""
    src = open(os.path.join(ROOT, "include", "zola_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    out = {}
    for m in re.finditer(r"ZOLA_API\s+[\w\s\*]+?\b(zola_\w+)\s*\(([^;]*?)\)\s*;", src, flags=re.S):
        params = m.group(2).strip()
        out[m.group(1)] = 0 if params in ("", "void") else params.count(",") + 1
    return out


def test_python_argtypes_match_the_header(zpkg):
    """Every function the Python mirror binds with argtypes takes as many
    arguments as the header declares (a mismatch would corrupt the call)."""
    L = zpkg.lib()
    arity = declared_arity()
    checked = 0
    for name, n in arity.items():
        fn = getattr(L, name)
        if fn.argtypes is None:
            continue
        assert len(fn.argtypes) == n, (name, len(fn.argtypes), n)
        checked += 1
    assert checked >= 20


def test_wide_return_types_are_declared(zpkg):
    """Functions that return a pointer or a 64-bit integer have a restype that
    keeps all 64 bits (ctypes would otherwise truncate them to a C int)."""
    src = open(os.path.join(ROOT, "include", "zola_b200.h")).read()
    L = zpkg.lib()
    wide = re.findall(r"ZOLA_API\s+(?!int\s)([\w\s]+?\*?)\s*\b(zola_\w+)\s*\(", src)
    assert len(wide) >= 3
    for ret, name in wide:
        rt = getattr(L, name).restype
        assert rt is not None and ctypes.sizeof(rt) == 8, (name, ret, rt)
