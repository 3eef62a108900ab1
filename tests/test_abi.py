"""CPU checks of the C ABI: the library loads, exports every declared entry
point, and rejects bad arguments before touching a device."""
import ctypes
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


@pytest.fixture(scope="module")
def lib():
    from nsrno_b200 import _lib, build
    build.build()
    return _lib.load()


def declared_symbols():
    names = set()
    for header in (ROOT / "include").glob("*.h"):
        text = header.read_text()
        names.update(re.findall(r"^\s*(?:[\w\*\s]+?)\b(nsr_\w+)\s*\(", text, flags=re.M))
    return sorted(names)


def test_every_declared_symbol_is_exported(lib):
    names = declared_symbols()
    assert "nsr_solve_batched" in names and len(names) >= 10
    for name in names:
        assert hasattr(lib, name), name


def test_binding_lists_every_declared_symbol():
    from nsrno_b200 import _lib
    assert set(declared_symbols()) <= set(_lib.EXPORTS)


def test_version_and_error_strings(lib):
    from nsrno_b200 import _lib
    assert lib.nsr_version() >= 100
    assert b"invalid argument" in lib.nsr_error_string(1001)
    assert b"prime factor" in lib.nsr_error_string(1002)
    with pytest.raises(RuntimeError, match="workspace"):
        _lib.check(1003)
    assert _lib.check(0) == 0


def grid(nz=768, nx=1024, **kw):
    from nsrno_b200 import _lib
    g = dict(nz=nz, nx=nx, n_pml=24, face=28, h=5e-5, c0=1500.0, rho0=1000.0, pml_strength=12.0,
             alpha_power=1.1, aperture_half_width=0.0192)
    g.update(kw)
    return _lib.NsrGrid(**g)


def test_argument_errors_need_no_device(lib):
    null = ctypes.c_void_p(0)
    bad = grid(nz=2)
    assert lib.nsr_setup_material(ctypes.byref(bad), null, null, null, null, null) == 1001
    good = grid()
    assert lib.nsr_setup_material(ctypes.byref(good), null, null, null, null, null) == 1001
    assert lib.nsr_apply(ctypes.byref(good), null, null, 1, 0, 0, null, null, null) == 1001
    assert lib.nsr_grad_accum(ctypes.byref(good), null, null, 1, 0, null, null, null, null, null) == 1001


def test_workspace_queries(lib):
    g = grid()
    n = 768 * 1024
    ws = lib.nsr_solve_workspace_size(ctypes.byref(g), 16)
    # seven complex64 vectors, the learned multiplier plane and two complex128
    # iterates per slot, plus tables
    assert ws >= 16 * n * (8 * 8 + 2 * 16)
    assert ws < 16 * n * (8 * 8 + 2 * 16) + (1 << 22)
    assert lib.nsr_solve_workspace_size(ctypes.byref(grid(nz=2 * 67)), 4) == 0   # prime factor 67 > 61
    assert lib.nsr_solve_workspace_size(ctypes.byref(grid(nz=7 * 16)), 4) > 0    # 112 = 7 * 2^4
    assert lib.nsr_solve_workspace_size(ctypes.byref(g), 0) == 0
    assert lib.nsr_precondition_workspace_size(ctypes.byref(g), 2) >= 2 * n * 8
    assert lib.nsr_precondition_workspace_size(ctypes.byref(grid(nx=4096)), 1) == 0


def test_header_is_plain_c(tmp_path):
    """include/nsrno_b200.h is a C99 header (no C++ or torch types at the boundary)."""
    import shutil
    import subprocess
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    src = tmp_path / "probe.c"
    src.write_text('#include "nsrno_b200.h"\nint main(void) { NsrSolveParams p; NsrLearned l; NsrGrid g;'
                   ' (void)p; (void)l; (void)g; return 0; }\n')
    subprocess.run([cc, "-std=c99", "-Wall", "-Werror", f"-I{ROOT / 'include'}", "-fsyntax-only", str(src)],
                   check=True)


def test_ctypes_structs_match_the_header(tmp_path):
    """The ctypes mirrors have the C layout: size and every field offset."""
    import shutil
    import subprocess
    from nsrno_b200 import _lib
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    structs = {"NsrGrid": _lib.NsrGrid, "NsrLearned": _lib.NsrLearned, "NsrTiles": _lib.NsrTiles,
               "NsrSolveParams": _lib.NsrSolveParams, "NsrGmresParams": _lib.NsrGmresParams,
               "NsrSolveStats": _lib.NsrSolveStats, "NsrDenseGrid": _lib.NsrDenseGrid,
               "NsrDenseSolveParams": _lib.NsrDenseSolveParams, "NsrDenseSolveInfo": _lib.NsrDenseSolveInfo}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "nsrno_b200.h"', 'int main(void) {']
    for name, cls in structs.items():
        lines.append(f'  printf("{name} size %zu\\n", sizeof({name}));')
        for field, _ in cls._fields_:
            lines.append(f'  printf("{name} {field} %zu\\n", offsetof({name}, {field}));')
    lines += ['  return 0;', '}']
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run([cc, "-std=c99", f"-I{ROOT / 'include'}", str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    for line in filter(None, out):
        name, field, value = line.split()
        cls = structs[name]
        got = ctypes.sizeof(cls) if field == "size" else getattr(cls, field).offset
        assert got == int(value), (name, field, got, value)
