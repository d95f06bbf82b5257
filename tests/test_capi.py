"""The C-ABI library loads and exports every entry point declared in include/*.h (no GPU)."""
import glob
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"\b(sod_[a-z0-9_]+)\s*\(", src):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared()
    assert "sod_rk4_main" in names and "sod_full_convec_ijk" in names and len(names) >= 20


def test_library_exports_declared_symbols():
    from sod2d_refmap_b200 import build, _lib
    build.build()
    _lib.load()
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True, check=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if ln.strip()}
    missing = [n for n in declared() if n not in exported]
    assert not missing, f"declared but not exported: {missing}"


def test_library_has_no_cpu_fallback_symbols():
    """The product library must not link the oracle."""
    from sod2d_refmap_b200 import _lib
    out = subprocess.run(["nm", "-D", _lib.LIB_PATH], capture_output=True, text=True, check=True).stdout
    assert "oracle_" not in out


def test_library_resolves_its_own_symbols():
    """No function of the library's own namespace is left undefined (a declaration in one source
    file that no longer matches its definition links and fails only at load time)."""
    from sod2d_refmap_b200 import _lib
    out = subprocess.run(["nm", "-C", "-u", _lib.LIB_PATH], capture_output=True, text=True, check=True).stdout
    assert not [ln for ln in out.splitlines() if "sod::" in ln]


def test_build_check_refuses_unresolved_internal_symbol(tmp_path):
    """build._check_resolved removes a library that references an undefined sod:: function."""
    from sod2d_refmap_b200 import build
    src = tmp_path / "bad.cpp"
    src.write_text("namespace sod { int missing(int); }\nextern \"C\" int entry(int x) { return sod::missing(x); }\n")
    lib = tmp_path / "libbad.so"
    subprocess.run(["g++", "-shared", "-fPIC", "-o", str(lib), str(src)], check=True)
    with pytest.raises(RuntimeError, match="undefined internal symbols"):
        build._check_resolved(str(lib))
    assert not lib.exists()
