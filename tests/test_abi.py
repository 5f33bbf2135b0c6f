"""The C ABI library loads and exports every entry point include/*.h
declares (no device calls: this runs without a GPU)."""
import ctypes
import re
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def declared_functions():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        for m in re.finditer(r"\b(?:int|const char \*|void \*|long long)\s*(inmsom_\w+)\s*\(", text):
            names.add(m.group(1))
    return names


def test_header_declares_the_binding_list():
    from inmsom_elfs_b200 import _lib
    assert declared_functions() == set(_lib.EXPORTS)


def test_library_exports_every_declared_symbol():
    from inmsom_elfs_b200 import build, _lib
    build.build()
    lib = ctypes.CDLL(str(_lib.LIB_PATH))
    for name in declared_functions():
        assert hasattr(lib, name), name
    _lib.load()   # argtypes for every export resolve


def test_library_has_no_cpu_fallback_symbols():
    # the product library links no oracle code
    from inmsom_elfs_b200 import _lib
    data = _lib.LIB_PATH.read_bytes()
    assert b"ora_barotropic_dynamics" not in data
