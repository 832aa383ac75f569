"""The C-ABI library loads without a GPU and exports every entry point include/*.h declares."""

import ctypes
import re
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def declared_symbols():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names |= set(re.findall(r"\b(zvfv_\w+)\s*\(", text))
    return names


def test_library_exports_every_declared_symbol():
    from zvcfd_b200 import _lib

    names = declared_symbols()
    assert len(names) > 25
    lib = ctypes.CDLL(str(_lib.LIB_PATH))
    for n in sorted(names):
        assert hasattr(lib, n), n
    # the ctypes binding declares exactly the header's entry points
    assert set(_lib.declared()) == names


def test_library_reports_errors_without_a_gpu():
    from zvcfd_b200 import _lib

    assert _lib.lib.zvfv_version() >= 1
    assert _lib.lib.zvfv_record_doubles(3) == 368          # hex: 2*24*3 + 24*9 + 8
    assert _lib.lib.zvfv_record_doubles(0) == 85            # tet: 2*12*3 + 9 + 4 (one Jacobian)
    # argument checks run before any CUDA call
    rc = _lib.lib.zvfv_gradient(10, 5, 0, None, None, None, None, None, None, None)
    assert rc == 1 and b"nc" in _lib.lib.zvfv_last_error()


def test_tables_header_is_current():
    from zvcfd_b200.topology import HEADER_PATH, header_source

    assert HEADER_PATH.read_text() == header_source()


def _prototypes():
    """``{name: [parameter type strings]}`` of every prototype in ``include/*.h``."""
    out = {}
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        text = re.sub(r"//[^\n]*", "", text)
        for m in re.finditer(r"\b(zvfv_\w+)\s*\(([^;{]*?)\)\s*;", text):
            params = [p.strip() for p in m.group(2).split(",")]
            out[m.group(1)] = [] if params in ([""], ["void"]) else params
    return out


def test_ctypes_signatures_match_the_header():
    """Each entry point's ctypes argument list has the header's parameter count, and each
    parameter's kind agrees: a pointer for ``*`` parameters, a double for ``double``, a 64-bit
    integer for ``int64_t``, a 32-bit one for ``int``."""
    import ctypes as C

    from zvcfd_b200._lib import _SIGNATURES

    protos = _prototypes()
    assert set(protos) == set(_SIGNATURES)
    for name, params in protos.items():
        args = _SIGNATURES[name][0]
        assert len(args) == len(params), (name, len(args), len(params))
        for a, p in zip(args, params):
            if "*" in p:
                assert a in (C.c_void_p, C.c_char_p) or a.__name__.startswith("LP_"), (name, p)
            elif p.startswith("double"):
                assert a is C.c_double, (name, p)
            elif p.startswith("int64_t"):
                assert a is C.c_int64, (name, p)
            elif p.startswith("int"):
                assert a is C.c_int, (name, p)
