"""The C ABI library loads on CPU and exports every symbol include/bem_b200.h declares."""
import ctypes
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    src = open(os.path.join(ROOT, "include", "bem_b200.h")).read()
    return sorted(set(re.findall(r"^\s*(?:int|int64_t|const char\*)\s+(bem_\w+)\s*\(", src, re.M)))


def test_header_and_library_agree():
    from bem_b200 import _lib
    names = _declared()
    assert names, "no declarations parsed"
    assert sorted(_lib.EXPORTS) == names
    lib = ctypes.CDLL(_lib.LIB_PATH)
    for n in names:
        assert hasattr(lib, n), n


def test_library_is_sm100a():
    from bem_b200 import _lib
    assert os.path.getsize(_lib.LIB_PATH) > 0
