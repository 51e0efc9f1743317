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


def test_build_targets_sm100a_only():
    """The library's only device target is sm_100a (the Makefile's -gencode);
    the GPU side of this check is tests/test_linalg_gpu.py's binary-version
    query."""
    mk = open(os.path.join(ROOT, "taichi-bem_b200", "Makefile")).read()
    arches = re.findall(r"arch=(compute_\w+),code=(sm_\w+)", mk)
    assert arches == [("compute_100a", "sm_100a")], arches


def test_every_entry_point_cites_what_it_replaces():
    """Each declaration's comment names the reference interface it replaces
    (file.py:line) or says it has no reference counterpart."""
    import re
    src = open(os.path.join(ROOT, "include", "bem_b200.h")).read()
    for m in re.finditer(r"^(?:int|int64_t|const char\*)\s+(bem_\w+)\(", src, re.M):
        before = src[:m.start()]
        comment = before[before.rfind("/*"):before.rfind("*/")]
        text = " ".join(comment.replace("*", " ").split())
        assert re.search(r"\.py:\d+|:\d+-\d+|no reference counterpart", text, re.I), m.group(1)
