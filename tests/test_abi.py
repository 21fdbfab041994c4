"""The C-ABI library loads and exports every function include/*.h declares.
No compute call (no GPU needed)."""
import ctypes as ct
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADERS = ["midapack_b200.h", "mapmat.h", "toeplitz.h", "mappraiser.h"]


def declared(header):
    src = open(os.path.join(ROOT, "include", header)).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    src = re.sub(r"//.*", "", src)
    names = set()
    for mt in re.finditer(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\(", src):
        name = mt.group(1)
        if name in ("if", "for", "while", "return", "sizeof", "defined"):
            continue
        # a declaration: preceded by a type at statement start
        line_start = src.rfind("\n", 0, mt.start()) + 1
        prefix = src[line_start:mt.start()].strip()
        if re.match(r"^(const\s+)?[A-Za-z_][A-Za-z0-9_ ]*\**$", prefix) and not prefix.startswith("#"):
            names.add(name)
    return names


@pytest.mark.parametrize("header", HEADERS)
def test_exports(header):
    import midapack_b200 as mb
    L = ct.CDLL(mb.LIB_PATH)
    names = declared(header)
    assert names, header
    missing = [n for n in sorted(names) if not hasattr(L, n)]
    assert not missing, missing


def test_python_binding_covers_headers():
    import midapack_b200 as mb
    allnames = set()
    for h in HEADERS:
        allnames |= declared(h)
    assert allnames <= set(mb._SIGS), sorted(allnames - set(mb._SIGS))
