"""The C-ABI library loads and exports every function declared in include/*.h, and the
product package never reaches into the oracle (no GPU needed)."""

import ctypes
import glob
import os
import re

from tests.conftest import ROOT


FIBRES_HEADER = "fibres.h"  # declarations of libfibres.so; every other header: the solver library


def declared_functions(headers=None):
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        base = os.path.basename(h)
        if headers is None and base == FIBRES_HEADER:
            continue
        if headers is not None and base not in headers:
            continue
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b([A-Za-z_]\w*)\s*\(",
                             text, flags=re.M):
            if m.group(1) not in {"if", "while", "for", "return", "sizeof"}:
                names.add(m.group(1))
    return names


def test_header_declares_reference_entry_point():
    names = declared_functions()
    assert "lippmann_schwinger_solve" in names
    assert {"lsb_create", "lsb_solve", "lsb_destroy", "lsb_c_eff"} <= names


def test_library_exports_every_declared_symbol(built_library):
    lib = ctypes.CDLL(built_library)
    missing = [n for n in sorted(declared_functions()) if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_every_symbol(built_library):
    from jaxmaterials_b200 import _lib

    lib = _lib.load()
    assert set(_lib.SIGNATURES) == declared_functions()
    assert lib.lsb_version() >= 1


def test_fibres_library_exports_and_binding(built_library):
    from jaxmaterials_b200 import _lib

    names = declared_functions({FIBRES_HEADER})
    assert {"dist_periodic", "initialise_rng", "move_fibres"} <= names
    lib = _lib.load_fibres()
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing
    assert set(_lib.FIBRES_SIGNATURES) == names


def test_product_does_not_import_oracle():
    pkg = os.path.join(ROOT, "jaxmaterials_b200")
    for path in glob.glob(os.path.join(pkg, "**", "*.py"), recursive=True):
        src = open(path).read()
        assert not re.search(r"^\s*(from|import)\s+oracle", src, flags=re.M), path
