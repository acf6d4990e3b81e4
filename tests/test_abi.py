"""The C-ABI library loads and exports every entry point that include/*.h declares
(no compute call: this runs without a GPU)."""
import glob
import os
import re

from conftest import ROOT


def declared_functions():
    names = set()
    for hdr in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(hdr).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(dgpu_[a-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    return names


def test_header_declares_entry_points():
    names = declared_functions()
    assert "dgpu_wavelet_transform" in names
    assert len(names) >= 7


def test_library_exports_every_declared_symbol():
    import dirac_b200

    lib = dirac_b200.load()
    missing = [n for n in sorted(declared_functions()) if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_header():
    from dirac_b200 import _lib

    assert declared_functions() <= set(_lib.SIGNATURES), declared_functions() - set(_lib.SIGNATURES)


def test_version_string_without_gpu():
    import dirac_b200

    assert b"sm_100a" in dirac_b200.load().dgpu_version()
