"""CPU: the C-ABI library loads and exports every entry point declared in include/anechoic.h (no compute calls)."""
import os
import re

from tests.conftest import ROOT


def declared_symbols():
    txt = open(os.path.join(ROOT, "include", "anechoic.h")).read()
    return sorted(set(re.findall(r"ANC_API\s+[\w\s\*]*?\b(anc_\w+)\s*\(", txt)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    for s in ("anc_instance_create", "anc_tables_create", "anc_tables_from_schedule", "anc_run", "anc_run_batch",
              "anc_last_error"):
        assert s in syms


def test_library_exports_every_declared_symbol(lib):
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_python_binding_covers_exports(lib):
    from anechoic_b200 import _lib
    assert set(_lib.EXPORTS) <= set(declared_symbols())


def test_version_and_np(lib):
    assert lib.anc_version().startswith(b"anechoic-b200")
    assert lib.anc_np(1) == 2048 and lib.anc_np(2048) == 2048 and lib.anc_np(2049) == 2304
    assert lib.anc_spin_words(2000) == 32 and lib.anc_spin_words(20000) == 316
