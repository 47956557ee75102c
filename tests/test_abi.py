"""The C-ABI library loads and exports every symbol include/p6cuda.h declares
(no compute calls: this runs without a GPU)."""
import re
from pathlib import Path

import pytest

from powder6_b200 import _lib

HEADER = Path(__file__).resolve().parent.parent / 'include' / 'p6cuda.h'


def declared():
    text = HEADER.read_text()
    text = re.sub(r'/\*.*?\*/', '', text, flags=re.S)
    return sorted(set(re.findall(r'\b(p6_[a-z0-9_]+)\s*\(', text)))


def test_header_declares_the_entry_points():
    names = declared()
    for must in ('p6_wy_create', 'p6_wy_dispatch', 'p6_wy_read_state', 'p6_wy_sync_state', 'p6_wy_run',
                 'p6_last_error'):
        assert must in names


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing
    assert lib.p6_abi_version() >= 1


def test_bindings_cover_the_header():
    assert sorted(_lib.declared_symbols()) == declared() or set(declared()) <= set(_lib.declared_symbols())


def test_host_side_fault_injection_and_argument_errors():
    lib = _lib.load()
    with pytest.raises(_lib.P6Error) as e:
        _lib.check(lib.p6_wy_destroy(None))
    assert e.value.status == 'INVALID_ARG'
    lib.p6_debug_inject_failure(3, 0)
    with pytest.raises(_lib.P6Error) as e:
        _lib.check(lib.p6_wy_set_params(None, 1, 1.0))
    assert e.value.status == 'DEVICE_LOST' and 'injected' in str(e.value)
    lib.p6_debug_inject_failure(0, 0)
