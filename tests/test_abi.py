"""CPU checks of the C-ABI boundary: liblsb.so loads, exports every function
include/lsb.h declares, and rejects bad arguments before touching the GPU."""
from __future__ import annotations

import ctypes as C

import numpy as np

from lslab_b200 import _lib
from lslab_b200.build import LIB


def test_library_exports_every_declared_symbol():
    lib = C.CDLL(str(LIB))
    names = _lib.header_symbols()
    assert len(names) >= 29
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_header():
    assert set(_lib.header_symbols()) == set(_lib._SIGS)


def test_null_handles_and_pointers_are_rejected():
    L = _lib.lib()
    assert L.lsb_map_get(None, None, None, 4, None) == _lib.LSB_ERR_ARG
    assert L.lsb_map_put(None, None, None, None, 4, None) == _lib.LSB_ERR_ARG
    assert L.lsb_set_insert(None, None, None, 4, None) == _lib.LSB_ERR_ARG
    assert L.lsb_map_destroy(None) == _lib.LSB_ERR_ARG
    assert L.lsb_map_create(0, 0, None) == _lib.LSB_ERR_ARG
    assert L.lsb_map_buckets(None) == 0


def test_error_strings_and_version():
    L = _lib.lib()
    for code in range(6):
        assert L.lsb_error_string(code)
    assert L.lsb_version() >= 100


def test_result_layout_matches_pair_bool_u64():
    # cuda::std::pair<bool, uint64_t>: bool at byte 0, value at byte 8, 16 bytes
    from tests.util import RESULT_DTYPE
    assert RESULT_DTYPE.itemsize == 16
    assert RESULT_DTYPE.fields["value"][1] == 8
    opts = _lib.Options()
    assert C.sizeof(opts) == 24


def test_oracle_library_loads():
    import oracle
    m = oracle.OracleMap(2)
    m.put(np.array([5], np.uint64), np.array([6], np.uint64))
    assert m.get(np.array([5], np.uint64))["value"][0] == 6
