"""CPU: the C-ABI library loads, exports every function include/b200signal.h declares, and the
ctypes signature table matches the header (no device calls)."""

import re
from pathlib import Path

import pytest

from mlx_signal_b200 import _lib

HEADER = Path(__file__).resolve().parents[1] / "include" / "b200signal.h"


def declared_functions():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"SP_API\s+[\w\s\*]+?\b(sp_\w+)\s*\(", text)))


def test_header_declares_functions():
    names = declared_functions()
    assert "sp_welch_f32" in names and "sp_last_error" in names


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, f"symbols declared in the header but not exported: {missing}"


def test_signature_table_matches_header():
    assert sorted(_lib.SIGNATURES) == declared_functions()


def test_version_and_error_text_without_device():
    lib = _lib.load()
    assert lib.sp_version() == 100
    assert isinstance(lib.sp_last_error(), bytes)


@pytest.mark.parametrize(
    "args",
    [
        (0, 1, 100, 0, 64, 32, 1),   # nperseg < 1
        (0, 1, 100, 128, 128, 64, 1),  # nperseg > n
        (0, 1, 1000, 128, 64, 64, 1),  # nfft < nperseg
        (0, 1, 1000, 128, 128, 0, 1),  # hop < 1
        (0, 1, 1000, 128, 128, 64, 7),  # bad detrend
    ],
)
def test_workspace_query_rejects_bad_arguments(args):
    lib = _lib.load()
    assert lib.sp_mean_workspace_size(*args) == _lib.SP_ERR_ARG
    assert "invalid" in _lib.last_error()


def test_workspace_query_rejects_non_pow2_nfft():
    lib = _lib.load()
    assert lib.sp_mean_workspace_size(0, 1, 1000, 100, 100, 50, 1) == _lib.SP_ERR_UNSUPPORTED
