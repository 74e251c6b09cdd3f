"""The C-ABI library loads on any host and exports every declared entry point.

No compute calls: these run without a GPU.
"""
import ctypes
import glob
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADERS = sorted(glob.glob(os.path.join(ROOT, "include", "*.h")))


def declared(headers=HEADERS):
    src = "".join(open(h).read() for h in headers)
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(ipie_b200_\w+)\s*\(", src)))


@pytest.fixture(scope="module")
def lib():
    from ipie_b200 import build

    path = build.build()
    return ctypes.CDLL(path)


def test_header_declares_entry_points():
    names = declared()
    assert "ipie_b200_greens_function_single_det_batch" in names
    assert len(names) >= 15


def test_product_header_holds_no_testing_entries():
    product = declared([os.path.join(ROOT, "include", "ipie_b200.h")])
    assert not [n for n in product if n.endswith("_test")]


def test_library_exports_every_declared_symbol(lib):
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing


def test_ctypes_signatures_cover_the_header():
    from ipie_b200._lib import SIGNATURES

    names = set(declared()) - {"ipie_b200_version", "ipie_b200_launch_count"}
    assert names == set(SIGNATURES), sorted(names ^ set(SIGNATURES))


def test_version_and_host_only_queries(lib):
    lib.ipie_b200_version.restype = ctypes.c_char_p
    assert b"sm_100a" in lib.ipie_b200_version()
    # workspace query: rows of exchange partials (no device work)
    rows = lib.ipie_b200_exchange_rows(2048, 1600, 200, 32)
    assert rows == 400  # 4 Cholesky vectors of 32 occupied rows per 128-row tile
    assert lib.ipie_b200_exchange_rows(64, 120, 26, 5) == 8  # 16 vectors per tile (8-row blocks)
    assert lib.ipie_b200_exchange_rows(8, 10, 10, 33) == -1  # more than 32 electrons per spin: rejected


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    import ipie_b200._lib as L

    monkeypatch.setattr(L, "LIB_PATH", str(tmp_path / "nope.so"))
    monkeypatch.setattr(L, "_lib", None)
    with pytest.raises(L.CudaLibError):
        L.lib()
