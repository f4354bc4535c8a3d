"""The C ABI libraries load and export every function their headers declare.

No GPU compute is called here; on a machine without a GPU the context
constructor must fail cleanly (no CPU fallback exists).
"""
from __future__ import annotations

import ctypes
import re

import numpy as np
import pytest

from conftest import ROOT

from spatialjoincountovershells_b200 import _native as nat

DECL = re.compile(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\**\s*\b(sjcs_\w+)\s*\(", re.M)


def declared(header: str):
    text = (ROOT / "include" / header).read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = set(DECL.findall(text))
    names = {n for n in names if not n.endswith("_t")}
    return names


@pytest.mark.parametrize("header,libfile", [("sjcs.h", "libsjcs.so"), ("sjcs_host.h", "libsjcs_host.so")])
def test_library_exports_every_declared_symbol(header, libfile, built):
    names = declared(header)
    assert len(names) > 10
    lib = ctypes.CDLL(str(ROOT / "spatialjoincountovershells_b200" / "lib" / libfile))
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, f"{libfile} lacks {missing}"


def test_python_bindings_cover_the_headers(built):
    assert declared("sjcs.h") == set(nat._SIGS)
    assert declared("sjcs_host.h") == set(nat._HOST_SIGS)


def test_radius_table_is_host_only(built):
    r2 = np.zeros(40, np.float32)
    assert nat.lib().sjcs_radius_table(5.0, 0.001, 40, r2.ctypes.data) == 0  # min > max is swapped
    assert np.array_equal(r2, nat.radius_table(0.001, 5.0, 40))
    assert nat.lib().sjcs_radius_table(1.0, 2.0, 0, r2.ctypes.data) == 1


def test_context_without_gpu_fails_cleanly(built):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(nat.SjcsError) as ei:
        nat.Context(0)
    assert ei.value.code == 2  # SJCS_ERR_CUDA
    assert "device" in ei.value.msg


def test_invalid_handles_are_rejected(built):
    L = nat.lib()
    assert L.sjcs_ctx_sync(None) == 4
    assert L.sjcs_index_destroy(None) == 4
    assert L.sjcs_query_destroy(None) == 4
    assert "invalid" in L.sjcs_last_error().decode()
