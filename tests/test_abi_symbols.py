"""The C-ABI library loads on a CPU-only host and exports every entry point include/pe_b200.h declares
(no compute call is made here)."""
import ctypes
import os
import re

from conftest import ROOT
from photonic_engines_b200 import _native as N


def _declared():
    src = open(os.path.join(ROOT, "include", "pe_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(pe_[a-z0-9_]+)\s*\(", src)))


def test_header_declarations_are_exported():
    lib = ctypes.CDLL(N.LIB_PATH)
    names = _declared()
    assert names, "no declarations parsed"
    for name in names:
        assert hasattr(lib, name), f"{name} declared in pe_b200.h but not exported"
    assert set(names) == set(N.EXPORTED)


def test_loader_sets_signatures_and_version():
    L = N.load()
    assert L.pe_version() >= 100
    assert L.pe_chain_workspace_bytes(1000) >= 64
    assert L.pe_status_string(-2).decode().startswith("size")
    assert L.pe_last_cuda_error().decode() == "no CUDA error recorded"     # no CUDA call has failed
