"""The C-ABI library builds, loads and exports every symbol its header declares (no GPU)."""
import ctypes
import re

import pytest

from conftest import ROOT

HEADER = ROOT / "include" / "treams_cuda.h"


def declared_symbols():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(tcu_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_the_hot_path():
    names = declared_symbols()
    for required in ("tcu_sphere_cluster_factor", "tcu_factor_solve", "tcu_iterative_solve",
                     "tcu_translation_block", "tcu_lsumsw2d_batch", "tcu_array_solve_batch"):
        assert required in names


def test_library_exports_every_declared_symbol():
    import treams_b200
    lib = ctypes.CDLL(str(treams_b200.library_path()))
    missing = [name for name in declared_symbols() if not hasattr(lib, name)]
    assert not missing, missing


def test_binding_signatures_cover_the_header():
    from treams_b200 import _lib
    assert set(declared_symbols()) <= set(_lib.SIGNATURES)


def test_context_creation_fails_loudly_without_a_b200():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    import treams_b200
    with pytest.raises(treams_b200.TreamsCudaError, match="no CPU path|no CUDA device"):
        treams_b200.Context(0)
