"""The C-ABI library loads and exports every symbol include/pyquante_b200.h
declares (no device needed)."""
import os
import re

from conftest import ROOT


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "pyquante_b200.h")).read()
    return sorted(set(re.findall(r"\b(pqb_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    from pyquante_b200 import _lib
    lib = _lib.load()
    syms = declared_symbols()
    assert len(syms) >= 16
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing
    # and the ctypes signature table covers them all
    assert sorted(_lib.SIGNATURES) == syms


def test_packed_index_is_64_bit_and_matches_reference_order():
    import pyq_oracle as O
    from pyquante_b200.Ints import ijkl2intindex
    for ijkl in [(0, 0, 0, 0), (3, 1, 2, 2), (1, 3, 2, 0), (6, 6, 6, 5), (50, 7, 49, 49)]:
        assert ijkl2intindex(*ijkl) == O.ijkl2intindex(*ijkl)
    # nbf = 308: the last index overflows a C int in Src/cints.c:413-425
    n = 308
    last = ijkl2intindex(n - 1, n - 1, n - 1, n - 1)
    P = n * (n + 1) // 2
    assert last == P * (P + 1) // 2 - 1 == 1132237490
    cints = O.ref_lib("cints")
    if cints is not None:
        assert cints.ref_cints_ijkl2intindex(6, 3, 5, 2) == ijkl2intindex(6, 3, 5, 2)
        assert cints.ref_cints_ijkl2intindex(n - 1, n - 1, n - 1, n - 1) != last   # the reference overflows


def test_engine_raises_without_device(monkeypatch):
    import pytest
    import torch
    from pyquante_b200 import _lib
    monkeypatch.setattr(torch.cuda, "is_available", lambda: False)
    with pytest.raises(_lib.EngineUnavailable):
        _lib.Context(0)
