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


def test_repeated_density_reuses_the_last_build(monkeypatch):
    """getJ(Ints, D) then getK(Ints, D) (the reference's call pattern) runs
    one J/K build, not two, and uhf's getJ(Da), getJ(Db), getK(Da), getK(Db)
    runs two.  A new density, an in-place change to the density or to the
    integrals, a new integral array, and changes a caller makes to returned
    arrays all behave as without the cache.  Host
    logic only: the build is replaced by a counting stand-in."""
    import numpy as np
    import torch
    from pyquante_b200 import Ints as I
    calls = []

    def fake_jk_packed(t, D):
        calls.append(1)
        s = float(t.sum())
        return D * 2.0 + s, D * 3.0 + s

    monkeypatch.setattr(I, "jk_packed", fake_jk_packed)
    ints = I.PackedInts(torch.ones(21, dtype=torch.float64), 5)
    rng = np.random.default_rng(0)
    Da = rng.standard_normal((5, 5))
    Db = rng.standard_normal((5, 5))
    J = I.getJ(ints, Da)
    K = I.getK(ints, Da)
    assert len(calls) == 1
    assert np.allclose(J, 2 * Da + 21) and np.allclose(K, 3 * Da + 21)
    J[:] = 0.0                                   # the caller's array, not the cache
    assert np.allclose(I.getJ(ints, Da), 2 * Da + 21) and len(calls) == 1
    assert np.allclose(I.get2JmK(ints, Da), 4 * Da + 42 - 3 * Da - 21) and len(calls) == 1
    I.getJ(ints, Db)
    I.getK(ints, Db)
    assert len(calls) == 2
    Db[0, 0] += 1.0                              # same array, new values
    assert np.allclose(I.getK(ints, Db), 3 * Db + 21) and len(calls) == 3
    ints.tensor.mul_(2.0)                        # the integrals changed in place
    assert np.allclose(I.getK(ints, Db), 3 * Db + 42) and len(calls) == 4
    Dt = torch.as_tensor(Da)
    Jt = I.getJ(ints, Dt)
    Jt.zero_()                                   # torch in, torch out: still a copy
    assert torch.allclose(I.getJ(ints, Dt), 2 * Dt + 42) and len(calls) == 5
    # uhf's order: J of alpha and beta, then K of alpha and beta -> two builds
    Da2, Db2 = Da + 1.0, Db + 1.0
    Ja, Jb, Ka, Kb = I.getJ(ints, Da2), I.getJ(ints, Db2), I.getK(ints, Da2), I.getK(ints, Db2)
    assert len(calls) == 7
    assert np.allclose(Ka, 3 * Da2 + 42) and np.allclose(Kb, 3 * Db2 + 42) and np.allclose(Jb, 2 * Db2 + 42)
    # a new integral array assigned to the same object: nothing remembered for the old one is served
    ints.tensor = torch.full((21,), 3.0, dtype=torch.float64)
    assert np.allclose(I.getK(ints, Db2), 3 * Db2 + 63) and len(calls) == 8


def test_get2jmk_of_a_host_density_on_direct_ints_is_one_host_call(monkeypatch):
    """get2JmK(DirectInts, D) with a host D (numpy in, numpy out; CPU tensor
    in, CPU tensor out) goes through the one host-array call, which fills G
    in place, and builds no J/K."""
    import numpy as np
    import torch

    import pyquante_b200.Ints as I
    calls = []
    d = object.__new__(I.DirectInts)
    d.nbf = 4

    def fake_host(D, G, stream=None):
        calls.append(type(D))
        G[...] = 2.0 * D + 1.0
        return G

    monkeypatch.setattr(d, "get2jmk_host", fake_host, raising=False)
    monkeypatch.setattr(d, "synchronize", lambda: None, raising=False)
    monkeypatch.setattr(I, "_jk", lambda *a, **k: (_ for _ in ()).throw(AssertionError("J/K path taken")))
    D = np.arange(16, dtype=np.float64).reshape(4, 4)
    G = I.get2JmK(d, D)
    assert isinstance(G, np.ndarray) and np.array_equal(G, 2.0 * D + 1.0)
    Gt = I.get2JmK(d, torch.as_tensor(D))
    assert isinstance(Gt, torch.Tensor) and not Gt.is_cuda and torch.equal(Gt, torch.as_tensor(2.0 * D + 1.0))
    assert calls == [np.ndarray, torch.Tensor]


def test_get2jmk_host_rejects_bad_arrays_before_the_call(monkeypatch):
    """BasisEngine.get2jmk_host checks shape, dtype and layout of both host
    arrays and raises before reaching the C entry point."""
    import numpy as np
    import pytest
    import torch

    from pyquante_b200.engine import BasisEngine
    eng = object.__new__(BasisEngine)
    eng.nbf = 3
    monkeypatch.setattr(eng, "_need_shells", lambda: None, raising=False)
    monkeypatch.setattr(eng, "plan", lambda *a, **k: None, raising=False)

    class NoCall:
        def __getattr__(self, name):
            raise AssertionError("C entry point reached")

    eng.ctx = NoCall()
    good = np.zeros((3, 3))
    for D, G in ((np.zeros((3, 4)), good), (good, np.zeros((3, 3), dtype=np.float32)),
                 (np.zeros((3, 6))[:, ::2], good), (torch.zeros(3, 3, dtype=torch.float32), good),
                 (good, torch.zeros(4, 3, dtype=torch.float64))):
        with pytest.raises(ValueError):
            eng.get2jmk_host(D, G)
