"""pqb_oneint_noalloc: the allocation-free one-electron entry point.

Some callers cannot allocate device memory (a framework's pool owns the GPU,
or the call sits where allocation is not allowed); this entry point keeps its
scratch in a static device array instead.  It must give the same S, T, V as
pqb_oneint, call after call (the scratch is shared and reused).  Collected
last (file name) so a stop-at-first-failure run has already run the rest."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def test_oneint_noalloc_matches_oneint_on_two_calls():
    from pyquante_b200 import _lib, geometries
    from pyquante_b200.Basis.basis import BasisSet
    from pyquante_b200.engine import FunctionTable, oneint

    ctx = _lib.context()
    mol = geometries.water_cluster(3, seed=9)
    bs = BasisSet(mol, "6-31g**")
    ft = FunctionTable(bs.bfs, ctx.device)
    S0, T0, V0 = oneint(ft, mol.atoms, ctx)
    xyz = torch.tensor([c for a in mol.atoms for c in a.pos()], dtype=torch.float64, device="cuda")
    z = torch.tensor([float(a.atno) for a in mol.atoms], dtype=torch.float64, device="cuda")
    n = ft.n
    for call in range(2):
        S = torch.full((n, n), float("nan"), dtype=torch.float64, device="cuda")
        T = torch.full_like(S, float("nan"))
        V = torch.full_like(S, float("nan"))
        before = torch.cuda.memory_allocated()
        rc = ctx.lib.pqb_oneint_noalloc(*ft.args(), len(mol.atoms), _lib.ptr(xyz), _lib.ptr(z), _lib.ptr(S),
                                        _lib.ptr(T), _lib.ptr(V), _lib.stream_ptr())
        assert rc == _lib.PQB_OK
        torch.cuda.synchronize()
        assert torch.cuda.memory_allocated() == before
        for got, want in ((S, S0), (T, T0), (V, V0)):
            assert float((got - want).abs().max()) < 1e-12, call


def test_oneint_noalloc_without_v_reads_no_atoms():
    """As with pqb_oneint, the atoms are needed only for V: S and T alone
    take null atom arrays."""
    from pyquante_b200 import _lib, geometries
    from pyquante_b200.Basis.basis import BasisSet
    from pyquante_b200.engine import FunctionTable, oneint

    ctx = _lib.context()
    mol = geometries.water()
    ft = FunctionTable(BasisSet(mol, "6-31g**").bfs, ctx.device)
    S0, T0, _ = oneint(ft, mol.atoms, ctx)
    S = torch.full_like(S0, float("nan"))
    T = torch.full_like(S0, float("nan"))
    rc = ctx.lib.pqb_oneint_noalloc(*ft.args(), len(mol.atoms), None, None, _lib.ptr(S), _lib.ptr(T), None,
                                    _lib.stream_ptr())
    assert rc == _lib.PQB_OK
    torch.cuda.synchronize()
    assert float((S - S0).abs().max()) < 1e-12 and float((T - T0).abs().max()) < 1e-12


def test_oneint_noalloc_rejects_too_many_atoms():
    from pyquante_b200 import _lib
    lib = _lib.load()
    d = torch.zeros(4, dtype=torch.float64, device="cuda")
    i = torch.zeros(4, dtype=torch.int32, device="cuda")
    P = _lib.ptr
    rc = lib.pqb_oneint_noalloc(1, P(d), P(i), P(i), P(d), P(d), P(d), 4097, P(d), P(d), P(d), P(d), P(d),
                                _lib.stream_ptr())
    assert rc == _lib.PQB_E_SHAPE
