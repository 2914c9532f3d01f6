"""Host-side pieces of the batched SCF's captured iteration (pyquante_b200.batch),
on CPU tensors: the batched Gauss-Jordan solver against LAPACK, and the
ring-buffer DIIS against the list form of Pulay DIIS (PyQuante/Convergence.py:
73-136, at most S vectors) over more steps than the ring holds."""
import types

import numpy as np
import torch

from pyquante_b200.batch import _Diis, _solve_small


def test_small_solver_matches_lapack():
    rng = np.random.default_rng(0)
    for n in (1, 2, 5, 9):
        A = torch.tensor(rng.standard_normal((7, n, n)))
        b = torch.tensor(rng.standard_normal((7, n)))
        x = _solve_small(A, b)
        ref = torch.linalg.solve(A, b)
        assert float((x - ref).abs().max()) < 1e-11 * float(ref.abs().max())
    # a zero leading pivot needs the row exchange
    A = torch.tensor([[[0.0, 1.0], [1.0, 0.0]]])
    x = _solve_small(A, torch.tensor([[2.0, 3.0]]))
    assert torch.allclose(x, torch.tensor([[3.0, 2.0]]))


def test_ring_diis_matches_list_diis():
    rng = np.random.default_rng(1)
    B, nb, S = 3, 4, 5
    bk = types.SimpleNamespace(idx=list(range(B)), nb=nb, S=torch.zeros(1, dtype=torch.float64))
    d = _Diis(bk, S)
    Fs, Es = [], []
    for step in range(12):
        F = torch.tensor(rng.standard_normal((B, nb, nb)))
        err = torch.tensor(rng.standard_normal((B, nb, nb))) * 0.5 ** step
        got = d.step(F, err)
        Fs.append(F)
        Es.append(err.reshape(B, -1))
        Fs, Es = Fs[-S:], Es[-S:]
        k = len(Fs)
        for m in range(B):
            E = torch.stack([e[m] for e in Es]).numpy()
            a = np.zeros((k + 1, k + 1))
            a[:k, :k] = E @ E.T
            a[k, :k] = a[:k, k] = -1.0
            rhs = np.zeros(k + 1)
            rhs[k] = -1.0
            c = np.linalg.solve(a, rhs)
            want = sum(c[i] * Fs[i][m].numpy() for i in range(k))
            assert np.abs(got[m].numpy() - want).max() < 1e-9 * np.abs(want).max(), (step, m)
