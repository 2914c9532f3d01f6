"""Pulay DIIS (PyQuante/Convergence.py:73-136), FP64, numpy or torch.

Two guards that the reference does not have:
  * the subspace keeps the last MAX_VECTORS Fock matrices (the reference keeps
    every one);
  * once the commutator error FDS - SDF is at rounding level, F is returned
    unextrapolated.
Without them, the solve for the extrapolation coefficients goes singular
near convergence and the extrapolated F, with the energy evaluated from it
(PyQuante/hartree_fock.py:134-136), can drift off the SCF solution: He /
6-31G** then ends at -2.8778 Eh, below the Hartree-Fock limit, instead of
the reference test's -2.85516 (Tests/he.py:15-16, which runs without DIIS).
"""
import numpy as np
import torch


MAX_VECTORS = 8
CONVERGED_ERROR = 1e-13


class DIIS:
    def __init__(self, S):
        self.Fs = []
        self.Errs = []
        self.Fold = None
        self.S = S
        self.started = True
        self.errcutoff = 0.1
        self.maxerr = None

    def error(self):
        return self.maxerr

    def getF(self, F, D):
        t = isinstance(F, torch.Tensor)
        err = (F @ D @ self.S - self.S @ D @ F).reshape(-1)
        self.maxerr = float(abs(err).max())
        if self.maxerr < CONVERGED_ERROR:
            return F
        self.Fs.append(F)
        self.Errs.append(err)
        if len(self.Errs) > MAX_VECTORS:
            del self.Fs[0]
            del self.Errs[0]
        nit = len(self.Errs)
        E = torch.stack(self.Errs) if t else np.stack(self.Errs)
        a = np.zeros((nit + 1, nit + 1))
        a[:nit, :nit] = (E @ E.T).cpu().numpy() if t else E @ E.T
        a[nit, :nit] = a[:nit, nit] = -1.0
        b = np.zeros(nit + 1)
        b[nit] = -1.0
        try:
            c = np.linalg.solve(a, b)
        except np.linalg.LinAlgError:
            self.Fold = F
            return F
        out = sum(float(c[i]) * self.Fs[i] for i in range(nit))
        return out
