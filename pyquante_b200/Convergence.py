"""Pulay DIIS (PyQuante/Convergence.py:73-136), FP64, numpy or torch."""
import numpy as np
import torch


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
        self.Fs.append(F)
        self.Errs.append(err)
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
