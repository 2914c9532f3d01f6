"""Linear algebra of the SCF step (PyQuante/LA2.py:35-131), FP64, for numpy
arrays or torch tensors (a CUDA tensor stays on its device: cuSOLVER)."""
import numpy as np
import torch


def _is_t(x):
    return isinstance(x, torch.Tensor)


def simx(A, B, trans="N"):
    """B^T A B (trans 'N') or B A B^T (trans 'T')."""
    if trans.lower().startswith("t"):
        return B @ A @ B.T
    return B.T @ A @ B


def SymOrth(S):
    if _is_t(S):
        val, vec = torch.linalg.eigh(S)
        return vec @ torch.diag(1.0 / torch.sqrt(val)) @ vec.T
    val, vec = np.linalg.eigh(S)
    return vec @ np.diag(1.0 / np.sqrt(val)) @ vec.T


def SymOrthCutoff(S, scut=1e-5):
    if _is_t(S):
        val, vec = torch.linalg.eigh(S)
        d = torch.where(val > scut, 1.0 / torch.sqrt(val.clamp(min=scut)), torch.zeros_like(val))
        return vec @ torch.diag(d) @ vec.T
    val, vec = np.linalg.eigh(S)
    d = np.where(val > scut, 1.0 / np.sqrt(np.maximum(val, scut)), 0.0)
    return vec @ np.diag(d) @ vec.T


def CanOrth(S):
    if _is_t(S):
        val, vec = torch.linalg.eigh(S)
        return vec / torch.sqrt(val)
    val, vec = np.linalg.eigh(S)
    return vec / np.sqrt(val)


def CholOrth(S):
    """X = inv(L)^T with L L^T = S (PyQuante/LA2.py:113-116)."""
    if _is_t(S):
        L = torch.linalg.cholesky(S)
        return torch.linalg.inv(L).T
    return np.linalg.inv(np.linalg.cholesky(S)).T


def geigh(H, A, **opts):
    """Generalised symmetric eigenproblem H c = e A c (PyQuante/LA2.py:47-75).
    orthog: 'Chol' (default), 'Sym', 'Can', 'Cut'; have_xfrm=True means A is
    already the orthogonalising transform X."""
    if not opts.get("have_xfrm", False):
        orthog = opts.get("orthog", "Chol")
        X = {"Can": CanOrth, "Chol": CholOrth, "Cut": SymOrthCutoff}.get(orthog, SymOrth)(A)
        opts = dict(opts, have_xfrm=True)
        return geigh(H, X, **opts)
    if _is_t(H):
        val, vec = torch.linalg.eigh(simx(H, A))
    else:
        val, vec = np.linalg.eigh(simx(H, A))
    return val, A @ vec


GHeigenvectors = geigh   # the older name BASELINE/README use


def mkdens(c, nstart, nstop):
    """D = C[:, nstart:nstop] C[:, nstart:nstop]^T (no factor 2, LA2.py:127-131)."""
    d = c[:, nstart:nstop]
    return d @ d.T


def trace2(H, D):
    """tr(H D) for symmetric arguments, as sum(H*D)."""
    return float((H * D).sum())


def outprod(A):
    return A @ A.T
