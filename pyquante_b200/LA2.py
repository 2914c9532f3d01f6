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


def purify(Fp, nocc, pad=None, tol=1e-13, maxit=200, fixed=False, check=1):
    """P, the projector on the nocc lowest eigenstates of each symmetric
    Fp (a batch (B, n, n) of CUDA tensors; nocc per matrix), without an
    eigensolver: the canonical purification of Palser and Manolopoulos
    (Phys. Rev. B 58, 12704 (1998)), GEMMs only.
      P_0 = (lambda/n)(mu - Fp) + nocc/n, mu = tr(Fp)/n, lambda from the
      Gershgorin bounds of Fp;
      c = tr(P^2 - P^3)/tr(P - P^2);  P <- ((1+c)P^2 - P^3)/c for c >= 1/2,
      else ((1-2c)P + (1+c)P^2 - P^3)/(1-c).
    pad (B, n) marks padded dimensions (batched bases), which are held above
    the real spectrum and stay empty.  The iteration stops when every P is
    idempotent to rounding (|tr(P - P^2)| < tol n), tested on the host every
    ``check`` steps (converged matrices are kept meanwhile); fixed=True runs exactly
    maxit steps with no host check instead (converged matrices are kept),
    so that the loop can be captured in a CUDA graph.  Each step is two
    batched GEMMs and one fused trace-and-update kernel (pqb_purify_step)."""
    from . import _lib
    lib = _lib.load()
    Fp = 0.5 * (Fp + Fp.transpose(1, 2))
    nb = Fp.shape[-1]
    nocc = torch.as_tensor(nocc, dtype=Fp.dtype, device=Fp.device).reshape(-1)
    radius = Fp.abs().sum(-1) - Fp.diagonal(dim1=1, dim2=2).abs()
    d = Fp.diagonal(dim1=1, dim2=2)
    if pad is None:
        pad = torch.zeros_like(d, dtype=torch.bool)
    hi = torch.where(pad, torch.full_like(d, -1e300), d + radius).amax(1)
    lo = torch.where(pad, torch.full_like(d, 1e300), d - radius).amin(1)
    top = hi + 1.0
    Fp = Fp + torch.diag_embed(pad.to(Fp.dtype) * (top[:, None] - d))
    hi = torch.maximum(hi, top)
    mu = Fp.diagonal(dim1=1, dim2=2).sum(1) / nb
    lam = torch.minimum(nocc / (hi - mu), (nb - nocc) / (mu - lo))
    eye = torch.eye(nb, dtype=Fp.dtype, device=Fp.device)
    P = ((lam / nb)[:, None, None] * (mu[:, None, None] * eye - Fp) + (nocc / nb)[:, None, None] * eye).contiguous()
    P2 = torch.empty_like(P)
    P3 = torch.empty_like(P)
    done = torch.zeros(P.shape[0], dtype=torch.int32, device=P.device)
    for step in range(maxit):
        torch.bmm(P, P, out=P2)
        torch.bmm(P2, P, out=P3)
        rc = lib.pqb_purify_step(P.shape[0], nb, _lib.ptr(P), _lib.ptr(P2), _lib.ptr(P3), _lib.ptr(P), _lib.ptr(done),
                                 float(tol), _lib.stream_ptr())
        if rc != _lib.PQB_OK:
            raise _lib.EngineError(rc, "pqb_purify_step")
        if not fixed and step % check == check - 1 and bool(done.all()):
            break
    return P


def purify_density(F, X, nocc, **opts):
    """The closed-shell density D = C_occ C_occ^T (mkdens) of the Fock
    matrix F, for the orthogonalising transform X (CholOrth), by purify
    instead of the eigenvectors: D = X P X^T, P the projector on the nocc
    lowest states of X^T F X.  Batched or single (n, n) CUDA tensors."""
    single = F.dim() == 2
    Fb, Xb = (F[None], X[None]) if single else (F, X)
    P = purify(Xb.transpose(1, 2) @ Fb @ Xb, nocc, **opts)
    D = Xb @ P @ Xb.transpose(1, 2)
    return D[0] if single else D


def mkdens(c, nstart, nstop):
    """D = C[:, nstart:nstop] C[:, nstart:nstop]^T (no factor 2, LA2.py:127-131)."""
    d = c[:, nstart:nstop]
    return d @ d.T


def trace2(H, D):
    """tr(H D) for symmetric arguments, as sum(H*D)."""
    return float((H * D).sum())


def outprod(A):
    return A @ A.T
