"""Moller-Plesset MP2 on the B200 engine (PyQuante/MP.py:20-97).

    moints = TransformIntsMP2(Ints, orbs, nclosed)     # packed (ai|bj), a, b occupied
    emp2 = MP2(Ints, orbs, orbe, nclosed, nvirt)        # second-order energy

``Ints`` is the packed AO array of ``Ints.getints`` (a PackedInts, a torch
tensor or an array).  The reference transforms one index at a time in
Python loops, O(N^5) calls of ``dot``; here the four quarter transformations
are FP64 GEMMs on the GPU (cuBLAS DGEMM through torch), fed by the engine's
own gather kernels (pqb_mo_unpack_rows, pqb_mo_unpack_pairs) that turn the
8-fold packed order into dense rows, and the pair energies are one kernel
(pqb_mp2_pairs).  Everything is FP64: no reduced-precision tensor-core path.

    1. (mu nu|sigma eta) -> (mu nu|b j): per batch of packed AO pairs mu >= nu,
       unpack the rows and contract eta with C[:, j] and sigma with C[:, b];
    2. (mu nu|b j) -> (a i|b j): unpack the pair index to (mu, nu) and
       contract nu with C[:, i] and mu with C[:, a].
MP2 takes i, j over the virtual orbitals only; TransformIntsMP2 over all MOs,
as the reference does, and stores (ai|bj) at ijkl2intindex(a, i, b, j) of a
packed MO array (zeros elsewhere).
"""
import numpy as np
import torch

from . import _lib
from ._lib import ptr, stream_ptr

# bytes of one batch of unpacked AO rows (N^2 doubles per row)
_ROW_BATCH_BYTES = 512 << 20


def _ao_tensor(Ints):
    t = getattr(Ints, "tensor", Ints)
    if not isinstance(t, torch.Tensor):
        t = torch.as_tensor(np.asarray(t, dtype=np.float64))
    if not t.is_cuda:
        t = t.to("cuda")
    return t.to(torch.float64).contiguous()


def _check(rc, what):
    if rc != _lib.PQB_OK:
        raise _lib.EngineError(rc, what)


def _half_transform(ints, nbf, Cb, Cj, stream=None):
    """Y[P, nb, nj] = (mu nu|b j) = sum_{sigma eta} Cb[sigma, b] Cj[eta, j]
    (mu nu|sigma eta) for every packed AO pair mu >= nu."""
    lib = _lib.load()
    P = nbf * (nbf + 1) // 2
    nb, nj = Cb.shape[1], Cj.shape[1]
    Y = torch.empty((P, nb, nj), dtype=torch.float64, device=ints.device)
    batch = max(1, min(P, _ROW_BATCH_BYTES // (8 * nbf * nbf)))
    X = torch.empty((batch, nbf, nbf), dtype=torch.float64, device=ints.device)
    CbT = Cb.T.contiguous()
    for r0 in range(0, P, batch):
        nr = min(batch, P - r0)
        Xb = X[:nr]
        _check(lib.pqb_mo_unpack_rows(ptr(ints), ints.numel(), nbf, r0, nr, ptr(Xb), stream_ptr(stream)),
               "pqb_mo_unpack_rows")
        T1 = torch.matmul(Xb.view(nr * nbf, nbf), Cj).view(nr, nbf, nj)     # eta -> j
        torch.matmul(CbT, T1, out=Y[r0:r0 + nr])                          # sigma -> b
    return Y


def _second_half(Y, nbf, Ca, Ci, stream=None):
    """Z[a, i, c] = sum_{mu nu} Ca[mu, a] Ci[nu, i] Y[pair(mu, nu), c]."""
    lib = _lib.load()
    P, ncol = Y.shape[0], Y.shape[1] * Y.shape[2]
    Yf = torch.empty((nbf, nbf, ncol), dtype=torch.float64, device=Y.device)
    _check(lib.pqb_mo_unpack_pairs(ptr(Y), nbf, ncol, ptr(Yf), stream_ptr(stream)), "pqb_mo_unpack_pairs")
    T = torch.matmul(Ca.T.contiguous(), Yf.view(nbf, nbf * ncol)).view(Ca.shape[1], nbf, ncol)   # mu -> a
    del Yf
    return torch.matmul(Ci.T.contiguous(), T)                                                 # nu -> i


class MOInts:
    """Packed MO integrals, indexable like the reference's array
    (``moints[ijkl2intindex(a, i, b, j)]``)."""

    def __init__(self, tensor):
        self.tensor = tensor

    def __len__(self):
        return self.tensor.numel()

    def __getitem__(self, idx):
        v = self.tensor[idx]
        return float(v) if v.dim() == 0 else v.cpu().numpy()

    def numpy(self):
        return self.tensor.cpu().numpy()


def TransformIntsMP2(Ints, orbs, nclosed):
    """(ai|bj) for occupied a, b and every MO i, j, packed at
    ijkl2intindex(a, i, b, j) (PyQuante/MP.py:20-75)."""
    ints = _ao_tensor(Ints)
    C = torch.as_tensor(np.asarray(orbs), dtype=torch.float64, device=ints.device).contiguous()
    nbf, nmo = C.shape
    Cocc = C[:, :nclosed].contiguous()
    Y = _half_transform(ints, nbf, Cocc, C)                  # (mu nu|b j)
    Z = _second_half(Y, nbf, Cocc, C)                        # (a i|b j): [nocc, nmo, nocc*nmo]
    del Y
    Q = nmo * (nmo + 1) // 2
    moints = torch.zeros(Q * (Q + 1) // 2, dtype=torch.float64, device=ints.device)
    _check(_lib.load().pqb_mo_pack(ptr(Z), nclosed, nmo, ptr(moints), moints.numel(), stream_ptr()), "pqb_mo_pack")
    return MOInts(moints)


def MP2(aoints, orbs, orbe, nclosed, nvirt):
    """Second-order Moller-Plesset energy (PyQuante/MP.py:77-97):
    sum over occupied a, b and virtual r, s of
    (ar|bs) (2 (ar|bs) - (as|br)) / (e_a + e_b - e_r - e_s)."""
    ints = _ao_tensor(aoints)
    dev = ints.device
    C = torch.as_tensor(np.asarray(orbs), dtype=torch.float64, device=dev).contiguous()
    e = torch.as_tensor(np.asarray(orbe), dtype=torch.float64, device=dev).contiguous()
    nbf = C.shape[0]
    Cocc = C[:, :nclosed].contiguous()
    Cvir = C[:, nclosed:nclosed + nvirt].contiguous()
    if nvirt == 0:
        return 0.0
    Y = _half_transform(ints, nbf, Cocc, Cvir)               # (mu nu|b s)
    V = _second_half(Y, nbf, Cocc, Cvir).contiguous()        # (a r|b s): [nocc, nvirt, nocc*nvirt]
    del Y
    Ep = torch.empty(nclosed * nclosed, dtype=torch.float64, device=dev)
    eo = e[:nclosed].contiguous()
    ev = e[nclosed:nclosed + nvirt].contiguous()
    _check(_lib.load().pqb_mp2_pairs(ptr(V), nclosed, nvirt, ptr(eo), ptr(ev), ptr(Ep), stream_ptr()),
           "pqb_mp2_pairs")
    return float(Ep.sum())
