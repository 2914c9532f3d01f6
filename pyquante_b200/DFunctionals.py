"""Exchange-correlation functionals of the DFT path on the GPU
(PyQuante/DFunctionals.py:17-74 XC, with S and VWN of :76-138).

``XC(dens, gamma, functional='SVWN')`` takes the spin densities as a
(2, npts) device tensor, like the reference, and returns
(fxc, dfxcdna, dfxcdnb, dfxcdgaa, dfxcdgab, dfxcdgbb); the gradient terms are
zero for the local functional built here (SVWN, the reference's default,
and its aliases LDA and SVWN5).  The point-wise work is pqb_xc_svwn.
"""
import torch

from . import _lib
from ._lib import ptr, stream_ptr

need_gradients = dict(LDA=False, SVWN=False, SVWN5=False)


def _svwn(rhoa, rhob, w=None):
    n = rhoa.numel()
    w = torch.ones_like(rhoa) if w is None else w.contiguous()
    out = [torch.empty_like(rhoa) for _ in range(3)]
    rc = _lib.load().pqb_xc_svwn(n, ptr(rhoa.contiguous()), ptr(rhob.contiguous()), ptr(w), *(ptr(x) for x in out),
                                 stream_ptr())
    if rc != _lib.PQB_OK:
        raise _lib.EngineError(rc, "pqb_xc_svwn")
    return out


def XC(dens, gamma=None, **opts):
    functional = opts.get("functional", "SVWN")
    if functional not in need_gradients:
        raise NotImplementedError("functional %s: only the local SVWN functional is built" % functional)
    f, va, vb = _svwn(dens[0].contiguous(), dens[1].contiguous())
    z = torch.zeros_like(f)
    return f, va, vb, z, z, z
