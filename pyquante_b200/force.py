"""Analytic RHF nuclear gradients on the GPU (PyQuante/force.py:31-70, Szabo &
Ostlund eq. C.12):

    dE/dR_a = 2 tr(D dh/dR_a) + tr(D dG[D]/dR_a) - 2 tr(W dS/dR_a) + dE_nuc/dR_a

with D = C_occ C_occ^T (no factor 2, PyQuante/LA2.py:127-131) and the
energy-weighted density W = C_occ diag(e_occ) C_occ^T (the Q matrix of
PyQuante/Wavefunction.py:143-149).  The two-electron term contracts the
derivative integrals with the density inside the kernel (pqb_grad_2e);
the one-electron term runs pqb_grad_1e.  Nothing of size N^4 is stored.

``RHFEnergy`` wraps the SCF energy as a torch.autograd.Function of the
nuclear coordinates, so ``torch.autograd.grad(E, coords)`` runs the adjoint
kernels.  ``rhf_force`` sets ``atom.f = -dE/dR`` as the reference does.
"""
import ctypes

import numpy as np
import torch

from . import _lib
from .Basis.basis import BasisSet
from .LA2 import geigh
from .Molecule import Molecule
from .engine import BasisEngine
from .hartree_fock import rhf


def nuclear_repulsion_gradient(mol):
    """dE_nuc/dR for every atom, (natoms, 3)."""
    R = np.array([a.r for a in mol.atoms])
    Z = np.array([a.get_nuke_chg() for a in mol.atoms], dtype=float)
    g = np.zeros_like(R)
    for a in range(len(R)):
        d = R[a] - R
        r3 = np.linalg.norm(d, axis=1) ** 3
        r3[a] = np.inf
        g[a] = -(Z[a] * Z[:, None] * d / r3[:, None]).sum(axis=0)
    return g


def _shell_atoms(eng):
    atid = [bf.atid for bf in eng.bfs]
    return [atid[f0] for f0 in eng.shells["f0"]]


def rhf_gradient_from_density(mol, eng, D, W, precision="fp64", schwarz=1e-12, fp32_threshold=1e-5):
    """Gradient (natoms, 3) for converged D, W on a BasisEngine of mol."""
    nat = len(mol.atoms)
    dev = eng.device
    D = torch.as_tensor(D, dtype=torch.float64, device=dev).contiguous()
    W = torch.as_tensor(W, dtype=torch.float64, device=dev).contiguous()
    grad = torch.zeros(3 * nat, dtype=torch.float64, device=dev)
    lib, h = eng.ctx.lib, eng.ctx.h
    sa = _shell_atoms(eng)
    eng.ctx.check(lib.pqb_set_shell_atoms(h, (ctypes.c_int * len(sa))(*sa)))
    eng.plan(schwarz, fp32_threshold)
    mode = _lib.PQB_MIXED if precision == "mixed" else _lib.PQB_FP64
    eng.ctx.check(lib.pqb_grad_2e(h, _lib.ptr(D), _lib.ptr(grad), mode, _lib.stream_ptr()))
    fa = torch.tensor([bf.atid for bf in eng.bfs], dtype=torch.int32, device=dev)
    xyz = (ctypes.c_double * (3 * nat))(*[c for a in mol.atoms for c in a.pos()])
    z = (ctypes.c_double * nat)(*[float(a.atno) for a in mol.atoms])
    ft = eng.ft
    eng.ctx.check(lib.pqb_grad_1e(h, *ft.args(), _lib.ptr(fa), nat, xyz, z, _lib.ptr(D), _lib.ptr(W), _lib.ptr(grad),
                                  _lib.stream_ptr()))
    g = grad.view(nat, 3).cpu().numpy()
    return g + nuclear_repulsion_gradient(mol)


def rhf_with_gradient(mol, basis_data=None, **opts):
    """(energy, gradient (natoms, 3), orbe, orbs) of a converged RHF."""
    bs = BasisSet(mol, basis_data)
    opts = dict(opts)
    opts.setdefault("ConvCriteria", 1e-10)
    opts.setdefault("MaxIter", 100)
    opts.setdefault("DoAveraging", True)
    precision = opts.get("precision", "fp64")
    schwarz = opts.get("schwarz", 1e-12)
    fp32 = opts.get("fp32_threshold", 1e-5)
    energy, orbe, orbs = rhf(mol, bfs=bs, direct=True, precision=precision, schwarz=schwarz, fp32_threshold=fp32,
                             **{k: v for k, v in opts.items() if k not in ("precision", "schwarz", "fp32_threshold")})
    nocc = mol.get_closedopen()[0]
    C = np.asarray(orbs)[:, :nocc]
    D = C @ C.T
    W = C @ np.diag(np.asarray(orbe)[:nocc]) @ C.T
    eng = bs._pqb_engine
    g = rhf_gradient_from_density(mol, eng, D, W, precision, schwarz, fp32)
    return energy, g, orbe, orbs


def rhf_force(mol, basis_data=None, **opts):
    """Set atom.f = -dE/dR for every atom (PyQuante/force.py:48-70)."""
    _, g, _, _ = rhf_with_gradient(mol, basis_data, **opts)
    for atom, gi in zip(mol.atoms, g):
        atom.f = -gi
    return -g


class RHFEnergy(torch.autograd.Function):
    """E_RHF(R) with an analytic backward: forward runs the SCF for nuclear
    coordinates R (natoms x 3, bohr), backward the gradient kernels."""

    @staticmethod
    def forward(ctx, coords, atnos, basis_data, opts):
        atoms = [(int(z), tuple(float(c) for c in r)) for z, r in zip(atnos, coords.detach().cpu().tolist())]
        mol = Molecule("rhf_energy", atoms, units="bohr")
        e, g, _, _ = rhf_with_gradient(mol, basis_data, **(opts or {}))
        ctx.save_for_backward(torch.as_tensor(g, dtype=coords.dtype, device=coords.device))
        return torch.tensor(e, dtype=coords.dtype, device=coords.device)

    @staticmethod
    def backward(ctx, grad_out):
        (g,) = ctx.saved_tensors
        return grad_out * g, None, None, None


def rhf_energy(coords, atnos, basis_data=None, **opts):
    """Differentiable RHF energy of nuclear coordinates (torch tensor)."""
    return RHFEnergy.apply(coords, list(atnos), basis_data, opts)
