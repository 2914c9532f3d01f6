"""Closed-shell Kohn-Sham DFT with the reference's semantics
(PyQuante/dft.py:29-215): the default grid (pyquante_b200.MolecularGrid,
32 Euler--Maclaurin shells x 194 Lebedev points per atom, Becke
partitioning), the SVWN functional, F = h + 2J + Fxc with J from
``Ints.getJ`` (stored, or integral-direct with the Coulomb digestion alone), DIIS on by default, and
E = 2 tr(D h) + 2 tr(D J) + Exc + E_nuc with the spin-averaged density
D = C_occ C_occ^T (+ half the open shells).

The grid work runs on the GPU: basis amplitudes (pqb_grid_amps), the
density (one DGEMM B D and pqb_grid_rowdot), the functional
(pqb_xc_svwn) and Fxc = B^T diag(w v) B (one DGEMM).
"""
import logging

import numpy as np
import torch

from .Convergence import DIIS
from .DFunctionals import XC, need_gradients
from .Ints import getbasis, getints, getJ
from .LA2 import geigh, mkdens, trace2
from .MolecularGrid import MolecularGrid

logger = logging.getLogger("pyquante")


def mkdens_spinavg(c, nclosed, nopen):
    """Spin-averaged density (PyQuante/LA2.py:133-136)."""
    D = mkdens(c, 0, nclosed)
    return D + 0.5 * mkdens(c, nclosed, nclosed + nopen) if nopen else D


def getXC(gr, nel, **kwargs):
    """(Exc, Fxc) for the density set on the grid (PyQuante/dft.py:29-65)."""
    functional = kwargs.get("functional", "SVWN")
    if need_gradients.get(functional, True):
        raise NotImplementedError("gradient-corrected functionals are not built")
    gr.floor_density()
    gr.renormalize(nel)
    w = gr.weights()
    fxc, va, vb, _, _, _ = XC(gr.density.T, None, functional=functional)
    exc = float(torch.dot(w, fxc))
    wva = w * va
    B = gr.bfgrid
    Fxc = torch.matmul(B.T, B * wva[:, None])
    return exc, Fxc


def dft(atoms, **kwargs):
    """dft(atoms, **kwargs) -> (energy, orbe, orbs) (PyQuante/dft.py:116-215).
    Options as the reference: ConvCriteria (1e-4), MaxIter (20),
    DoAveraging (True: DIIS), functional ('SVWN'), bfs / basis_data,
    integrals, orbs, grid_nrad (32), grid_fineness (1); plus the
    integral options of ``getints`` (direct, precision, schwarz,
    fp32_threshold)."""
    ConvCriteria = kwargs.get("ConvCriteria", 1e-4)
    MaxIter = kwargs.get("MaxIter", 20)
    DoAveraging = kwargs.get("DoAveraging", True)
    functional = kwargs.get("functional", "SVWN")
    if kwargs.get("ETemp", False):
        raise NotImplementedError("finite-temperature DFT is not built")
    bfs = kwargs.get("bfs")
    if not bfs:
        bfs = getbasis(atoms, kwargs.get("basis_data"))
    integrals = kwargs.get("integrals")
    if integrals:
        S, h, Ints = integrals
    else:
        keys = ("direct", "precision", "schwarz", "fp32_threshold")
        S, h, Ints = getints(bfs, atoms, **{k: kwargs[k] for k in keys if k in kwargs})
    nel = atoms.get_nel()
    enuke = atoms.get_enuke()
    gr = MolecularGrid(atoms, kwargs.get("grid_nrad", 32), kwargs.get("grid_fineness", 1))
    gr.set_bf_amps(bfs)
    dev = gr.device
    S = torch.as_tensor(np.asarray(S), dtype=torch.float64, device=dev)
    h = torch.as_tensor(np.asarray(h), dtype=torch.float64, device=dev)
    orbs = kwargs.get("orbs")
    if orbs is None:
        orbe, orbs = geigh(h, S)
    else:
        orbs = torch.as_tensor(np.asarray(orbs), dtype=torch.float64, device=dev)
    nclosed, nopen = atoms.get_closedopen()
    avg = DIIS(S) if DoAveraging else None
    eold = 0.0
    energy = 0.0
    for it in range(MaxIter):
        D = mkdens_spinavg(orbs, nclosed, nopen)
        gr.setdens(D)
        J = getJ(Ints, D, coulomb_only=True)
        Exc, Fxc = getXC(gr, nel, functional=functional)
        F = h + 2 * J + Fxc
        if avg is not None:
            F = avg.getF(F, D)
        orbe, orbs = geigh(F, S)
        energy = float(2 * trace2(D, J) + 2 * trace2(D, h) + Exc + enuke)
        logger.debug("%d %f", it, energy)
        if abs(energy - eold) < ConvCriteria:
            break
        eold = energy
    return energy, orbe.cpu().numpy(), orbs.cpu().numpy()
