"""Closed-shell (and unrestricted) Hartree-Fock drivers with PyQuante's
semantics (PyQuante/hartree_fock.py:29-253): same defaults (ConvCriteria 1e-4,
MaxIter 20, DoAveraging False), same energy expression
E = tr(D h) + tr(D F) + E_nuc with D = C_occ C_occ^T, Fock builds through
``Ints.get2JmK``.  Extra options: ``integrals`` as in the reference,
``direct=True`` / ``precision`` / ``schwarz`` / ``fp32_threshold`` forwarded
to ``getints``, ``device=True`` to keep the SCF loop on the GPU, and (rhf)
``solver='purify'``: each iteration's density from the Fock matrix by
canonical purification on the GPU (GEMMs, no eigensolver; implies
device=True), one eigensolve at the end for the returned orbitals."""
import logging

import numpy as np
import torch

from .Convergence import DIIS
from .Ints import get2JmK, getbasis, getints, getJ, getJK2, getK  # noqa: F401  (getJ/getK re-exported)
from .LA2 import CholOrth, geigh, mkdens, purify_density, trace2

logger = logging.getLogger("pyquante")


def get_fock(D, Ints, h):
    return h + get2JmK(Ints, D)


def get_energy(h, F, D, enuke=0.0, **opts):
    return trace2(D, h) + trace2(D, F) + enuke


def get_guess(h, S):
    return geigh(h, S)[1]


def hf(atoms, **opts):
    nclosed, nopen = atoms.get_closedopen()
    return uhf(atoms, **opts) if nopen else rhf(atoms, **opts)


def _setup(atoms, opts):
    bfs = opts.get("bfs")
    if not bfs:
        bfs = getbasis(atoms, opts.get("basis_data"))
    integrals = opts.get("integrals")
    if integrals:
        S, h, Ints = integrals
    else:
        keys = ("direct", "precision", "schwarz", "fp32_threshold")
        S, h, Ints = getints(bfs, atoms, **{k: opts[k] for k in keys if k in opts})
    if opts.get("device", False):
        S = torch.as_tensor(np.asarray(S), dtype=torch.float64, device="cuda")
        h = torch.as_tensor(np.asarray(h), dtype=torch.float64, device="cuda")
    return bfs, S, h, Ints


def rhf(atoms, **opts):
    """rhf(atoms, **opts) -> (energy, orbe, orbs) (PyQuante/hartree_fock.py:66-149)."""
    ConvCriteria = opts.get("ConvCriteria", 1e-4)
    MaxIter = opts.get("MaxIter", 20)
    DoAveraging = opts.get("DoAveraging", False)
    nclosed, nopen = atoms.get_closedopen()
    if nopen != 0:
        raise ValueError("SCF currently only works for closed-shell systems")
    solver = opts.get("solver", "eigh")
    if solver not in ("eigh", "purify"):
        raise ValueError("solver must be 'eigh' or 'purify'")
    if solver == "purify":
        opts = dict(opts, device=True)
    bfs, S, h, Ints = _setup(atoms, opts)
    orbs = opts.get("orbs")
    if orbs is None:
        orbe, orbs = geigh(h, S)
    elif isinstance(S, torch.Tensor):
        orbs = torch.as_tensor(np.asarray(orbs), dtype=torch.float64, device=S.device)
    X = CholOrth(S) if solver == "purify" else None
    enuke = atoms.get_enuke()
    eold = 0.0
    avg = DIIS(S) if DoAveraging else None
    energy = 0.0
    D = mkdens(orbs, 0, nclosed)
    F = None
    for it in range(MaxIter):
        G = get2JmK(Ints, D)
        F = h + G
        if avg is not None:
            F = avg.getF(F, D)
        if solver == "purify":
            Dn = purify_density(F, X, nclosed, check=4)
        else:
            orbe, orbs = geigh(F, S)
            Dn = mkdens(orbs, 0, nclosed)
        energy = get_energy(h, F, D, enuke)
        logger.debug("%d %f", it, energy)
        D = Dn
        if abs(energy - eold) < ConvCriteria:
            break
        eold = energy
    if solver == "purify" and F is not None:
        orbe, orbs = geigh(F, S)
    if isinstance(orbs, torch.Tensor):
        orbe, orbs = orbe.cpu().numpy(), orbs.cpu().numpy()
    return energy, orbe, orbs


def uhf(atoms, **opts):
    """Unrestricted HF (PyQuante/hartree_fock.py:151-253): defaults
    ConvCriteria 1e-5, MaxIter 40, density averaging 0.5 on; F_a = h + J_a +
    J_b - K_a; E = (E_a + E_b)/2 + E_nuc with E_x = tr(D_x h) + tr(D_x F_x).
    The reference's getJ(Da), getJ(Db), getK(Da), getK(Db) come from one
    getJK2 call: integral-direct, both densities digest every integral of
    one pass."""
    ConvCriteria = opts.get("ConvCriteria", 1e-5)
    MaxIter = opts.get("MaxIter", 40)
    DoAveraging = opts.get("DoAveraging", True)
    averaging = opts.get("averaging", 0.5)
    nalpha, nbeta = atoms.get_alphabeta()
    bfs, S, h, Ints = _setup(atoms, opts)
    orbs = opts.get("orbs")
    if orbs is not None:
        orbsa, orbsb = orbs
    else:
        orbe, orbs = geigh(h, S)
        orbsa = orbsb = orbs
    enuke = atoms.get_enuke()
    eold = 0.0
    energy = 0.0
    Da0 = Db0 = None
    for it in range(MaxIter):
        Da = mkdens(orbsa, 0, nalpha)
        Db = mkdens(orbsb, 0, nbeta)
        if DoAveraging:
            if it:
                Da = averaging * Da + (1 - averaging) * Da0
                Db = averaging * Db + (1 - averaging) * Db0
            Da0, Db0 = Da, Db
        # getJ(Da), getJ(Db), getK(Da), getK(Db) of the reference, from one
        # pass over the integrals
        Ja, Jb, Ka, Kb = getJK2(Ints, Da, Db)
        Fa = h + Ja + Jb - Ka
        Fb = h + Ja + Jb - Kb
        orbea, orbsa = geigh(Fa, S)
        orbeb, orbsb = geigh(Fb, S)
        energy = (get_energy(h, Fa, Da) + get_energy(h, Fb, Db)) / 2 + enuke
        if abs(energy - eold) < ConvCriteria:
            break
        eold = energy
    if isinstance(orbsa, torch.Tensor):
        orbea, orbeb = orbea.cpu().numpy(), orbeb.cpu().numpy()
        orbsa, orbsb = orbsa.cpu().numpy(), orbsb.cpu().numpy()
    return energy, (orbea, orbeb), (orbsa, orbsb)
