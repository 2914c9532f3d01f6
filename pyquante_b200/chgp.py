"""Drop-in for the reference's ``chgp`` extension (Src/chgp.c:893-899):
``contr_coulomb``, ``coulomb_repulsion`` (= ``hrr``) and ``vrr``, evaluated on
the GPU by the Head-Gordon--Pople VRR/HRR with the Boys function from tables
(the reference uses a 3e-7-accurate incomplete gamma, so its values differ
from these by ~1e-8 relative)."""
from . import _lib, _scalar


def contr_coulomb(*args):
    return _scalar.contr_coulomb(_lib.PQB_ENGINE_HGP, args)


def coulomb_repulsion(*args):
    return _scalar.primitive(_lib.PQB_ENGINE_HGP, args)


hrr = coulomb_repulsion


def vrr(xyza, norma, lmna, alphaa, xyzb, normb, alphab, xyzc, normc, lmnc, alphac, xyzd, normd, alphad, m):
    """(a0|c0)^(m) with the norms and prefactor of Src/chgp.c:244-300."""
    return _scalar.primitive(_lib.PQB_ENGINE_HGP,
                             (xyza, norma, lmna, alphaa, xyzb, normb, (0, 0, 0), alphab,
                              xyzc, normc, lmnc, alphac, xyzd, normd, (0, 0, 0), alphad), aux_m=int(m))
