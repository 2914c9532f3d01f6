"""Drop-in for the reference's ``crys`` extension (Src/crys.c:1713-1717):
``contr_coulomb`` and ``coulomb_repulsion`` with the same positional
signatures, evaluated on the GPU by Rys quadrature.  Unlike the reference,
bad sequence lengths raise instead of returning NULL, and total angular
momentum above 9 raises instead of silently using stale roots
(Src/crys.c:1440-1443)."""
from . import _lib, _scalar


def contr_coulomb(*args):
    return _scalar.contr_coulomb(_lib.PQB_ENGINE_RYS, args)


def coulomb_repulsion(*args):
    return _scalar.primitive(_lib.PQB_ENGINE_RYS, args)
