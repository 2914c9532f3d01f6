"""Shared implementation of the scalar ERI entry points of the reference's C
extensions (crys, chgp, cints): build a 4-function device table from the
Python arguments and evaluate on the GPU."""
from types import SimpleNamespace

from . import _lib
from .engine import FunctionTable, eri_functions


def _func(exps, coefs, norms, origin, powers):
    if not (len(exps) == len(coefs) == len(norms)) or len(exps) == 0:
        raise ValueError("exponent, coefficient and norm sequences must have the same non-zero length")
    return SimpleNamespace(pexps=[float(e) for e in exps], pcoefs=[float(c) for c in coefs],
                           pnorms=[float(n) for n in norms], origin=tuple(float(c) for c in origin),
                           powers=tuple(int(p) for p in powers), norm=1.0)


def contr_coulomb(engine, args):
    """Sum over primitive quartets of c_a c_b c_c c_d (primitive ERI with
    primitive norms): the 20-argument contr_coulomb of Src/crys.c:1556-1674."""
    if len(args) != 20:
        raise TypeError("contr_coulomb takes 20 arguments (%d given)" % len(args))
    fs = [_func(*args[5 * i:5 * i + 5]) for i in range(4)]
    ctx = _lib.context()
    ft = FunctionTable(fs, ctx.device)
    return float(eri_functions(ft, [(0, 1, 2, 3)], ctx, engine)[0])


def primitive(engine, args, aux_m=0):
    """coulomb_repulsion((xa,ya,za),norma,(la,ma,na),alphaa, x4) of
    Src/crys.c:1676-1711 / Src/chgp.c:820-855."""
    if len(args) != 16:
        raise TypeError("coulomb_repulsion takes 16 arguments (%d given)" % len(args))
    fs = [_func([args[4 * i + 3]], [1.0], [args[4 * i + 1]], args[4 * i], args[4 * i + 2]) for i in range(4)]
    ctx = _lib.context()
    ft = FunctionTable(fs, ctx.device)
    return float(eri_functions(ft, [(0, 1, 2, 3)], ctx, engine, aux_m)[0])
