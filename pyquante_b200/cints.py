"""Drop-in for the reference's ``cints`` extension (Src/cints.c:948-967).

The two-electron entry points keep their signatures but evaluate on the GPU
(by Rys quadrature: the THO closed form of Src/cints.c:110-187 is not rebuilt
as a kernel).  ``ijkl2intindex`` is 64-bit.  One-electron entry points run
the GPU one-electron kernel on single primitives.  The small combinatorial
helpers are plain Python."""
import math

from . import _lib, _scalar
from .Atom import Atom
from .PGBF import fact2  # noqa: F401


def ijkl2intindex(i, j, k, l):
    return int(_lib.load().pqb_ijkl2intindex(int(i), int(j), int(k), int(l)))


def contr_coulomb(*args):
    return _scalar.contr_coulomb(_lib.PQB_ENGINE_RYS, args)


def coulomb_repulsion(*args):
    return _scalar.primitive(_lib.PQB_ENGINE_RYS, args)


def fact(n):
    return math.factorial(n) if n > 1 else 1


def binomial(a, b):
    return fact(a) // (fact(b) * fact(a - b))


def dist2(a, b):
    return sum((x - y) ** 2 for x, y in zip(a, b))


def dist(a, b):
    return math.sqrt(dist2(a, b))


def _prim_pair(alpha1, powers1, origin1, alpha2, powers2, origin2, norm1=1.0, norm2=1.0):
    from types import SimpleNamespace
    from .engine import FunctionTable
    fs = [SimpleNamespace(pexps=[float(alpha1)], pcoefs=[1.0], pnorms=[float(norm1)], origin=tuple(origin1),
                          powers=tuple(powers1), norm=1.0),
          SimpleNamespace(pexps=[float(alpha2)], pcoefs=[1.0], pnorms=[float(norm2)], origin=tuple(origin2),
                          powers=tuple(powers2), norm=1.0)]
    ctx = _lib.context()
    return FunctionTable(fs, ctx.device), ctx


def overlap(alpha1, powers1, origin1, alpha2, powers2, origin2):
    """Unnormalised primitive overlap (Src/cints.c:215-234)."""
    from .engine import oneint
    ft, ctx = _prim_pair(alpha1, powers1, origin1, alpha2, powers2, origin2)
    return float(oneint(ft, [], ctx)[0][0, 1])


def kinetic(alpha1, powers1, origin1, alpha2, powers2, origin2):
    """Unnormalised primitive kinetic energy (Src/cints.c:190-213)."""
    from .engine import oneint
    ft, ctx = _prim_pair(alpha1, powers1, origin1, alpha2, powers2, origin2)
    return float(oneint(ft, [], ctx)[1][0, 1])


def nuclear_attraction(origin1, norm1, powers1, alpha1, origin2, norm2, powers2, alpha2, C):
    """-norm1 norm2 <a|1/|r-C||b> (Src/cints.c:248-281)."""
    from .engine import oneint
    ft, ctx = _prim_pair(alpha1, powers1, origin1, alpha2, powers2, origin2, norm1, norm2)
    return float(oneint(ft, [Atom(1, *C)], ctx)[2][0, 1])


def Fgamma(m, x):
    """Boys function F_m(x) = 0.5 x^(-m-1/2) gamma(m+1/2, x) (Src/cints.c:340-346).
    Integer m runs the device kernel (table + downward recursion); other m
    (a utility the reference also accepts) use the regularised incomplete
    gamma function."""
    x = max(float(x), 1e-8)   # the reference clamps |x| < 1e-8 the same way
    if float(m).is_integer() and 0 <= m <= 16:
        import torch
        ctx = _lib.context()
        T = torch.tensor([x], dtype=torch.float64, device="cuda")
        F = torch.empty(int(m) + 1, dtype=torch.float64, device="cuda")
        ctx.check(ctx.lib.pqb_boys_eval(ctx.h, int(m), 1, _lib.ptr(T), _lib.ptr(F), _lib.stream_ptr()))
        return float(F[int(m)])
    from scipy.special import gamma, gammainc
    a = m + 0.5
    return 0.5 * x ** (-a) * gamma(a) * gammainc(a, x)
