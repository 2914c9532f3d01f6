"""Primitive cartesian Gaussian (PyQuante/PGBF.py, with the normalisation of
Src/lib/primitive-gto.c:76-83 applied at construction as PrimitiveGTO does):

    g(r) = norm * x^l y^m z^n exp(-alpha |r - origin|^2)
    norm = sqrt(2^(2L+1.5) alpha^(L+1.5) / ((2l-1)!! (2m-1)!! (2n-1)!! pi^1.5))
"""
import math


def fact2(n):
    """Double factorial, 1 for n <= 1 (Src/cints.c:315-318)."""
    r = 1
    while n > 1:
        r *= n
        n -= 2
    return r


def primitive_norm(alpha, powers):
    l, m, n = powers
    L = l + m + n
    return math.sqrt(2.0 ** (2 * L + 1.5) * alpha ** (L + 1.5) /
                     (fact2(2 * l - 1) * fact2(2 * m - 1) * fact2(2 * n - 1) * math.pi ** 1.5))


class PGBF:
    def __init__(self, exponent, origin, powers=(0, 0, 0), norm=1.0):
        self.exp = float(exponent)
        self.origin = tuple(float(c) for c in origin)
        self.powers = tuple(int(p) for p in powers)
        self.norm = primitive_norm(self.exp, self.powers)
        self.coef = 1.0

    @property
    def alpha(self):
        return self.exp

    def reset_powers(self, px, py, pz):
        self.powers = (px, py, pz)
        self.norm = primitive_norm(self.exp, self.powers)

    def move_center(self, dx, dy, dz):
        self.origin = (self.origin[0] + dx, self.origin[1] + dy, self.origin[2] + dz)

    def amp(self, x, y, z):
        l, m, n = self.powers
        x0, y0, z0 = self.origin
        r2 = (x - x0) ** 2 + (y - y0) ** 2 + (z - z0) ** 2
        return self.norm * self.coef * (x - x0) ** l * (y - y0) ** m * (z - z0) ** n * math.exp(-self.exp * r2)

    def coulomb(self, b, c, d):
        from .chgp import coulomb_repulsion
        return coulomb_repulsion(self.origin, self.norm, self.powers, self.exp, b.origin, b.norm, b.powers, b.exp,
                                 c.origin, c.norm, c.powers, c.exp, d.origin, d.norm, d.powers, d.exp)
