"""Contracted cartesian Gaussian (PyQuante/CGBF.py:25-75, 191-199).

As in the reference, ``norm`` starts at 1 and is left there by BasisSet (the
contraction is not renormalised); each primitive carries its own
per-component norm in ``pnorms``.  ``coulomb(a, b, c, d)`` is
``a.norm b.norm c.norm d.norm crys.contr_coulomb(...)`` and runs on the GPU.
"""
from .PGBF import PGBF


class CGBF:
    def __init__(self, origin, powers=(0, 0, 0), atid=0):
        self.origin = tuple(float(c) for c in origin)
        self.powers = tuple(int(p) for p in powers)
        self.norm = 1.0
        self.prims = []
        self.pnorms = []
        self.pexps = []
        self.pcoefs = []
        self.ang_mom = sum(self.powers)
        self.atid = atid

    def __repr__(self):
        return '<cgbf atomid=%d origin="(%f,%f,%f)" powers="(%d,%d,%d)" nprim=%d>' % (
            (self.atid,) + self.origin + self.powers + (len(self.prims),))

    def add_primitive(self, exponent, coefficient):
        pbf = PGBF(exponent, self.origin, self.powers)
        pbf.coef = float(coefficient)
        self.prims.append(pbf)
        self.pnorms.append(pbf.norm)
        self.pexps.append(float(exponent))
        self.pcoefs.append(float(coefficient))

    def reset_powers(self, px, py, pz):
        self.powers = (px, py, pz)
        self.ang_mom = px + py + pz
        for p in self.prims:
            p.reset_powers(px, py, pz)
        self.pnorms = [p.norm for p in self.prims]

    def move_center(self, dx, dy, dz):
        self.origin = (self.origin[0] + dx, self.origin[1] + dy, self.origin[2] + dz)
        for p in self.prims:
            p.move_center(dx, dy, dz)

    def amp(self, x, y, z):
        return self.norm * sum(p.amp(x, y, z) for p in self.prims)

    # one-electron matrix elements between two functions (GPU, one-off calls)
    def _pair(self, other, atoms=None):
        from .Ints import _oneint_functions
        return _oneint_functions([self, other], atoms)

    def overlap(self, other):
        return float(self._pair(other)[0][0, 1])

    def kinetic(self, other):
        return float(self._pair(other)[1][0, 1])

    def nuclear(self, other, C):
        """<self| -1/|r-C| |other> (unit charge at C), as PyQuante's CGBF.nuclear."""
        from .Atom import Atom
        S, T, V = self._pair(other, [Atom(1, *C)])
        return float(V[0, 1])

    def normalize(self):
        """Scale ``norm`` so that <self|self> = 1 (Src/lib/contracted-gto.c:104-111)."""
        s = self.overlap(self)
        self.norm = self.norm / s ** 0.5


def coulomb(a, b, c, d):
    """Coulomb interaction between 4 contracted Gaussians (PyQuante/CGBF.py:191-199)."""
    from .crys import contr_coulomb
    return a.norm * b.norm * c.norm * d.norm * contr_coulomb(
        a.pexps, a.pcoefs, a.pnorms, a.origin, a.powers,
        b.pexps, b.pcoefs, b.pnorms, b.origin, b.powers,
        c.pexps, c.pcoefs, c.pnorms, c.origin, c.powers,
        d.pexps, d.pcoefs, d.pnorms, d.origin, d.powers)
