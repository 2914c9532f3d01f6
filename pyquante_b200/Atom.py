"""Atom record (PyQuante/Atom.py:22-60): atomic number, position (bohr unless
the owning Molecule converted it), atom id."""
import numpy as np


class Atom:
    def __init__(self, atno, x, y, z, atid=0):
        self.atno = int(atno)
        self.r = np.array([x, y, z], dtype=float)
        self.atid = atid

    def __repr__(self):
        return "Atom ID: %d Atomic Num: %2d (%6.3f,%6.3f,%6.3f)" % (self.atid, self.atno, *self.r)

    def __getitem__(self, i):
        return self.r[i]

    def pos(self):
        return tuple(float(v) for v in self.r)

    def dist2(self, other):
        return float(((self.r - other.r) ** 2).sum())

    def dist(self, other):
        return self.dist2(other) ** 0.5

    def atuple(self):
        return (self.atno, self.r)

    def get_nel(self):
        return self.atno

    def get_nuke_chg(self):
        return self.atno

    def update_coords(self, xyz):
        self.r = np.array(xyz, dtype=float)
