"""Molecule container with PyQuante's semantics (PyQuante/Molecule.py:31-200):
coordinates in bohr unless ``units='angs'``, ``get_nel``, ``get_enuke``,
``get_closedopen``."""
from .Atom import Atom
from .Constants import ang2bohr
from .Element import sym2no

allowed_units = ["bohr", "angs"]


class Molecule:
    def __init__(self, name="molecule", atomlist=(), **opts):
        self.name = name
        self.atoms = []
        units = opts.get("units", "bohr").lower()[:4]
        if units not in allowed_units:
            raise ValueError("units must be one of %s" % allowed_units)
        self.units = units
        self.charge = int(opts.get("charge", 0))
        self.multiplicity = int(opts.get("multiplicity", 1))
        if atomlist:
            self.add_atuples(atomlist)

    def __iter__(self):
        return iter(self.atoms)

    def __len__(self):
        return len(self.atoms)

    def __getitem__(self, i):
        return self.atoms[i]

    def __repr__(self):
        return "\n%s: %s" % (self.__class__.__name__, self.name) + "".join("\n\t%s" % a for a in self.atoms)

    def add_atuple(self, atno, xyz, atid):
        if self.units != "bohr":
            xyz = [c * ang2bohr for c in xyz]
        if isinstance(atno, str):
            atno = sym2no[atno]
        self.atoms.append(Atom(atno, xyz[0], xyz[1], xyz[2], atid))

    def add_atuples(self, atoms):
        for i, (atno, xyz) in enumerate(atoms):
            self.add_atuple(atno, xyz, i)

    def atuples(self):
        return [a.atuple() for a in self.atoms]

    def update_coords(self, coords):
        coords = list(coords)
        assert len(coords) == 3 * len(self.atoms)
        for i, a in enumerate(self.atoms):
            a.update_coords(coords[3 * i:3 * i + 3])

    def get_charge(self):
        return self.charge

    def get_multiplicity(self):
        return self.multiplicity

    def get_nel(self, charge=None):
        if charge:
            self.charge = int(charge)
        return -self.charge + sum(a.get_nel() for a in self.atoms)

    def get_enuke(self):
        e = 0.0
        for i, ai in enumerate(self.atoms):
            for aj in self.atoms[:i]:
                e += ai.get_nuke_chg() * aj.get_nuke_chg() / ai.dist(aj)
        return e

    def get_closedopen(self):
        nel = self.get_nel()
        mult = self.multiplicity
        if mult <= 0 or (nel % 2 == 0 and mult % 2 == 0) or (nel % 2 == 1 and mult % 2 == 1):
            raise ValueError("Incompatible number of electrons (%d) and spin multiplicity (%d)" % (nel, mult))
        nopen = mult - 1
        nclosed, ierr = divmod(nel - nopen, 2)
        if ierr:
            raise ValueError("Error in Molecule.get_closedopen()")
        return nclosed, nopen

    def get_alphabeta(self):
        nclosed, nopen = self.get_closedopen()
        return nclosed + nopen, nclosed
