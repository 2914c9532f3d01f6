"""BasisSet (PyQuante/Basis/basis.py:8-57): contracted functions atom by atom,
shell by shell in basis-file order, cartesian components in PyQuante order
(PyQuante/Ints.py:23-29).  Contracted norms stay 1, as in the reference."""
from ..CGBF import CGBF
from .Tools import get_basis_data

sym2powerlist = {
    "S": [(0, 0, 0)],
    "P": [(1, 0, 0), (0, 1, 0), (0, 0, 1)],
    "D": [(2, 0, 0), (1, 1, 0), (1, 0, 1), (0, 2, 0), (0, 1, 1), (0, 0, 2)],
    "F": [(3, 0, 0), (2, 1, 0), (2, 0, 1), (1, 2, 0), (1, 1, 1), (1, 0, 2), (0, 3, 0), (0, 2, 1), (0, 1, 2),
          (0, 0, 3)],
}


class Shell:
    """The functions of one shell (indices into BasisSet.bfs)."""

    def __init__(self, sym):
        self.sym = sym
        self.functions = []
        self.indices = []

    def append(self, cgbf, index):
        self.functions.append(cgbf)
        self.indices.append(index)

    def __len__(self):
        return len(self.functions)


class BasisSet:
    def __init__(self, atoms, basis_data=None, **opts):
        omit_f = opts.get("omit_f", False)
        if not basis_data:
            from .p631ss import basis_data
        elif isinstance(basis_data, str):
            basis_data = get_basis_data(basis_data)
        bfs, shells = [], []
        for atom in atoms:
            for sym, prims in basis_data[atom.atno]:
                if omit_f and sym == "F":
                    continue
                shell = Shell(sym)
                for power in sym2powerlist[sym]:
                    cgbf = CGBF(atom.pos(), power, atom.atid)
                    for alpha, coef in prims:
                        cgbf.add_primitive(alpha, coef)
                    bfs.append(cgbf)
                    shell.append(cgbf, len(bfs) - 1)
                shells.append(shell)
        self.bfs = bfs
        self.shells = shells

    def __len__(self):
        return len(self.bfs)

    def __iter__(self):
        return iter(self.bfs)

    def __getitem__(self, item):
        return self.bfs[item]
