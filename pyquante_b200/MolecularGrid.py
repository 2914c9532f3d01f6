"""Molecular integration grid of the DFT path on the GPU: the reference's
default grid (PyQuante/dft.py:174-176 builds MG2(atoms, 32, 1), and
PyQuante/MG2.py:95-130 builds it from per-atom grids and Becke's
partitioning).

Per atom: 32 Euler--Maclaurin radial shells with the SG-1 radii
(Gill, Johnson and Pople, Chem. Phys. Lett. 209, 506 (1993);
PyQuante/AtomicGrid.py:284-294)
    r_i = R i^2 / (n+1-i)^2,  w_i = 8 pi R^3 (n+1) i^5 / (n+1-i)^7,
each with the 194-point Lebedev rule (PyQuante/AtomicGrid.py:85-99,
pyquante_b200.Lebedev).  Becke's cell weights (J. Chem. Phys. 88, 2547
(1988), with the heteronuclear size adjustment of its appendix;
PyQuante/MolecularGrid.py:228-263) come from pqb_becke_weights, the basis
amplitudes on the points from pqb_grid_amps, the density from
pqb_grid_rowdot -- all on the device.
"""
import numpy as np
import torch

from . import Lebedev, _lib
from ._lib import ptr, stream_ptr

# SG-1 atomic radii (bohr) by atomic number, as the reference tabulates them
# (PyQuante/AtomicGrid.py:42-47)
POPLE_RADII = [None, 1.0000, 0.5882, 3.0769, 2.0513, 1.5385, 1.2308, 1.0256, 0.8791, 0.7692, 0.6839, 4.0909,
               3.1579, 2.5714, 2.1687, 1.8750, 1.6514, 1.4754, 1.3333]
# atomic size parameters of the heteronuclear Becke adjustment, as the
# reference tabulates them (PyQuante/AtomicGrid.py:26-40), Z <= 18
BRAGG = [None, 0.50, 2.00, 1.45, 1.05, 0.85, 0.70, 0.65, 0.60, 0.50, 2.25, 1.80, 1.50, 1.25, 1.10, 1.00, 1.00,
         1.00, 2.50]


def _check(rc, what):
    if rc != _lib.PQB_OK:
        raise _lib.EngineError(rc, what)


def atomic_points(atoms, nrad=32):
    """Host-side (npts, 4) x, y, z, w_radial * w_angular and the owning atom
    of every point (the unpartitioned atomic grids)."""
    ang = Lebedev.points()
    pts, owner = [], []
    for ia, (z, xyz) in enumerate(atoms):
        if z >= len(POPLE_RADII):
            raise ValueError("no SG-1 radius for Z = %d" % z)
        R = POPLE_RADII[z]
        i = np.arange(1, nrad + 1, dtype=np.float64)
        r = R * i * i * (nrad + 1 - i) ** -2.0
        w = 8.0 * np.pi * R ** 3 * (nrad + 1.0) * i ** 5 * (nrad + 1 - i) ** -7.0
        p = np.empty((nrad, len(ang), 4))
        p[:, :, :3] = r[:, None, None] * ang[None, :, :3] + np.asarray(xyz, dtype=np.float64)
        p[:, :, 3] = w[:, None] * ang[None, :, 3]
        pts.append(p.reshape(-1, 4))
        owner.append(np.full(nrad * len(ang), ia, dtype=np.int32))
    return np.concatenate(pts), np.concatenate(owner)


def becke_adjust(atoms):
    """nat x nat table a_ij of the heteronuclear adjustment
    mu' = mu + a_ij (1 - mu^2) (0 for equal atoms)."""
    nat = len(atoms)
    a = np.zeros((nat, nat))
    for i in range(nat):
        for j in range(nat):
            zi, zj = atoms[i][0], atoms[j][0]
            if i == j or zi == zj:
                continue
            chi = BRAGG[zi] / BRAGG[zj]
            u = (chi - 1.0) / (chi + 1.0)
            a[i, j] = min(max(u / (u * u - 1), -0.5), 0.5)
    return a


class MolecularGrid:
    """The reference's MG2 grid with its data on the GPU (points, weights,
    basis amplitudes bfgrid[npts, nbf], density[npts, 2])."""

    version = 2

    def __init__(self, atoms, nrad=32, fineness=1, **opts):
        self.atoms = atoms
        at = [(a.atno, tuple(float(c) for c in a.pos())) for a in atoms]
        self.nrad = nrad
        self.fineness = fineness
        pts, owner = atomic_points(at, nrad)
        self.ng = len(pts)
        self.device = torch.device("cuda", torch.cuda.current_device())
        dev = dict(dtype=torch.float64, device=self.device)
        self._pts0 = torch.as_tensor(pts, **dev).contiguous()
        self._owner = torch.as_tensor(owner, dtype=torch.int32, device=self.device)
        self._atoms = torch.as_tensor(np.array([xyz for _, xyz in at]).reshape(-1), **dev).contiguous()
        self._adj = torch.as_tensor(becke_adjust(at).reshape(-1), **dev).contiguous()
        w = torch.empty(self.ng, **dev)
        _check(_lib.load().pqb_becke_weights(self.ng, ptr(self._pts0), ptr(self._owner), len(at), ptr(self._atoms),
                                             ptr(self._adj), ptr(w), stream_ptr()), "pqb_becke_weights")
        self.xyzw = self._pts0.clone()
        self.xyzw[:, 3] = w
        self.bfgrid = None
        self.nbf = 0
        self.density = torch.zeros((self.ng, 2), **dev)

    def __len__(self):
        return self.ng

    def add_basis(self, bfs):
        """bfgrid[g, i] = amplitude of basis function i at point g."""
        from .engine import FunctionTable
        ft = FunctionTable(list(bfs), self.device.index)
        self.nbf = ft.n
        self.bfgrid = torch.empty((self.ng, self.nbf), dtype=torch.float64, device=self.device)
        _check(_lib.load().pqb_grid_amps(*ft.args(), self.ng, ptr(self.xyzw), ptr(self.bfgrid), stream_ptr()),
               "pqb_grid_amps")

    set_bf_amps = add_basis

    def set_density(self, D, Db=None):
        """density[:, 0] = sum_ij B_gi D_ij B_gj; density[:, 1] the same for
        Db (or a copy of the first column)."""
        lib = _lib.load()
        for col, M in ((0, D), (1, Db)):
            if M is None:
                self.density[:, 1] = self.density[:, 0]
                continue
            Mt = torch.as_tensor(np.asarray(M) if not isinstance(M, torch.Tensor) else M, dtype=torch.float64,
                                 device=self.device)
            BD = torch.matmul(self.bfgrid, Mt)
            out = torch.empty(self.ng, dtype=torch.float64, device=self.device)
            _check(lib.pqb_grid_rowdot(self.ng, self.nbf, ptr(BD), ptr(self.bfgrid), ptr(out), stream_ptr()),
                   "pqb_grid_rowdot")
            self.density[:, col] = out

    def setdens(self, D):
        self.set_density(D)

    def floor_density(self, tol=1e-9):
        self.density[self.density < tol] = 0.0

    def renormalize(self, nel):
        factor = nel / float(torch.dot(self.xyzw[:, 3], self.density.sum(1)))
        self.density *= factor

    def dens(self):
        return self.density[:, 0] + self.density[:, 1]

    def weights(self):
        return self.xyzw[:, 3]

    def points(self):
        return self.xyzw

    def get_nbf(self):
        return self.nbf

    def get_gamma(self):
        return None
