"""CPU oracle for the ERI / Fock-build path — TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may
import this module; the product (pyquante_b200) never does.

Two independent CPU sources of truth, both driven through ctypes:
  * the REFERENCE's own C engines, compiled from its sources by
    ``make -C oracle ref`` into oracle/_ref/ (Src/lib/utils/crys.c — the Rys
    engine PyQuante/CGBF.py:24 binds for get2ints — plus Src/chgp.c and
    Src/cints.c through include-shims, and ref_fock.c, a C driver with the
    loop of PyQuante/Ints.py:146-167);
  * this project's plain-C restatement (oracle/eri_oracle.c, built by
    ``make -C oracle``): Head-Gordon--Pople ERIs with a long-double Boys
    function, THO one-electron integrals, get2ints/getJ/getK.

The Python layer restates what the reference's Python 2 code does
(it cannot run here): the integral loop order and packing
(PyQuante/Ints.py:146-193), get2JmK (Ints.py:225-238), and the RHF loop
(PyQuante/hartree_fock.py:66-149 with LA2.geigh's Cholesky orthogonalisation,
PyQuante/LA2.py:47-75,113-131, and Convergence.DIIS, :73-136).

Parity pin: the restatement is checked against the compiled reference
(tests/test_oracle.py) and against the reference's own known answers
(Boys values of Src/lib/utils/tests/TestMath.c:18-20; RHF energies of
Tests/h2o.py:16 and Tests/h2.py:16; see tests/golden/).
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
BUILD_DIR = os.path.join(HERE, "_build")

_d = ctypes.c_double
_i = ctypes.c_int
_i64 = ctypes.c_int64
_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_i64p = ctypes.POINTER(ctypes.c_int64)

_libs = {}


def _load(name, path):
    if name not in _libs:
        if not os.path.exists(path):
            return None
        _libs[name] = ctypes.CDLL(path)
    return _libs[name]


def oracle_lib():
    lib = _load("oracle", os.path.join(BUILD_DIR, "liboracle.so"))
    if lib is None:
        raise RuntimeError("oracle not built: make -C oracle")
    lib.orc_boys.restype = _d
    lib.orc_boys.argtypes = [_i, _d]
    lib.orc_ijkl2intindex.restype = _i64
    lib.orc_ijkl2intindex.argtypes = [_i64] * 4
    lib.orc_get2ints.argtypes = [_i64, _dp, _i64p, _i64p, _dp, _dp, _dp, _dp, _dp]
    lib.orc_get1ints.argtypes = [_i64, _dp, _i64p, _i64p, _dp, _dp, _dp, _dp, _i64, _dp, _dp, _dp, _dp]
    lib.orc_getJK.argtypes = [_i64, _dp, _dp, _dp, _dp]
    lib.orc_contr_eri.restype = _d
    return lib


def ref_available():
    return all(os.path.exists(os.path.join(REF_DIR, f)) for f in
               ("libref_crys.so", "libref_chgp.so", "libref_cints.so", "libref_fock.so", "ref_fock"))


def ref_lib(which):
    """which in {'crys', 'chgp', 'cints', 'fock'}; None when not built."""
    lib = _load("ref_" + which, os.path.join(REF_DIR, "libref_%s.so" % which))
    if lib is None:
        return None
    if which == "crys":
        lib.coulomb_repulsion.restype = _d
        lib.coulomb_repulsion.argtypes = [_d, _d, _d, _d, _i, _i, _i, _d] * 4
        lib.contr_coulomb.restype = _d
        lib.contr_coulomb.argtypes = [_i, _dp, _dp, _dp, _d, _d, _d, _i, _i, _i] * 4
        lib.Fgamma.restype = _d
        lib.Fgamma.argtypes = [_d, _d]
        lib.Fm.restype = _d
        lib.Fm.argtypes = [_i, _d]
    elif which == "chgp":
        lib.ref_chgp_hrr.restype = _d
        lib.ref_chgp_hrr.argtypes = [_d, _d, _d, _d, _i, _i, _i, _d] * 4
        lib.ref_chgp_vrr.restype = _d
        lib.ref_chgp_vrr.argtypes = ([_d, _d, _d, _d, _i, _i, _i, _d] + [_d, _d, _d, _d, _d] +
                                     [_d, _d, _d, _d, _i, _i, _i, _d] + [_d, _d, _d, _d, _d] + [_i])
        lib.ref_chgp_contr.restype = _d
        lib.ref_chgp_contr.argtypes = [_i, _dp, _dp, _dp, _dp, _ip] * 4
        lib.ref_chgp_Fgamma.restype = _d
        lib.ref_chgp_Fgamma.argtypes = [_d, _d]
    elif which == "cints":
        lib.ref_cints_coulomb_repulsion.restype = _d
        lib.ref_cints_coulomb_repulsion.argtypes = [_d, _d, _d, _d, _i, _i, _i, _d] * 4
        for f in ("ref_cints_overlap", "ref_cints_kinetic"):
            getattr(lib, f).restype = _d
            getattr(lib, f).argtypes = [_d, _i, _i, _i, _d, _d, _d] * 2
        lib.ref_cints_nuclear.restype = _d
        lib.ref_cints_nuclear.argtypes = [_d, _d, _d, _d, _i, _i, _i, _d] * 2 + [_d, _d, _d]
        lib.ref_cints_ijkl2intindex.restype = _i
        lib.ref_cints_ijkl2intindex.argtypes = [_i] * 4
        lib.ref_cints_Fgamma.restype = _d
        lib.ref_cints_Fgamma.argtypes = [_d, _d]
    elif which == "fock":
        lib.ref_get2ints.restype = _i
        lib.ref_get2ints.argtypes = [_i64, _dp, _i64p, _i64p, _dp, _dp, _dp, _dp, _dp, _i]
        lib.ref_get2JmK.argtypes = [_i64, _dp, _dp, _dp]
        lib.ref_ijkl2intindex64.restype = _i64
        lib.ref_ijkl2intindex64.argtypes = [_i64] * 4
        lib.ref_time_rows.restype = _d
        lib.ref_time_rows.argtypes = [_i64, _dp, _i64p, _i64p, _dp, _dp, _dp, _dp, _i64p, _i64, _i, _i64p, _dp]
    return lib


# ------------------------------------------------------------------ basis --
def _fact2(n):
    r = 1
    while n > 1:
        r *= n
        n -= 2
    return r


def prim_norm(alpha, powers):
    """Src/lib/primitive-gto.c:76-83."""
    l, m, n = powers
    L = l + m + n
    return np.sqrt(2.0 ** (2 * L + 1.5) * alpha ** (L + 1.5) /
                   (_fact2(2 * l - 1) * _fact2(2 * m - 1) * _fact2(2 * n - 1) * np.pi ** 1.5))


SYM2POWERS = {
    "S": [(0, 0, 0)],
    "P": [(1, 0, 0), (0, 1, 0), (0, 0, 1)],
    "D": [(2, 0, 0), (1, 1, 0), (1, 0, 1), (0, 2, 0), (0, 1, 1), (0, 0, 2)],
}


class BF:
    """One contracted function as PyQuante's BasisSet builds it
    (PyQuante/Basis/basis.py:27-46, CGBF.py:27-75): norm 1, per-primitive
    per-component norms."""

    def __init__(self, origin, powers, prims):
        self.origin = tuple(float(c) for c in origin)
        self.powers = tuple(powers)
        self.pexps = [float(a) for a, _ in prims]
        self.pcoefs = [float(c) for _, c in prims]
        self.pnorms = [prim_norm(a, powers) for a in self.pexps]
        self.norm = 1.0


def build_basis(atoms, basis_data):
    """atoms: [(Z, (x, y, z) bohr)], basis_data: {Z: [(sym, [(exp, coef)])]}."""
    bfs = []
    for z, xyz in atoms:
        for sym, prims in basis_data[z]:
            for p in SYM2POWERS[sym]:
                bfs.append(BF(xyz, p, prims))
    return bfs


class Table:
    """Flat per-function arrays (the layout ref_fock.c / eri_oracle.c read)."""

    def __init__(self, bfs):
        self.nbf = len(bfs)
        self.origin = np.ascontiguousarray([bf.origin for bf in bfs], dtype=np.float64).reshape(-1)
        self.powers = np.ascontiguousarray([bf.powers for bf in bfs], dtype=np.int64).reshape(-1)
        off = [0]
        for bf in bfs:
            off.append(off[-1] + len(bf.pexps))
        self.prim_off = np.array(off, dtype=np.int64)
        self.exps = np.array([e for bf in bfs for e in bf.pexps], dtype=np.float64)
        self.coefs = np.array([c for bf in bfs for c in bf.pcoefs], dtype=np.float64)
        self.pnorms = np.array([c for bf in bfs for c in bf.pnorms], dtype=np.float64)
        self.norms = np.array([bf.norm for bf in bfs], dtype=np.float64)

    def args(self):
        P = lambda a, t: a.ctypes.data_as(t)  # noqa: E731
        return (self.nbf, P(self.origin, _dp), P(self.powers, _i64p), P(self.prim_off, _i64p),
                P(self.exps, _dp), P(self.coefs, _dp), P(self.pnorms, _dp), P(self.norms, _dp))

    def write(self, path):
        with open(path, "wb") as f:
            np.array([self.nbf, len(self.exps)], dtype=np.int64).tofile(f)
            for a in (self.origin, self.powers, self.prim_off, self.exps, self.coefs, self.pnorms, self.norms):
                a.tofile(f)


def nquartets(nbf):
    P = nbf * (nbf + 1) // 2
    return P * (P + 1) // 2


def ijkl2intindex(i, j, k, l):
    if i < j:
        i, j = j, i
    if k < l:
        k, l = l, k
    ij, kl = i * (i + 1) // 2 + j, k * (k + 1) // 2 + l
    if ij < kl:
        ij, kl = kl, ij
    return ij * (ij + 1) // 2 + kl


# -------------------------------------------------------------- integrals --
def ref_get2ints(bfs, nproc=1):
    """Every unique (ij|kl) from the reference's compiled Rys engine."""
    lib = ref_lib("fock")
    if lib is None:
        raise RuntimeError("reference not built: make -C oracle ref")
    t = Table(bfs)
    out = np.zeros(nquartets(t.nbf))
    rc = lib.ref_get2ints(*t.args(), out.ctypes.data_as(_dp), nproc)
    if rc != 0:
        raise RuntimeError("ref_get2ints failed (%d)" % rc)
    return out


def _carr(x):
    return (ctypes.c_double * len(x))(*x)


def ref_contr(a, b, c, d):
    """CGBF.coulomb (PyQuante/CGBF.py:191-199) on the reference's compiled
    crys.contr_coulomb for one function quartet."""
    crys = ref_lib("crys")
    args = []
    for f in (a, b, c, d):
        args += [len(f.pexps), _carr(f.pexps), _carr(f.pcoefs), _carr(f.pnorms), *f.origin, *f.powers]
    return crys.contr_coulomb(*args) * a.norm * b.norm * c.norm * d.norm


def orc_contr(a, b, c, d):
    """The same quartet from this project's C restatement (HGP)."""
    t = Table([a, b, c, d])
    out = np.zeros(nquartets(4))
    oracle_lib().orc_get2ints(*t.args(), out.ctypes.data_as(_dp))
    return out[ijkl2intindex(0, 1, 2, 3)]


def orc_get2ints(bfs):
    """Every unique (ij|kl) from this project's C restatement (HGP)."""
    t = Table(bfs)
    out = np.zeros(nquartets(t.nbf))
    oracle_lib().orc_get2ints(*t.args(), out.ctypes.data_as(_dp))
    return out


def orc_get1ints(bfs, atoms):
    t = Table(bfs)
    n = t.nbf
    S = np.zeros((n, n))
    h = np.zeros((n, n))
    xyz = np.ascontiguousarray([p for _, p in atoms], dtype=np.float64).reshape(-1)
    z = np.array([float(zz) for zz, _ in atoms])
    oracle_lib().orc_get1ints(*t.args(), len(atoms), xyz.ctypes.data_as(_dp), z.ctypes.data_as(_dp),
                              S.ctypes.data_as(_dp), h.ctypes.data_as(_dp))
    return S, h


def ref_get1ints(bfs, atoms):
    """PyQuante/Ints.py:73-87 over the reference's compiled cints
    (CGBF.overlap/kinetic/nuclear -> PGBF -> cints, PyQuante/PGBF.py:72-99)."""
    lib = ref_lib("cints")
    if lib is None:
        raise RuntimeError("reference not built: make -C oracle ref")
    n = len(bfs)
    S = np.zeros((n, n))
    h = np.zeros((n, n))
    for i, a in enumerate(bfs):
        for j, b in enumerate(bfs):
            s = t = v = 0.0
            for ea, ca, na in zip(a.pexps, a.pcoefs, a.pnorms):
                for eb, cb, nb in zip(b.pexps, b.pcoefs, b.pnorms):
                    s += ca * cb * na * nb * lib.ref_cints_overlap(ea, *a.powers, *a.origin, eb, *b.powers, *b.origin)
                    t += ca * cb * na * nb * lib.ref_cints_kinetic(ea, *a.powers, *a.origin, eb, *b.powers, *b.origin)
                    for z, c in atoms:
                        v += z * ca * cb * lib.ref_cints_nuclear(*a.origin, na, *a.powers, ea,
                                                                 *b.origin, nb, *b.powers, eb, *c)
            S[i, j] = a.norm * b.norm * s
            h[i, j] = a.norm * b.norm * (t + v)
    return S, h


def unpack(ints, nbf):
    """Full (n,n,n,n) tensor from the packed array (small n only)."""
    idx = np.zeros((nbf, nbf, nbf, nbf), dtype=np.int64)
    r = np.arange(nbf)
    i, j, k, l = np.meshgrid(r, r, r, r, indexing="ij")
    a, b = np.maximum(i, j), np.minimum(i, j)
    c, d = np.maximum(k, l), np.minimum(k, l)
    ij, kl = a * (a + 1) // 2 + b, c * (c + 1) // 2 + d
    hi, lo = np.maximum(ij, kl), np.minimum(ij, kl)
    idx[...] = hi * (hi + 1) // 2 + lo
    return np.asarray(ints)[idx]


def getJK(ints, D):
    """J_ij = sum_kl (ij|kl) D_kl, K_ij = sum_kl (ik|jl) D_kl (PyQuante/Ints.py:195-223)."""
    n = D.shape[0]
    full = unpack(ints, n)
    J = np.einsum("ijkl,kl->ij", full, D)
    K = np.einsum("ikjl,kl->ij", full, D)
    return J, K


def get2JmK(ints, D):
    J, K = getJK(ints, D)
    return 2 * J - K


# -------------------------------------------------------------------- SCF --
def geigh(H, S):
    X = np.linalg.inv(np.linalg.cholesky(S)).T
    e, v = np.linalg.eigh(X.T @ H @ X)
    return e, X @ v


def enuke(atoms):
    e = 0.0
    for i, (zi, ri) in enumerate(atoms):
        for zj, rj in atoms[:i]:
            e += zi * zj / np.linalg.norm(np.subtract(ri, rj))
    return e


def rhf(atoms, S, h, ints, nclosed, conv=1e-10, maxiter=100, diis=False):
    """PyQuante/hartree_fock.py:66-149 (DIIS per Convergence.py:73-136, with a
    subspace of the last 8 Fock matrices and no extrapolation once the
    commutator error is at rounding level: the reference's unbounded DIIS can
    drift off the SCF solution near convergence)."""
    en = enuke(atoms)
    orbe, orbs = geigh(h, S)
    eold = 0.0
    Fs, Es = [], []
    energy = 0.0
    for _ in range(maxiter):
        D = orbs[:, :nclosed] @ orbs[:, :nclosed].T
        F = h + get2JmK(ints, D)
        err = (F @ D @ S - S @ D @ F).ravel()
        if diis and abs(err).max() >= 1e-13:
            Fs.append(F)
            Es.append(err)
            del Fs[:-8], Es[:-8]
            m = len(Es)
            a = np.zeros((m + 1, m + 1))
            a[:m, :m] = np.array(Es) @ np.array(Es).T
            a[m, :m] = a[:m, m] = -1.0
            b = np.zeros(m + 1)
            b[m] = -1.0
            c = np.linalg.solve(a, b)
            F = sum(c[i] * Fs[i] for i in range(m))
        orbe, orbs = geigh(F, S)
        energy = float((D * h).sum() + (D * F).sum() + en)
        if abs(energy - eold) < conv:
            break
        eold = energy
    return energy, orbe, orbs


# -------------------------------------------------------------------- MP2 --
def transform_ints_mp2_loops(ints, orbs, nclosed):
    """PyQuante/MP.py:20-75 (TransformIntsMP2) step by step: sigma -> b,
    mu -> a, eta -> j, nu -> i over the packed AO integrals, stored at
    ijkl2intindex(a, i, b, j) of a packed MO array.  O(N^5) Python loops:
    small bases only."""
    nbf, nmo = orbs.shape
    totlen = nmo * (nmo + 1) * (nmo * nmo + nmo + 2) // 8
    occs, mos, bfs = range(nclosed), range(nmo), range(nbf)
    temp = np.zeros((nbf, nbf, nclosed, nbf))
    tempvec = np.zeros(nbf)
    for mu in bfs:
        for nu in bfs:
            for eta in bfs:
                for b in occs:
                    for sigma in bfs:
                        tempvec[sigma] = ints[ijkl2intindex(mu, nu, sigma, eta)]
                    temp[mu, nu, b, eta] = orbs[:, b] @ tempvec
    temp2 = np.zeros((nclosed, nbf, nclosed, nbf))
    for nu in bfs:
        for eta in bfs:
            for b in occs:
                for a in occs:
                    temp2[a, nu, b, eta] = orbs[:, a] @ temp[:, nu, b, eta]
    temp = np.zeros((nclosed, nbf, nclosed, nmo))
    for a in occs:
        for nu in bfs:
            for b in occs:
                for j in mos:
                    temp[a, nu, b, j] = orbs[:, j] @ temp2[a, nu, b, :]
    moints = np.zeros(totlen)
    for a in occs:
        for j in mos:
            for b in occs:
                for i in mos:
                    moints[ijkl2intindex(a, i, b, j)] = orbs[:, i] @ temp[a, :, b, j]
    return moints


def transform_ovov(ints, orbs, nclosed, nmo=None):
    """(a i|b j) = sum C_mu,a C_nu,i C_la,b C_si,j (mu nu|la si) as a dense
    [nocc, nmo, nocc, nmo] array (numpy einsum over the unpacked integrals)."""
    nbf = orbs.shape[0]
    C = orbs if nmo is None else orbs[:, :nmo]
    full = unpack(ints, nbf)
    Co = orbs[:, :nclosed]
    t = np.einsum("mnls,sj->mnlj", full, C)
    t = np.einsum("mnlj,lb->mnbj", t, Co)
    t = np.einsum("mnbj,ni->mibj", t, C)
    return np.einsum("mibj,ma->aibj", t, Co)


def mp2(ints, orbs, orbe, nclosed, nvirt):
    """PyQuante/MP.py:77-97: sum over occupied a, b and virtual r, s of
    (ar|bs)(2(ar|bs) - (as|br))/(e_a + e_b - e_r - e_s)."""
    V = transform_ovov(ints, orbs, nclosed)[:, nclosed:nclosed + nvirt, :, nclosed:nclosed + nvirt]
    eo, ev = orbe[:nclosed], orbe[nclosed:nclosed + nvirt]
    den = eo[:, None, None, None] + eo[None, None, :, None] - ev[None, :, None, None] - ev[None, None, None, :]
    return float((V * (2 * V - V.transpose(0, 3, 2, 1)) / den).sum())


# --------------------------------------------------------------- gradient --
def _deriv_parts(bf, x):
    """d phi / dA_x of a contracted function on centre A as up to two
    functions: raising, sum_p c_p N_p(l) 2 alpha_p x^(l+1) e^(-alpha_p r^2),
    and lowering, -l sum_p c_p N_p(l) x^(l-1) e^(-alpha_p r^2).  (The
    reference builds the same derivative from normalised primitives,
    PyQuante/AnalyticDerivatives.py:457-674.)  BF renormalises per
    primitive, so the coefficients divide that norm back out."""
    parts = []
    up = list(bf.powers)
    up[x] += 1
    c_up = [c * n * 2.0 * a / prim_norm(a, up) for a, c, n in zip(bf.pexps, bf.pcoefs, bf.pnorms)]
    parts.append(BF(bf.origin, up, list(zip(bf.pexps, c_up))))
    if bf.powers[x] > 0:
        dn = list(bf.powers)
        dn[x] -= 1
        l = bf.powers[x]
        c_dn = [-l * c * n / prim_norm(a, dn) for a, c, n in zip(bf.pexps, bf.pcoefs, bf.pnorms)]
        parts.append(BF(bf.origin, dn, list(zip(bf.pexps, c_dn))))
    return parts


def rhf_gradient(atoms, basis_data, D, Q):
    """dE/dR for closed-shell RHF, the formula of PyQuante/force.py:48-70
    (Szabo eq. C.12) with D = C_occ C_occ^T and Q = C_occ e_occ C_occ^T
    (Wavefunction.py:143-149):
      dE/dR_a = 2 tr(D dH/dR_a) + tr(D dG[D]/dR_a) - 2 tr(Q dS/dR_a) + dE_nuc/dR_a,
    dG[D]_ij = sum_kl D_kl [2 d(ij|kl) - (d(ik|jl) + d(il|kj))/2]
    (force.py:310-357).  With D symmetric, every derivative of a product of
    functions reduces to four times the derivative of the first one, and the
    operator derivative of the nuclear attraction follows from translational
    invariance.  Integrals come from this oracle's C restatement over the
    basis extended by the derivative functions; meant for small bases."""
    bfs = build_basis(atoms, basis_data)
    n = len(bfs)
    atid = []
    for ia, (z, _) in enumerate(atoms):
        for sym, _ in basis_data[z]:
            atid += [ia] * len(SYM2POWERS[sym])
    ext = list(bfs)
    dparts = {}
    for i, bf in enumerate(bfs):
        for x in range(3):
            ps = _deriv_parts(bf, x)
            dparts[i, x] = list(range(len(ext), len(ext) + len(ps)))
            ext += ps
    m = len(ext)
    _, h = orc_get1ints(ext, atoms)
    S, T = orc_get1ints(ext, [])
    Va = [orc_get1ints(ext, [at])[1] - T for at in atoms]
    # (p j | k l) for p in ext, j, k, l in the original basis, one contracted
    # integral at a time (p over the derivative functions only)
    lib = oracle_lib()
    arr = [(len(f.pexps), _carr(f.pexps), _carr(f.pcoefs), _carr(f.pnorms), _carr(f.origin),
            (ctypes.c_int * 3)(*f.powers)) for f in ext]
    base = orc_get2ints(bfs)
    I = np.empty((m, n, n, n))
    for j in range(n):
        for k in range(n):
            for l in range(n):
                for p in range(n):
                    I[p, j, k, l] = base[ijkl2intindex(p, j, k, l)]
    for p in range(n, m):
        for j in range(n):
            for k in range(n):
                for l in range(k + 1):
                    I[p, j, k, l] = I[p, j, l, k] = lib.orc_contr_eri(*arr[p], *arr[j], *arr[k], *arr[l])
    Jp = np.einsum("pjkl,kl->pj", I, D)
    Kp = np.einsum("pkjl,kl->pj", I, D)
    grad = np.zeros((len(atoms), 3))
    for a, (za, ra) in enumerate(atoms):
        for x in range(3):
            g = 0.0
            for i in range(n):
                dsum = lambda M: sum(M[p, :n] for p in dparts[i, x])  # noqa: E731
                if atid[i] == a:
                    g += 4.0 * D[i] @ dsum(h)
                    g += 4.0 * D[i] @ (2.0 * sum(Jp[p] for p in dparts[i, x]) - sum(Kp[p] for p in dparts[i, x]))
                    g -= 4.0 * Q[i] @ dsum(S)
                # operator part of the attraction to nucleus a
                g -= 4.0 * D[i] @ sum(Va[a][p, :n] for p in dparts[i, x])
            for b, (zb, rb) in enumerate(atoms):
                if b != a:
                    d = np.subtract(rb, ra)
                    g += za * zb * d[x] / np.linalg.norm(d) ** 3
            grad[a, x] = g
    return grad


# -------------------------------------------------------------------- DFT --
# The default grid and SVWN functional of the reference's dft()
# (PyQuante/dft.py:116-215 with MG2 grids, PyQuante/MG2.py:50-250):
# per atom, 32 Euler--Maclaurin radial shells (PyQuante/AtomicGrid.py:284-294,
# SG-1 radii) times the 194-point Lebedev rule, Becke partitioning with the
# heteronuclear size adjustment (PyQuante/MolecularGrid.py:228-263), basis
# amplitudes, density, SVWN (PyQuante/DFunctionals.py:76-138,319-389,603-623),
# Fxc = sum_g w v phi_i phi_j (PyQuante/dft.py:29-65).
def dft_grid(atoms, nrad=32):
    """(npts, 4) x, y, z, w of the reference's default molecular grid;
    atoms: [(Z, (x, y, z))] in bohr."""
    from pyquante_b200 import Lebedev
    from pyquante_b200.MolecularGrid import BRAGG, POPLE_RADII
    ang = Lebedev.points()
    pts = []
    owner = []
    for ia, (z, xyz) in enumerate(atoms):
        R = POPLE_RADII[z]
        for i in range(1, nrad + 1):
            w = 8.0 * np.pi * R ** 3 * (nrad + 1.0) * i ** 5 * (nrad + 1 - i) ** -7.0
            r = R * i * i * (nrad + 1 - i) ** -2.0
            for x, y, zz, wa in ang:
                pts.append((r * x + xyz[0], r * y + xyz[1], r * zz + xyz[2], w * wa))
                owner.append(ia)
    pts = np.array(pts)
    nat = len(atoms)
    pos = np.array([xyz for _, xyz in atoms], dtype=float)

    def cell(i, p):
        s = 1.0
        rip = np.linalg.norm(pos[i] - p)
        for j in range(nat):
            if j == i:
                continue
            rjp = np.linalg.norm(pos[j] - p)
            rij = np.linalg.norm(pos[i] - pos[j])
            mu = (rip - rjp) / rij
            if atoms[i][0] != atoms[j][0]:
                chi = BRAGG[atoms[i][0]] / BRAGG[atoms[j][0]]
                u = (chi - 1.0) / (chi + 1.0)
                a = min(max(u / (u * u - 1), -0.5), 0.5)
                mu += a * (1 - mu * mu)
            for _ in range(3):
                mu = 1.5 * mu - 0.5 * mu ** 3
            s *= 0.5 * (1 - mu)
        return s

    for g in range(len(pts)):
        p = pts[g, :3]
        cells = [cell(j, p) for j in range(nat)]
        pts[g, 3] *= cells[owner[g]] / sum(cells)
    return pts


def bf_amps(bfs, pts):
    """(npts, nbf) amplitudes: norm * sum_p c_p N_p x^l y^m z^n exp(-a r^2)."""
    B = np.zeros((len(pts), len(bfs)))
    for k, bf in enumerate(bfs):
        d = pts[:, :3] - np.array(bf.origin)
        r2 = (d * d).sum(1)
        poly = d[:, 0] ** bf.powers[0] * d[:, 1] ** bf.powers[1] * d[:, 2] ** bf.powers[2]
        B[:, k] = bf.norm * poly * sum(c * n * np.exp(-a * r2) for a, c, n in zip(bf.pexps, bf.pcoefs, bf.pnorms))
    return B


def svwn(rhoa, rhob, tol=1e-10):
    """(fxc, vxc_a, vxc_b) per point: Slater exchange with X-alpha 2/3 per
    spin plus VWN correlation (the reference's xs and cvwn)."""
    fac = -2.25 * (2.0 / 3.0) * (3.0 / 4.0 / np.pi) ** (1.0 / 3.0)
    n = len(rhoa)
    f = np.zeros(n)
    va = np.zeros(n)
    vb = np.zeros(n)

    def xx(x, b, c):
        return x * x + b * x + c

    def eps(x, a, x0, b, c):
        q = np.sqrt(4 * c - b * b)
        return a * (np.log(x * x / xx(x, b, c)) - b * (x0 / xx(x0, b, c)) * np.log((x - x0) ** 2 / xx(x, b, c))
                    + (2 * b / q) * (1 - (x0 * (2 * x0 + b) / xx(x0, b, c))) * np.arctan(q / (2 * x + b)))

    def deps(x, a, x0, b, c):
        q = np.sqrt(4 * c - b * b)
        return a * (2 / x - (2 * x + b) / xx(x, b, c) - 4 * b / ((2 * x + b) ** 2 + q * q) - (b * x0 / xx(x0, b, c))
                    * (2 / (x - x0) - (2 * x + b) / xx(x, b, c) - 4 * (2 * x0 + b) / ((2 * x + b) ** 2 + q * q)))

    P = (0.0310907, -0.10498, 3.72744, 12.9352)
    Fm = (0.01554535, -0.32500, 7.06042, 13.0045)
    for g in range(n):
        for rho, vv in ((rhoa[g], va), (rhob[g], vb)):
            r = 0.0 if rho < tol else rho
            r3 = r ** (1.0 / 3.0)
            f[g] += fac * r * r3
            vv[g] += (4.0 / 3.0) * fac * r3
        rho = rhoa[g] + rhob[g]
        if rho < tol:
            continue
        zeta = (rhoa[g] - rhob[g]) / rho
        x = (3.0 / 4.0 / np.pi / rho) ** (1.0 / 6.0)
        ep, dep = eps(x, *P), deps(x, *P)
        gz = 1.125 * ((1 + zeta) ** (4.0 / 3.0) + (1 - zeta) ** (4.0 / 3.0) - 2)
        if gz < tol:
            f[g] += ep * rho
            va[g] += ep - (x / 6.0) * dep
            vb[g] += ep - (x / 6.0) * dep
            continue
        ef, def_ = eps(x, *Fm), deps(x, *Fm)
        e = ep + gz * (ef - ep)
        f[g] += e * rho
        dg = 1.5 * ((1 + zeta) ** (1.0 / 3.0) - (1 - zeta) ** (1.0 / 3.0))
        dx = dep + gz * (def_ - dep)
        dgg = (ef - ep) * dg
        va[g] += e - (x / 6.0) * dx + dgg * (1 - zeta)
        vb[g] += e - (x / 6.0) * dx - dgg * (1 + zeta)
    return f, va, vb


def get_xc(B, w, D, nel):
    """(Exc, Fxc) of PyQuante/dft.py:29-65 for a closed-shell (spin-averaged)
    density D = C_occ C_occ^T: rho_a = rho_b = sum_ij B_i D_ij B_j, floored at
    1e-9, renormalised to nel electrons."""
    rho = ((B @ D) * B).sum(1)
    rho[rho < 1e-9] = 0.0
    rho *= nel / (w @ (2 * rho))
    f, va, _ = svwn(rho, rho)
    return float(w @ f), B.T @ (B * (w * va)[:, None])


def dft(atoms, S, h, ints, bfs, nclosed, conv=1e-10, maxiter=100):
    """PyQuante/dft.py:116-215 (closed shell, SVWN): F = h + 2J + Fxc,
    E = 2 tr(D h) + 2 tr(D J) + Exc + E_nuc, with the DIIS of rhf()."""
    pts = dft_grid(atoms)
    B = bf_amps(bfs, pts)
    w = pts[:, 3]
    nel = 2 * nclosed
    en = enuke(atoms)
    orbe, orbs = geigh(h, S)
    eold = 0.0
    Fs, Es = [], []
    energy = 0.0
    for _ in range(maxiter):
        D = orbs[:, :nclosed] @ orbs[:, :nclosed].T
        J, _ = getJK(ints, D)
        exc, fxc = get_xc(B, w, D, nel)
        F = h + 2 * J + fxc
        err = (F @ D @ S - S @ D @ F).ravel()
        if abs(err).max() >= 1e-13:
            Fs.append(F)
            Es.append(err)
            del Fs[:-8], Es[:-8]
            m = len(Es)
            a = np.zeros((m + 1, m + 1))
            a[:m, :m] = np.array(Es) @ np.array(Es).T
            a[m, :m] = a[:m, m] = -1.0
            b = np.zeros(m + 1)
            b[m] = -1.0
            c = np.linalg.solve(a, b)
            F = sum(c[i] * Fs[i] for i in range(m))
        orbe, orbs = geigh(F, S)
        energy = float(2 * (D * h).sum() + 2 * (D * J).sum() + exc + en)
        if abs(energy - eold) < conv:
            break
        eold = energy
    return energy, orbe, orbs
