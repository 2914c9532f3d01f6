"""PyQuante's integral API (PyQuante/Ints.py:35-238) on the B200 engine.

    S, h, Ints = getints(bfs, atoms)       # S, h: numpy (n x n); Ints: PackedInts
    G = get2JmK(Ints, D)                    # D numpy or torch -> same type

``Ints`` holds every unique (ij|kl) (i>=j, k>=l, ij>=kl) at
``ijkl2intindex(i,j,k,l)`` in a float64 CUDA tensor (64-bit index, so nbf >= 304
works, unlike Src/cints.c:413-425).  ``getints(..., direct=True)`` instead
returns a DirectInts handle: nothing is stored and getJ/getK/get2JmK run the
fused integral-direct kernels (``precision='fp64'|'mixed'``, ``schwarz``,
``fp32_threshold`` options).

Differences from the reference that are deliberate:
  * no module-global ``jints``/``kints`` caches (Ints.py:31-33,169-193): the
    stored-integral J/K kernel reads the packed array directly, so results
    never depend on which ``get2ints`` ran last;
  * everything runs on the GPU; there is no CPU fallback.
"""
import numpy as np
import torch

from . import _lib
from .Basis.basis import BasisSet, sym2powerlist  # noqa: F401  (re-exported like the reference)
from .engine import BasisEngine, FunctionTable, eri_functions, jk_packed, oneint

__all__ = ["getbasis", "getints", "get1ints", "get2ints", "getJ", "getK", "get2JmK", "getJK2", "getS", "getT", "getV",
           "ijkl2intindex", "PackedInts", "DirectInts", "sym2powerlist"]


def ijkl2intindex(i, j, k, l):
    """Canonical packed index, 64-bit (same ordering as Src/cints.c:413-425)."""
    return int(_lib.load().pqb_ijkl2intindex(i, j, k, l))


def _bfs_list(bfs):
    return list(bfs.bfs) if hasattr(bfs, "bfs") else list(bfs)


def _engine_for(bfs):
    """One BasisEngine per basis object, cached on it."""
    holder = bfs if hasattr(bfs, "bfs") else None
    eng = getattr(holder, "_pqb_engine", None) if holder is not None else None
    if eng is None:
        eng = BasisEngine(_bfs_list(bfs))
        if holder is not None:
            holder._pqb_engine = eng
    return eng


def getbasis(atoms, basis_data=None, **opts):
    """bfs = getbasis(atoms, basis_data=None): a BasisSet (default 6-31G**)."""
    return BasisSet(atoms, basis_data, **opts)


def _oneint_functions(bfs, atoms):
    ctx = _lib.context()
    ft = FunctionTable(bfs, ctx.device)
    S, T, V = oneint(ft, atoms, ctx)
    return S.cpu().numpy(), T.cpu().numpy(), V.cpu().numpy()


def get1ints(bfs, atoms):
    """Overlap S and h = T + V_nuc (PyQuante/Ints.py:73-87), numpy arrays."""
    S, T, V = _oneint_functions(_bfs_list(bfs), atoms)
    return S, T + V


def getS(bfs):
    return _oneint_functions(_bfs_list(bfs), [])[0]


def getT(bfs):
    return _oneint_functions(_bfs_list(bfs), [])[1]


def getV(bfs, atoms):
    return _oneint_functions(_bfs_list(bfs), atoms)[2]


class PackedInts:
    """Packed unique two-electron integrals on the GPU, indexable like the
    reference's ``array('d')`` (``Ints[ijkl2intindex(i,j,k,l)]``)."""

    def __init__(self, tensor, nbf, engine=None):
        self.tensor = tensor
        self.nbf = nbf
        self.engine = engine

    @property
    def tensor(self):
        return self._tensor

    @tensor.setter
    def tensor(self, t):
        # a new integral array invalidates every J/K remembered for the old one
        self._tensor = t
        self.__dict__.pop("_jk_cache", None)

    def __len__(self):
        return self.tensor.numel()

    def __getitem__(self, idx):
        v = self.tensor[idx]
        return float(v) if v.dim() == 0 else v.cpu().numpy()

    def __array__(self, dtype=None, copy=None):
        a = self.tensor.cpu().numpy()
        return a if dtype is None else a.astype(dtype)

    def numpy(self):
        return self.tensor.cpu().numpy()


class DirectInts:
    """Integral-direct handle: J/K are rebuilt from the basis on every call."""

    def __init__(self, engine, precision="fp64", schwarz=1e-12, fp32_threshold=1e-5):
        if precision not in ("fp64", "mixed"):
            raise ValueError("precision must be 'fp64' or 'mixed'")
        self.engine = engine
        self.nbf = engine.nbf
        self.precision = precision
        self.schwarz = schwarz
        self.fp32_threshold = fp32_threshold
        engine.plan(schwarz, fp32_threshold)

    def jk(self, D):
        return self.engine.jk(D, self.precision, self.schwarz, self.fp32_threshold)

    def j(self, D):
        return self.engine.j(D, self.precision, self.schwarz, self.fp32_threshold)

    def synchronize(self):
        """Wait for the engine device's current stream (host results complete)."""
        torch.cuda.current_stream(self.engine.device).synchronize()

    def get2jmk_host(self, D, G, stream=None):
        """G = 2J - K into the host array G for the host density D, by one
        C-ABI call (copies in and out on the stream; synchronise before
        reading G)."""
        return self.engine.get2jmk_host(D, G, self.precision, self.schwarz, self.fp32_threshold, stream)


def _general_packed(bfs, eng):
    """Packed integrals for function lists that do not form s/p/d shells:
    one GPU thread per unique function quartet (Rys, any L with total <= 9)."""
    n = len(bfs)
    idx = []
    for i in range(n):
        for j in range(i + 1):
            for k in range(n):
                for l in range(k + 1):
                    if i * (i + 1) // 2 + j <= k * (k + 1) // 2 + l:
                        idx.append((i, j, k, l))
    q = np.array(idx, dtype=np.int32).reshape(-1, 4)
    vals = eri_functions(eng.ft, q, eng.ctx)
    P = n * (n + 1) // 2
    out = torch.zeros(P * (P + 1) // 2, dtype=torch.float64, device=eng.device)
    ij = q[:, 0].astype(np.int64) * (q[:, 0] + 1) // 2 + q[:, 1]
    kl = q[:, 2].astype(np.int64) * (q[:, 2] + 1) // 2 + q[:, 3]
    pos = kl * (kl + 1) // 2 + ij
    out[torch.from_numpy(pos).to(eng.device)] = vals
    return out


def get2ints(bfs, **opts):
    """All unique (ij|kl) (PyQuante/Ints.py:146-167), or a DirectInts handle
    with ``direct=True``."""
    eng = _engine_for(bfs)
    if opts.get("direct", False):
        return DirectInts(eng, opts.get("precision", "fp64"), opts.get("schwarz", 1e-12),
                          opts.get("fp32_threshold", 1e-5))
    t = eng.eri_packed() if eng.has_shells else _general_packed(eng.bfs, eng)
    return PackedInts(t, eng.nbf, eng)


def getints(bfs, atoms, **opts):
    """(S, h, Ints) as PyQuante/Ints.py:66-71."""
    S, h = get1ints(bfs, atoms)
    return S, h, get2ints(bfs, **opts)


def _as_device(D, like_device=None):
    if isinstance(D, torch.Tensor):
        dev = D.device if D.is_cuda else (like_device or torch.device("cuda", torch.cuda.current_device()))
        return D.to(device=dev, dtype=torch.float64).contiguous(), True
    dev = like_device or torch.device("cuda", torch.cuda.current_device())
    return torch.as_tensor(np.asarray(D, dtype=np.float64), device=dev).contiguous(), False


def _back(x, orig):
    if isinstance(orig, torch.Tensor):
        return x.to(orig.device)
    return x.cpu().numpy()


_JK_CACHE = 2   # densities remembered per integral object (uhf: alpha and beta)


def _jk(Ints, D, coulomb_only=False):
    """J and K of D.  One build gives both, and PyQuante's callers ask for
    them one at a time: getJ(Ints, D) then getK(Ints, D), and uhf does
    getJ(Da), getJ(Db), getK(Da), getK(Db).  So PackedInts and DirectInts
    keep their last two densities with J and K, and serve a repeated density
    without a second build.  The key is the density's values plus the
    precision and thresholds (direct) or the integral tensor's address, size
    and in-place version (packed); assigning a new tensor to PackedInts.tensor
    empties the cache.  The cache holds copies and hands out copies,
    so nothing a caller does to its arrays changes a later answer."""
    if isinstance(Ints, (PackedInts, DirectInts)):
        direct = isinstance(Ints, DirectInts)
        Dd, _ = _as_device(D, Ints.engine.device if direct else Ints.tensor.device)
        key = ((Ints.precision, Ints.schwarz, Ints.fp32_threshold) if direct
               else (Ints.tensor.data_ptr(), Ints.tensor.numel(), Ints.tensor._version))
        cache = Ints.__dict__.setdefault("_jk_cache", [])
        for i, (k, Dc, Jc, Kc) in enumerate(cache):
            if k == key and Dc.shape == Dd.shape and torch.equal(Dc, Dd) and (Kc is not None or coulomb_only):
                cache.insert(0, cache.pop(i))
                return Jc.clone(), (None if Kc is None else Kc.clone())
        if direct and coulomb_only:
            J, K = Ints.j(Dd), None
        else:
            J, K = Ints.jk(Dd) if direct else jk_packed(Ints.tensor.contiguous(), Dd)
        cache.insert(0, (key, Dd.clone(), J.clone(), None if K is None else K.clone()))
        del cache[_JK_CACHE:]
        return J, K
    if isinstance(Ints, torch.Tensor):
        t = Ints.to(dtype=torch.float64)
        if not t.is_cuda:
            t = t.cuda()
    else:
        t = torch.as_tensor(np.asarray(Ints, dtype=np.float64), device="cuda")
    Dd, _ = _as_device(D, t.device)
    return jk_packed(t.contiguous(), Dd)


def getJK2(Ints, Da, Db):
    """(Ja, Jb, Ka, Kb) of two densities: the four calls getJ(Ints, Da),
    getJ(Ints, Db), getK(Ints, Da), getK(Ints, Db) of the reference's UHF
    iteration (PyQuante/hartree_fock.py:233-236).  Integral-direct handles
    evaluate every integral once for both densities (pqb_jk_direct2); stored
    integrals run one build per density.  Both results are remembered like a
    getJ/getK build, so later getJ/getK calls with either density reuse them."""
    if isinstance(Ints, DirectInts):
        Dad, _ = _as_device(Da, Ints.engine.device)
        Dbd, _ = _as_device(Db, Ints.engine.device)
        if Dad.shape == Dbd.shape and torch.equal(Dad, Dbd):
            J, K = _jk(Ints, Da)
            return _back(J, Da), _back(J.clone(), Db), _back(K, Da), _back(K.clone(), Db)
        Ja, Ka, Jb, Kb = Ints.engine.jk2(Dad, Dbd, Ints.precision, Ints.schwarz, Ints.fp32_threshold)
        key = (Ints.precision, Ints.schwarz, Ints.fp32_threshold)
        cache = Ints.__dict__.setdefault("_jk_cache", [])
        for Dd, J, K in ((Dbd, Jb, Kb), (Dad, Ja, Ka)):
            cache.insert(0, (key, Dd.clone(), J.clone(), K.clone()))
        del cache[_JK_CACHE:]
        return _back(Ja, Da), _back(Jb, Db), _back(Ka, Da), _back(Kb, Db)
    Ja, Ka = _jk(Ints, Da)
    Jb, Kb = _jk(Ints, Db)
    return _back(Ja, Da), _back(Jb, Db), _back(Ka, Da), _back(Kb, Db)


def getJ(Ints, D, coulomb_only=False):
    """J_ij = sum_kl (ij|kl) D_kl (PyQuante/Ints.py:195-208).  One build gives
    J and K, so a following getK(Ints, D) costs nothing; ``coulomb_only=True``
    (the DFT driver, which never asks for K) runs the integral-direct
    Coulomb digestion alone instead."""
    J, _ = _jk(Ints, D, coulomb_only)
    return _back(J, D)


def getK(Ints, D):
    """K_ij = sum_kl (ik|jl) D_kl (PyQuante/Ints.py:210-223)."""
    _, K = _jk(Ints, D)
    return _back(K, D)


def get2JmK(Ints, D):
    """G = 2J - K (PyQuante/Ints.py:225-238).  A host density on
    integral-direct Ints (the reference's own call: numpy in, numpy out) goes
    through pqb_get2jmk_host, which copies D in, builds and copies G out in
    one call; J and K are not kept for a later getJ/getK."""
    if isinstance(Ints, DirectInts) and _is_host(D):
        n = Ints.nbf
        if isinstance(D, torch.Tensor):
            Dh = D.to(torch.float64).contiguous()
            G = torch.empty((n, n), dtype=torch.float64)
        else:
            Dh = np.ascontiguousarray(D, dtype=np.float64)
            G = np.empty((n, n))
        Ints.get2jmk_host(Dh, G)
        Ints.synchronize()
        return G
    J, K = _jk(Ints, D)
    return _back(2.0 * J - K, D)


def _is_host(D):
    return not (isinstance(D, torch.Tensor) and D.is_cuda)
