"""Batched RHF over many molecules of uneven size.

All molecules share one device basis (``pqb_shells_upload_batch``): shell
pairs and quartets stay inside a molecule, and every class kernel of a Fock
build serves all molecules in one launch.  D, J, K live as the molecules'
dense blocks back to back; the SCF linear algebra (FP64, cuSOLVER through
torch) runs on the blocks padded per size bucket:

    per iteration (all molecules at once)
      D = C_occ C_occ^T                  (PyQuante/LA2.py:127-131)
      J, K = pqb_jk_direct(D)            (one launch per class for the batch)
      F = h + 2J - K,  E = tr(Dh) + tr(DF) + E_nuc   (hartree_fock.py:29-38)
      Pulay DIIS per molecule            (Convergence.py:73-136)
      D' = projector on the occupied states of F' = X^T F X by batched
    canonical purification (or eigh), D = X D' X^T   (Cholesky X, LA2.py:47-75,113-116)

The molecules are grouped into at most 8 buckets of similar basis size
for the dense work, so small molecules are not padded to the largest one.
The Fock-build part of an iteration (densities, block gather/scatter, the
multi-stream J/K launches, F and E of every bucket) is captured once in a
CUDA graph and replayed; DIIS and the density update run eagerly per
bucket, as batched GEMMs.  A molecule is converged when its energy changes
by less than ``conv`` and its commutator FDS - SDF is below ``err_tol`` (its
SCF time is the time of that iteration); converged molecules keep their
last solution, and from the next iteration on their DIIS step and density
update are skipped.
"""
import ctypes
import time

import numpy as np
import torch

from . import _lib, autotune
from .Basis.basis import BasisSet
from .engine import FunctionTable, detect_shells, oneint

PAD_SHIFT = 1.0e6   # padded orbital energies, sorted above every real one


class BatchEngine:
    def __init__(self, systems, device=None):
        if device is None:
            device = torch.cuda.current_device()
        self.device = torch.device("cuda", device)
        self.ctx = _lib.Context(device)
        self.mols = [m for m, _ in systems]
        self.bases = [BasisSet(m, b) for m, b in systems]
        self.n = [len(b) for b in self.bases]
        self.f0 = np.concatenate([[0], np.cumsum(self.n)[:-1]]).astype(np.int64)
        self.block_off = np.concatenate([[0], np.cumsum([n * n for n in self.n])[:-1]]).astype(np.int64)
        L, NP, OFF, F0, XYZ, EXP, COEF, FS, MOLS = [], [], [], [], [], [], [], [], [0]
        for bs, f0 in zip(self.bases, self.f0):
            sh = detect_shells(bs.bfs)
            if sh is None:
                raise _lib.EngineError(_lib.PQB_E_CLASS, "batched bases need complete s/p/d shells")
            L += sh["l"]
            NP += sh["nprim"]
            OFF += [o + len(EXP) for o in sh["off"]]
            F0 += [f + int(f0) for f in sh["f0"]]
            XYZ += sh["xyz"]
            EXP += sh["exps"]
            COEF += sh["coefs"]
            FS += sh["fscale"]
            MOLS.append(len(L))
        ns, nbf, nm = len(L), int(sum(self.n)), len(self.mols)
        I, Dd = ctypes.c_int, ctypes.c_double
        self.ctx.check(self.ctx.lib.pqb_shells_upload_batch(
            self.ctx.h, nm, (I * (nm + 1))(*MOLS), ns, (I * ns)(*L), (I * ns)(*NP), (I * ns)(*OFF), (I * ns)(*F0),
            (Dd * (3 * ns))(*XYZ), (Dd * len(EXP))(*EXP), (Dd * len(COEF))(*COEF), nbf, (Dd * nbf)(*FS)))
        autotune.apply(self)
        dl = ctypes.c_int64()
        self.ctx.check(self.ctx.lib.pqb_dense_len(self.ctx.h, ctypes.byref(dl)))
        self.dense_len = dl.value
        self.plan_counts = None

    def plan(self, schwarz=1e-12, fp32_threshold=1e-5):
        np_ = self.ctx.lib.pqb_num_pairs(self.ctx.h)
        self.ctx.check(self.ctx.lib.pqb_schwarz(self.ctx.h, (ctypes.c_double * np_)(), _lib.stream_ptr()))
        c = (ctypes.c_int64 * 4)()
        self.ctx.check(self.ctx.lib.pqb_plan(self.ctx.h, schwarz, fp32_threshold, c))
        self.plan_counts = dict(shell_quartets=c[0], fp64=c[1], fp32=c[2], dropped=c[3])
        return self.plan_counts

    def jk(self, Dflat, J, K, mode):
        m = _lib.PQB_MIXED if mode == "mixed" else _lib.PQB_FP64
        self.ctx.check(self.ctx.lib.pqb_jk_direct(self.ctx.h, _lib.ptr(Dflat), _lib.ptr(J), _lib.ptr(K), m,
                                                  _lib.stream_ptr()))


def _bucket_edges(sizes, max_buckets=8):
    """Padded sizes: split the sorted basis sizes into at most max_buckets
    groups of similar size (equal counts), each padded to its largest."""
    order = np.argsort(sizes, kind="stable")
    groups = [g for g in np.array_split(order, min(max_buckets, len(sizes))) if len(g)]
    return [np.sort(g) for g in groups]


class _Bucket:
    """Molecules of similar basis size, padded to nb for the dense FP64 work."""

    def __init__(self, idx, eng, S_list, h_list, dev):
        f64 = dict(dtype=torch.float64, device=dev)
        self.idx = idx
        self.n = [eng.n[b] for b in idx]
        nb = max(self.n)
        B = len(idx)
        self.nb = nb
        S = torch.zeros((B, nb, nb), **f64)
        h = torch.zeros_like(S)
        for t, b in enumerate(idx):
            n = eng.n[b]
            S[t, :n, :n] = S_list[b]
            h[t, :n, :n] = h_list[b]
        nvec = torch.tensor(self.n, device=dev)
        self.pad = torch.arange(nb, device=dev)[None, :] >= nvec[:, None]
        self.padmask = self.pad[:, :, None] | self.pad[:, None, :]
        eye = torch.eye(nb, **f64).expand(B, nb, nb)
        self.S = torch.where(self.padmask, eye, S)
        self.h = h
        self.X = torch.linalg.inv(torch.linalg.cholesky(self.S)).transpose(1, 2)
        self.shift = torch.diag_embed(self.pad.to(torch.float64) * PAD_SHIFT)
        nocc = torch.tensor([eng.mols[b].get_closedopen()[0] for b in idx], device=dev)
        self.occ = (torch.arange(nb, device=dev)[None, :] < nocc[:, None]).to(torch.float64)
        self.enuc = torch.tensor([eng.mols[b].get_enuke() for b in idx], **f64)
        # padded position <-> position in the flat block layout
        pos, flat = [], []
        for t, b in enumerate(idx):
            n = eng.n[b]
            r = torch.arange(n, device=dev)
            pos.append((t * nb * nb + r[:, None] * nb + r[None, :]).reshape(-1))
            flat.append(int(eng.block_off[b]) + torch.arange(n * n, device=dev))
        self.pos = torch.cat(pos)
        self.flat = torch.cat(flat)
        # static buffers of the captured Fock build
        self.C = torch.zeros_like(self.S)
        self.D = torch.zeros_like(self.S)
        self.J = torch.zeros_like(self.S)
        self.K = torch.zeros_like(self.S)
        self.F = torch.zeros_like(self.S)
        self.E = torch.zeros(B, **f64)
        self.Fs, self.Es = [], []

    def solve(self, Fm, ia=None):
        """Orbitals of the Fock matrices Fm (all molecules of the bucket, or
        the positions ia)."""
        X, shift = (self.X, self.shift) if ia is None else (self.X.index_select(0, ia), self.shift.index_select(0, ia))
        e, V = torch.linalg.eigh(X.transpose(1, 2) @ Fm @ X + shift)
        return X @ V

    def density(self, Fm, ia=None, tol=1e-13, maxit=200):
        """Densities D = X P X^T of the Fock matrices Fm without an
        eigensolver: P, the projector on the nocc lowest states of
        F' = X^T F X, by the canonical purification of Palser and
        Manolopoulos (Phys. Rev. B 58, 12704 (1998)) -- batched GEMMs only.
        Padded dimensions sit above the real spectrum and stay empty."""
        X = self.X if ia is None else self.X.index_select(0, ia)
        pad = self.pad if ia is None else self.pad.index_select(0, ia)
        nocc = self.occ.sum(1) if ia is None else self.occ.index_select(0, ia).sum(1)
        Fp = X.transpose(1, 2) @ Fm @ X
        Fp = 0.5 * (Fp + Fp.transpose(1, 2))
        nb = Fp.shape[-1]
        # Gershgorin bounds of the real block; padded states just above them
        radius = Fp.abs().sum(-1) - Fp.diagonal(dim1=1, dim2=2).abs()
        d = Fp.diagonal(dim1=1, dim2=2)
        hi = torch.where(pad, torch.full_like(d, -1e300), d + radius).amax(1)
        lo = torch.where(pad, torch.full_like(d, 1e300), d - radius).amin(1)
        top = hi + 1.0
        Fp = Fp + torch.diag_embed(pad.to(Fp.dtype) * (top[:, None] - d))
        hi = torch.maximum(hi, top)
        mu = Fp.diagonal(dim1=1, dim2=2).sum(1) / nb
        lam = torch.minimum(nocc / (hi - mu), (nb - nocc) / (mu - lo))
        eye = torch.eye(nb, dtype=Fp.dtype, device=Fp.device)
        P = (lam / nb)[:, None, None] * (mu[:, None, None] * eye - Fp) + (nocc / nb)[:, None, None] * eye
        for _ in range(maxit):
            P2 = P @ P
            P3 = P2 @ P
            num = (P2 - P3).diagonal(dim1=1, dim2=2).sum(1)
            den = (P - P2).diagonal(dim1=1, dim2=2).sum(1)
            done = den.abs() < tol * nb          # idempotent to rounding: keep
            if bool(done.all()):
                break
            c = torch.where(done, torch.full_like(num, 0.5), num / torch.where(done, torch.ones_like(den), den))
            c = c.clamp(0.0, 1.0)
            hi_branch = ((1 + c)[:, None, None] * P2 - P3) / c.clamp(min=1e-300)[:, None, None]
            lo_branch = ((1 - 2 * c)[:, None, None] * P + (1 + c)[:, None, None] * P2 - P3) / \
                (1 - c).clamp(min=1e-300)[:, None, None]
            Pn = torch.where((c >= 0.5)[:, None, None], hi_branch, lo_branch)
            P = torch.where(done[:, None, None], P, Pn)
        return X @ P @ X.transpose(1, 2)


def batched_rhf(systems, precision="mixed", conv=1e-8, maxiter=60, diis_size=8, graph=True, schwarz=1e-12,
                fp32_threshold=1e-5, device=None, max_buckets=8, solver="purify", err_tol=1e-6):
    """Solve RHF for every (molecule, basis) in ``systems`` together.

    The Fock build of every iteration is one engine call for all molecules;
    the dense FP64 algebra runs per size bucket (molecules padded to the
    bucket's largest basis).  ``solver='purify'`` (default) gets each new
    density from the DIIS Fock matrix by batched canonical purification
    (GEMMs only, no per-molecule eigensolver); ``'eigh'`` diagonalises.
    A molecule is converged when its energy changes by less than ``conv``
    and its commutator max|FDS - SDF| is below ``err_tol``.  Returns a
    dict: energies, iterations, per-molecule SCF times (s), total time (s),
    and the plan counts."""
    if solver not in ("purify", "eigh"):
        raise ValueError("solver must be 'purify' or 'eigh'")
    t_start = time.perf_counter()
    eng = BatchEngine(systems, device)
    dev = eng.device
    f64 = dict(dtype=torch.float64, device=dev)
    B = len(systems)
    counts = eng.plan(schwarz, fp32_threshold)
    S_list, h_list = [], []
    for bs, mol in zip(eng.bases, eng.mols):
        ft = FunctionTable(bs.bfs, dev.index)
        Sb, Tb, Vb = oneint(ft, mol.atoms, eng.ctx)
        S_list.append(Sb)
        h_list.append(Tb + Vb)
    buckets = [_Bucket(idx, eng, S_list, h_list, dev) for idx in _bucket_edges(np.array(eng.n), max_buckets)]
    def new_density(bk, Fm, ia=None):
        if solver == "purify":
            return bk.density(Fm, ia)
        C = bk.solve(Fm, ia)
        occ = bk.occ if ia is None else bk.occ.index_select(0, ia)
        Co = C * occ[:, None, :]
        return Co @ Co.transpose(1, 2)

    for bk in buckets:
        bk.D.copy_(new_density(bk, bk.h))
    Dflat = torch.zeros(eng.dense_len, **f64)
    Jf = torch.zeros_like(Dflat)
    Kf = torch.zeros_like(Dflat)

    def fock_build():
        for bk in buckets:
            Dflat.index_copy_(0, bk.flat, bk.D.reshape(-1).index_select(0, bk.pos))
        eng.jk(Dflat, Jf, Kf, precision)
        for bk in buckets:
            bk.J.view(-1).index_copy_(0, bk.pos, Jf.index_select(0, bk.flat))
            bk.K.view(-1).index_copy_(0, bk.pos, Kf.index_select(0, bk.flat))
            bk.F.copy_(bk.h + 2.0 * bk.J - bk.K)
            bk.E.copy_((bk.D * bk.h).sum(dim=(1, 2)) + (bk.D * bk.F).sum(dim=(1, 2)) + bk.enuc)

    fock_build()                       # warm-up (kernel attributes, allocator)
    torch.cuda.synchronize()
    g = None
    if graph:
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            fock_build()
        torch.cuda.current_stream().wait_stream(s)
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            fock_build()
    energies = np.zeros(B)
    iters = np.zeros(B, dtype=np.int64)
    done = np.zeros(B, dtype=bool)
    times = np.zeros(B)
    eold = [torch.zeros(len(bk.idx), **f64) for bk in buckets]
    bdone = [torch.zeros(len(bk.idx), dtype=torch.bool, device=dev) for bk in buckets]
    t0 = time.perf_counter()
    for it in range(maxiter):
        if g is not None:
            g.replay()
        else:
            fock_build()
        for q, bk in enumerate(buckets):
            nb, Bb = bk.nb, len(bk.idx)
            # molecules converged in earlier iterations keep their orbitals: the
            # eigensolves (one per molecule) run for the others only
            act = ~done[bk.idx]
            if not act.any():
                continue
            err = bk.F @ bk.D @ bk.S - bk.S @ bk.D @ bk.F
            err = torch.where(bk.padmask, torch.zeros_like(err), err)
            bk.Fs.append(bk.F.clone())
            bk.Es.append(err.reshape(Bb, -1))
            if len(bk.Fs) > diis_size:
                bk.Fs.pop(0)
                bk.Es.pop(0)
            k = len(bk.Fs)
            Em = torch.stack(bk.Es, dim=1)
            A = torch.zeros((Bb, k + 1, k + 1), **f64)
            A[:, :k, :k] = Em @ Em.transpose(1, 2)
            scale = A[:, :k, :k].diagonal(dim1=1, dim2=2).abs().amax(dim=1).clamp(min=1e-300)
            A[:, :k, :k] /= scale[:, None, None]
            A[:, :k, k] = -1.0
            A[:, k, :k] = -1.0
            rhs = torch.zeros((Bb, k + 1), **f64)
            rhs[:, k] = -1.0
            c, info = torch.linalg.solve_ex(A, rhs)
            c = torch.where((info == 0)[:, None], c, torch.nn.functional.one_hot(
                torch.full((Bb,), k - 1, device=dev), k + 1).to(torch.float64))
            Fd = (c[:, :k, None, None] * torch.stack(bk.Fs, dim=1)).sum(dim=1)
            emax = err.abs().amax(dim=(1, 2))
            energy = bk.E.clone()
            if act.all():
                bk.D.copy_(new_density(bk, Fd))
            else:
                ia = torch.from_numpy(np.nonzero(act)[0]).to(dev)
                bk.D.index_copy_(0, ia, new_density(bk, Fd.index_select(0, ia), ia))
            newly = (~bdone[q]) & ((energy - eold[q]).abs() < conv) & (emax < err_tol)
            eold[q] = torch.where(bdone[q], eold[q], energy)
            bdone[q] = bdone[q] | newly
        flags = [(bd.cpu().numpy(), e.cpu().numpy()) for bd, e in zip(bdone, eold)]
        now = time.perf_counter() - t0
        for bk, (bd, e) in zip(buckets, flags):
            fresh = bd & ~done[bk.idx]
            times[bk.idx[fresh]] = now
            iters[bk.idx[~done[bk.idx]]] = it + 1
            done[bk.idx] = bd
            energies[bk.idx] = e
        if done.all():
            break
    torch.cuda.synchronize()
    t_end = time.perf_counter()
    times[times == 0] = t_end - t0
    return dict(energies=energies, iterations=iters, converged=done, scf_times=times, scf_seconds=t_end - t0,
                total_seconds=t_end - t_start, plan=counts, nbf=np.array(eng.n), graph=g is not None,
                buckets=[bk.nb for bk in buckets])
