"""Batched RHF over many molecules of uneven size.

All molecules share one device basis (``pqb_shells_upload_batch``): shell
pairs and quartets stay inside a molecule, and every class kernel of a Fock
build serves all molecules in one launch.  D, J, K live as the molecules'
dense blocks back to back; the SCF linear algebra (FP64, cuSOLVER through
torch) runs on the blocks padded to the largest basis:

    per iteration (all molecules at once)
      D = C_occ C_occ^T                  (PyQuante/LA2.py:127-131)
      J, K = pqb_jk_direct(D)            (one launch per class for the batch)
      F = h + 2J - K,  E = tr(Dh) + tr(DF) + E_nuc   (hartree_fock.py:29-38)
      Pulay DIIS per molecule            (Convergence.py:73-136)
      F' = X^T F X, eigh, C = X C'        Cholesky X (LA2.py:47-75,113-116)

The Fock-build part of an iteration (density, block gather/scatter, the
multi-stream J/K launches, F and E) is captured once in a CUDA graph and
replayed; DIIS and the eigensolve run eagerly.  A molecule is converged when
its energy changes by less than ``conv`` (its SCF time is the time of that
iteration); converged molecules keep their last solution.
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


def _padded_index(n_list, nmax, device):
    """Flat block-layout position k -> position in the (B, nmax, nmax) padding."""
    idx = []
    for b, n in enumerate(n_list):
        r = torch.arange(n, device=device)
        idx.append((b * nmax * nmax + r[:, None] * nmax + r[None, :]).reshape(-1))
    return torch.cat(idx)


def batched_rhf(systems, precision="mixed", conv=1e-8, maxiter=60, diis_size=8, graph=True, schwarz=1e-12,
                fp32_threshold=1e-5, device=None):
    """Solve RHF for every (molecule, basis) in ``systems`` together.

    Returns a dict: energies, iterations, per-molecule SCF times (s), total
    time (s), and the plan counts."""
    t_start = time.perf_counter()
    eng = BatchEngine(systems, device)
    dev = eng.device
    f64 = dict(dtype=torch.float64, device=dev)
    B, nmax = len(systems), max(eng.n)
    counts = eng.plan(schwarz, fp32_threshold)
    # one-electron integrals per molecule, padded
    S = torch.zeros((B, nmax, nmax), **f64)
    h = torch.zeros_like(S)
    for b, (bs, mol) in enumerate(zip(eng.bases, eng.mols)):
        ft = FunctionTable(bs.bfs, dev.index)
        Sb, Tb, Vb = oneint(ft, mol.atoms, eng.ctx)
        n = eng.n[b]
        S[b, :n, :n] = Sb
        h[b, :n, :n] = Tb + Vb
    nvec = torch.tensor(eng.n, device=dev)
    pad = torch.arange(nmax, device=dev)[None, :] >= nvec[:, None]              # (B, nmax)
    eye = torch.eye(nmax, **f64).expand(B, nmax, nmax)
    S = torch.where(pad[:, :, None] | pad[:, None, :], eye, S)
    X = torch.linalg.inv(torch.linalg.cholesky(S)).transpose(1, 2)            # S^-1/2 by Cholesky
    shift = torch.diag_embed(pad.to(torch.float64) * PAD_SHIFT)
    nocc = torch.tensor([m.get_closedopen()[0] for m in eng.mols], device=dev)
    occ = (torch.arange(nmax, device=dev)[None, :] < nocc[:, None]).to(torch.float64)   # (B, nmax)
    enuc = torch.tensor([m.get_enuke() for m in eng.mols], **f64)
    pidx = _padded_index(eng.n, nmax, dev)

    def solve(Fm):
        e, V = torch.linalg.eigh(X.transpose(1, 2) @ Fm @ X + shift)
        return X @ V

    C = solve(h)
    # static buffers for the captured Fock build
    Cs = C.clone()
    D = torch.zeros_like(S)
    Dflat = torch.zeros(eng.dense_len, **f64)
    Jf = torch.zeros_like(Dflat)
    Kf = torch.zeros_like(Dflat)
    J = torch.zeros_like(S)
    K = torch.zeros_like(S)
    F = torch.zeros_like(S)
    E = torch.zeros(B, **f64)

    def fock_build():
        Co = Cs * occ[:, None, :]
        D.copy_(Co @ Co.transpose(1, 2))
        torch.take(D.reshape(-1), pidx, out=Dflat)
        eng.jk(Dflat, Jf, Kf, precision)
        J.view(-1).index_copy_(0, pidx, Jf)
        K.view(-1).index_copy_(0, pidx, Kf)
        F.copy_(h + 2.0 * J - K)
        E.copy_((D * h).sum(dim=(1, 2)) + (D * F).sum(dim=(1, 2)) + enuc)

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
    Fs, Es = [], []
    eold = torch.zeros(B, **f64)
    done = torch.zeros(B, dtype=torch.bool, device=dev)
    iters = torch.zeros(B, dtype=torch.int64, device=dev)
    times = np.zeros(B)
    t0 = time.perf_counter()
    for it in range(maxiter):
        Cs.copy_(C)
        if g is not None:
            g.replay()
        else:
            fock_build()
        # Pulay DIIS per molecule on the error FDS - SDF
        err = F @ D @ S - S @ D @ F
        err = torch.where(pad[:, :, None] | pad[:, None, :], torch.zeros_like(err), err)
        Fs.append(F.clone())
        Es.append(err.reshape(B, -1))
        if len(Fs) > diis_size:
            Fs.pop(0)
            Es.pop(0)
        k = len(Fs)
        Em = torch.stack(Es, dim=1)                                   # (B, k, n^2)
        A = torch.zeros((B, k + 1, k + 1), **f64)
        A[:, :k, :k] = Em @ Em.transpose(1, 2)
        A[:, :k, k] = -1.0
        A[:, k, :k] = -1.0
        rhs = torch.zeros((B, k + 1), **f64)
        rhs[:, k] = -1.0
        scale = A[:, :k, :k].diagonal(dim1=1, dim2=2).abs().amax(dim=1).clamp(min=1e-300)
        A[:, :k, :k] /= scale[:, None, None]
        c, info = torch.linalg.solve_ex(A, rhs)
        c = torch.where((info == 0)[:, None], c, torch.nn.functional.one_hot(
            torch.full((B,), k - 1, device=dev), k + 1).to(torch.float64))
        Fd = (c[:, :k, None, None] * torch.stack(Fs, dim=1)).sum(dim=1)
        Cn = solve(Fd)
        energy = E.clone()
        newly = (~done) & ((energy - eold).abs() < conv)
        iters = torch.where(done, iters, torch.full_like(iters, it + 1))
        C = torch.where(done[:, None, None], C, Cn)
        done = done | newly
        eold = torch.where(done & ~newly, eold, energy)
        nd = newly.cpu().numpy()
        if nd.any():
            torch.cuda.synchronize()
            times[nd] = time.perf_counter() - t0
        if bool(done.all()):
            break
    torch.cuda.synchronize()
    t_end = time.perf_counter()
    times[times == 0] = t_end - t0
    return dict(energies=eold.cpu().numpy(), iterations=iters.cpu().numpy(), converged=done.cpu().numpy(),
                scf_times=times, scf_seconds=t_end - t0, total_seconds=t_end - t_start, plan=counts,
                nbf=np.array(eng.n), graph=g is not None)
