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
With the purification solver the whole iteration is captured once in a CUDA
graph and replayed: the Fock build (densities, block gather/scatter, the
multi-stream J/K launches, F and E of every bucket), DIIS (histories in
fixed rings on the device, the DIIS equations by a batched Gauss-Jordan
elimination), the purification (a fixed number of steps; converged states
are frozen) and the convergence flags.  The host reads one flag per
molecule per iteration.  A molecule is converged when its energy changes by
less than ``conv`` and its commutator FDS - SDF is below ``err_tol`` (its
SCF time is the time of that iteration); converged molecules keep their
last density, and from the next iteration on the Fock build skips their
quartets (a per-molecule mask read by the kernels).

The Fock builds are incremental: each iteration digests the density change
D - D_prev into accumulated J and K (J and K are linear in D), with work
items skipped when their Schwarz bound times the largest density change of
their shells is below ``screen_tau``; as the SCF converges the changes
shrink and most items drop out.  Every ``rebuild_every`` iterations the
accumulators restart from a full build.
"""
import ctypes
import time

import numpy as np
import torch

from . import _lib, autotune
from .Basis.basis import BasisSet
from .engine import FunctionTable, detect_shells, oneint
from .LA2 import purify

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
        self.nshell = ns
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

    def set_mask(self, mask):
        """Build only the molecules m with mask[m] != 0 (a device int32
        tensor of one entry per molecule, kept alive by the caller), or every
        molecule (None)."""
        self._mask = mask
        self.ctx.check(self.ctx.lib.pqb_set_molecule_mask(self.ctx.h, None if mask is None else _lib.ptr(mask)))

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

    def density(self, Fm, ia=None, tol=1e-13, maxit=200, fixed=False):
        """Densities D = X P X^T of the Fock matrices Fm without an
        eigensolver: P, the projector on the nocc lowest states of
        F' = X^T F X, by the canonical purification of Palser and
        Manolopoulos (Phys. Rev. B 58, 12704 (1998)) -- batched GEMMs only.
        Padded dimensions sit above the real spectrum and stay empty.
        fixed: run exactly maxit steps with no host check (states that are
        idempotent to rounding are kept), so that the loop can be captured
        in a CUDA graph."""
        X = self.X if ia is None else self.X.index_select(0, ia)
        pad = self.pad if ia is None else self.pad.index_select(0, ia)
        nocc = self.occ.sum(1) if ia is None else self.occ.index_select(0, ia).sum(1)
        P = purify(X.transpose(1, 2) @ Fm @ X, nocc, pad=pad, tol=tol, maxit=maxit, fixed=fixed)
        return X @ P @ X.transpose(1, 2)


def _solve_small(A, b):
    """x with A x = b for a batch of small systems (A: (B, n, n), b: (B, n)) by
    Gauss-Jordan elimination with partial pivoting, in plain tensor
    operations (no library solver, no host synchronisation), so that it can
    be captured in a CUDA graph.  A singular system gives non-finite x."""
    Bn, n = A.shape[0], A.shape[-1]
    M = torch.cat([A, b[..., None]], dim=-1)
    ar = torch.arange(n, device=A.device)[None, :]
    for j in range(n):
        col = M[:, :, j].abs()
        col = torch.where(ar >= j, col, torch.full_like(col, -1.0))
        p = col.argmax(1)[:, None]
        perm = torch.where(ar == j, p, torch.where(ar == p, torch.full_like(p, j), ar))
        M = M.gather(1, perm[:, :, None].expand(-1, -1, n + 1))
        piv = M[:, j, :] / M[:, j, j:j + 1]
        M = M - M[:, :, j:j + 1] * piv[:, None, :]
        M[:, j, :] = piv
    return M[:, :, n]


class _Diis:
    """Pulay DIIS of one bucket (Convergence.py:73-136, the same guarded
    form as Convergence.DIIS: at most S vectors) on fixed device buffers: the
    last S Fock matrices and commutators in rings, the slot and fill count
    as device scalars, so that a step has static shapes and no host
    synchronisation."""

    def __init__(self, bk, S):
        B, nb = len(bk.idx), bk.nb
        dev = bk.S.device
        self.S = S
        self.F = torch.zeros((B, S, nb, nb), dtype=torch.float64, device=dev)
        self.E = torch.zeros((B, S, nb * nb), dtype=torch.float64, device=dev)
        self.slot = torch.zeros(1, dtype=torch.int64, device=dev)
        self.nfill = torch.zeros((), dtype=torch.int64, device=dev)
        self.ar = torch.arange(S, device=dev)
        self.eye = torch.eye(S, dtype=torch.float64, device=dev)

    def step(self, F, err):
        """Store (F, err) and return the extrapolated Fock matrices."""
        B, S = F.shape[0], self.S
        self.F.index_copy_(1, self.slot, F[:, None])
        self.E.index_copy_(1, self.slot, err.reshape(B, 1, -1))
        newest = (self.ar == self.slot).to(torch.float64)[None, :].expand(B, S)
        self.nfill.copy_(torch.clamp(self.nfill + 1, max=S))
        self.slot.copy_((self.slot + 1) % S)
        filled = self.ar < self.nfill
        G = self.E @ self.E.transpose(1, 2)
        scale = torch.where(filled[None, :], G.diagonal(dim1=1, dim2=2), torch.zeros_like(newest))
        scale = scale.abs().amax(1).clamp(min=1e-300)
        fm = filled[:, None] & filled[None, :]
        G = torch.where(fm[None], G / scale[:, None, None], self.eye[None])
        fcol = -filled.to(torch.float64)
        A = torch.zeros((B, S + 1, S + 1), dtype=torch.float64, device=F.device)
        A[:, :S, :S] = G
        A[:, :S, S] = fcol
        A[:, S, :S] = fcol
        rhs = torch.zeros((B, S + 1), dtype=torch.float64, device=F.device)
        rhs[:, S] = -1.0
        c = _solve_small(A, rhs)[:, :S]
        ok = torch.isfinite(c).all(1, keepdim=True)
        c = torch.where(ok, c, newest)
        return torch.einsum("bs,bsij->bij", c, self.F)


def batched_rhf(systems, precision="mixed", conv=1e-8, maxiter=60, diis_size=8, graph=True, schwarz=1e-12,
                fp32_threshold=1e-5, device=None, max_buckets=8, solver="purify", err_tol=1e-6, purify_steps=48,
                incremental=True, screen_tau=1e-12, rebuild_every=8):
    """Solve RHF for every (molecule, basis) in ``systems`` together.

    The Fock build of every iteration is one engine call for all molecules;
    the dense FP64 algebra runs per size bucket (molecules padded to the
    bucket's largest basis).  ``solver='purify'`` (default) gets each new
    density from the DIIS Fock matrix by batched canonical purification
    (GEMMs only, ``purify_steps`` steps, no per-molecule eigensolver), and
    with ``graph=True`` the whole iteration is one CUDA graph replay;
    ``'eigh'`` diagonalises (then only the Fock build is captured).
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

    def new_density(bk, Fm):
        if solver == "purify":
            return bk.density(Fm, maxit=purify_steps, fixed=True)
        C = bk.solve(Fm)
        Co = C * bk.occ[:, None, :]
        return Co @ Co.transpose(1, 2)

    for bk in buckets:
        # core guess (outside the loop: purification to idempotency)
        bk.D.copy_(bk.density(bk.h) if solver == "purify" else new_density(bk, bk.h))
        bk.diis = _Diis(bk, diis_size)
        bk.eold = torch.zeros(len(bk.idx), **f64)
        bk.bdone = torch.zeros(len(bk.idx), dtype=torch.bool, device=dev)
        bk.conv_it = torch.full((len(bk.idx),), -1, dtype=torch.int64, device=dev)
    Dflat = torch.zeros(eng.dense_len, **f64)
    Jf = torch.zeros_like(Dflat)
    Kf = torch.zeros_like(Dflat)
    lib, h_ctx = eng.ctx.lib, eng.ctx.h
    if incremental:
        # J, K accumulated over density changes, screened by shell bounds of the change
        Dprev, dD = torch.zeros_like(Dflat), torch.zeros_like(Dflat)
        Jacc, Kacc = torch.zeros_like(Dflat), torch.zeros_like(Dflat)
        dsh = torch.zeros(eng.nshell, **f64)
        eng.ctx.check(lib.pqb_set_density_screen(h_ctx, _lib.ptr(dsh), float(screen_tau)))
    it_dev = torch.zeros((), dtype=torch.int64, device=dev)
    # per molecule (in input order): converged flag and energy, gathered on the device
    all_idx = torch.cat([torch.as_tensor(bk.idx, device=dev) for bk in buckets])
    flags = torch.zeros(B, dtype=torch.bool, device=dev)
    # molecules still iterating: the Fock build skips the others' quartets
    active = torch.ones(B, dtype=torch.int32, device=dev)
    eng.set_mask(active)

    def fock_build():
        for bk in buckets:
            Dflat.index_copy_(0, bk.flat, bk.D.reshape(-1).index_select(0, bk.pos))
        if incremental:
            torch.sub(Dflat, Dprev, out=dD)
            eng.ctx.check(lib.pqb_shell_dmax(h_ctx, _lib.ptr(dD), _lib.ptr(dsh), _lib.stream_ptr()))
            eng.jk(dD, Jf, Kf, precision)
            Jacc.add_(Jf)
            Kacc.add_(Kf)
            Dprev.copy_(Dflat)
            Js, Ks = Jacc, Kacc
        else:
            eng.jk(Dflat, Jf, Kf, precision)
            Js, Ks = Jf, Kf
        for bk in buckets:
            bk.J.view(-1).index_copy_(0, bk.pos, Js.index_select(0, bk.flat))
            bk.K.view(-1).index_copy_(0, bk.pos, Ks.index_select(0, bk.flat))
            bk.F.copy_(bk.h + 2.0 * bk.J - bk.K)
            bk.E.copy_((bk.D * bk.h).sum(dim=(1, 2)) + (bk.D * bk.F).sum(dim=(1, 2)) + bk.enuc)

    def update():
        """DIIS, new densities and convergence flags of every bucket (static
        shapes; converged molecules keep their density)."""
        for bk in buckets:
            err = bk.F @ bk.D @ bk.S - bk.S @ bk.D @ bk.F
            err = torch.where(bk.padmask, torch.zeros_like(err), err)
            Fd = bk.diis.step(bk.F, err)
            emax = err.abs().amax(dim=(1, 2))
            Dn = new_density(bk, Fd)
            bk.D.copy_(torch.where(bk.bdone[:, None, None], bk.D, Dn))
            newly = (~bk.bdone) & ((bk.E - bk.eold).abs() < conv) & (emax < err_tol)
            bk.eold.copy_(torch.where(bk.bdone, bk.eold, bk.E))
            bk.conv_it.copy_(torch.where(newly, it_dev, bk.conv_it))
            bk.bdone.copy_(bk.bdone | newly)
        flags.index_copy_(0, all_idx, torch.cat([bk.bdone for bk in buckets]))
        active.copy_((~flags).to(torch.int32))
        it_dev.add_(1)

    def iteration():
        fock_build()
        update()

    # warm-up of the kernels' attributes and the allocator, then the state is reset
    snapshot = [bk.D.clone() for bk in buckets]
    iteration()
    torch.cuda.synchronize()
    whole = graph and solver == "purify"
    g = None
    if graph:
        body = iteration if whole else fock_build
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            body()
        torch.cuda.current_stream().wait_stream(s)
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            body()
    for bk, D0 in zip(buckets, snapshot):
        bk.D.copy_(D0)
        bk.diis.F.zero_()
        bk.diis.E.zero_()
        bk.diis.slot.zero_()
        bk.diis.nfill.zero_()
        bk.eold.zero_()
        bk.bdone.zero_()
        bk.conv_it.fill_(-1)
    it_dev.zero_()
    flags.zero_()
    active.fill_(1)
    torch.cuda.synchronize()

    def restart():
        # the next build is a full one: accumulators from zero
        if incremental:
            Dprev.zero_()
            Jacc.zero_()
            Kacc.zero_()
    iter_time = []
    t0 = time.perf_counter()
    for it in range(maxiter):
        if it % rebuild_every == 0:
            restart()
        if g is not None:
            g.replay()
            if not whole:
                update()
        else:
            iteration()
        done = flags.cpu().numpy()
        iter_time.append(time.perf_counter() - t0)
        if done.all():
            break
    torch.cuda.synchronize()
    t_end = time.perf_counter()
    eng.ctx.check(lib.pqb_set_density_screen(h_ctx, None, 0.0))
    eng.set_mask(None)
    energies = np.zeros(B)
    iters = np.zeros(B, dtype=np.int64)
    times = np.zeros(B)
    done = np.zeros(B, dtype=bool)
    for bk in buckets:
        ci = bk.conv_it.cpu().numpy()
        ok = ci >= 0
        energies[bk.idx] = bk.eold.cpu().numpy()
        done[bk.idx] = ok
        iters[bk.idx] = np.where(ok, ci + 1, len(iter_time))
        times[bk.idx] = np.where(ok, [iter_time[c] if c >= 0 else 0.0 for c in ci], t_end - t0)
    return dict(energies=energies, iterations=iters, converged=done, scf_times=times, scf_seconds=t_end - t0,
                total_seconds=t_end - t_start, plan=counts, nbf=np.array(eng.n), graph=g is not None,
                whole_iteration_graph=whole and g is not None, incremental=incremental,
                buckets=[bk.nb for bk in buckets])
