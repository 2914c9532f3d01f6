"""Device-side view of a basis and the calls into the CUDA engine.

``BasisEngine`` turns a list of contracted functions (CGBF-like objects with
``origin, powers, pexps, pcoefs, pnorms, norm``) into
  * a per-function table (device tensors) for the stateless kernels
    (one-electron integrals, scalar ERIs), and
  * a shell table for the class-templated ERI engine, when consecutive
    functions form complete cartesian shells (s, p, d) sharing exponents,
    which is what ``BasisSet`` produces.
It owns its own ``pqb_ctx`` so several bases can coexist.
"""
import ctypes

import numpy as np
import torch

from . import _lib
from ._lib import ptr, stream_ptr

# cartesian components in PyQuante order (PyQuante/Ints.py:23-29): x descending, then y descending
_CART = {L: [(x, y, L - x - y) for x in range(L, -1, -1) for y in range(L - x, -1, -1)] for L in range(5)}


def _host_ptr(x):
    """Address of a host array (CPU torch tensor or numpy array)."""
    if isinstance(x, torch.Tensor):
        return ctypes.c_void_p(x.data_ptr())
    return ctypes.c_void_p(x.ctypes.data)


def cart_components(L):
    return _CART[L]


def _weights(bf):
    return [bf.norm * c * n for c, n in zip(bf.pcoefs, bf.pnorms)]


def detect_shells(bfs, max_l=2):
    """Group functions into shells for the class engine, or return None.

    A shell is a run of consecutive functions with one origin, one exponent
    list and the complete cartesian component set of its angular momentum
    in PyQuante order, whose per-primitive weights norm*pcoef*pnorm factor
    as (shell coefficient c_p) x (component scale r_f)."""
    n = len(bfs)
    sh_l, sh_np, sh_off, sh_f0, sh_xyz, exps, coefs, fscale = [], [], [], [], [], [], [], [0.0] * n
    i = 0
    while i < n:
        bf = bfs[i]
        L = sum(bf.powers)
        if L > max_l:
            return None
        comps = cart_components(L)
        grp = bfs[i:i + len(comps)]
        if len(grp) != len(comps):
            return None
        w0 = _weights(bf)
        if any(abs(w) == 0.0 for w in w0):
            return None
        for f, comp in zip(grp, comps):
            if tuple(f.powers) != comp or tuple(f.origin) != tuple(bf.origin) or list(f.pexps) != list(bf.pexps):
                return None
            wf = _weights(f)
            r = wf[0] / w0[0]
            if any(abs(a - r * b) > 1e-12 * abs(a) for a, b in zip(wf, w0)):
                return None
        sh_l.append(L)
        sh_np.append(len(bf.pexps))
        sh_off.append(len(exps))
        sh_f0.append(i)
        sh_xyz.extend(bf.origin)
        exps.extend(bf.pexps)
        coefs.extend(w0)
        for k, f in enumerate(grp):
            fscale[i + k] = _weights(f)[0] / w0[0]
        i += len(comps)
    return dict(l=sh_l, nprim=sh_np, off=sh_off, f0=sh_f0, xyz=sh_xyz, exps=exps, coefs=coefs, fscale=fscale)


class FunctionTable:
    """Per-function device table: origin, powers, prim_off, exps, cn, norms."""

    def __init__(self, bfs, device):
        n = len(bfs)
        off = [0]
        exps, cn = [], []
        for bf in bfs:
            if len(bf.pexps) != len(bf.pcoefs) or len(bf.pexps) != len(bf.pnorms) or not bf.pexps:
                raise ValueError("inconsistent primitive lists in %r" % (bf,))
            exps.extend(bf.pexps)
            cn.extend(c * m for c, m in zip(bf.pcoefs, bf.pnorms))
            off.append(len(exps))
        dev = torch.device("cuda", device)
        f64 = dict(dtype=torch.float64, device=dev)
        i32 = dict(dtype=torch.int32, device=dev)
        self.n = n
        self.powers_host = np.array([bf.powers for bf in bfs], dtype=np.int32).reshape(n, 3)
        self.origin = torch.tensor([bf.origin for bf in bfs], **f64).reshape(n, 3).contiguous()
        self.powers = torch.tensor(self.powers_host, **i32).contiguous()
        self.prim_off = torch.tensor(off, **i32)
        self.exps = torch.tensor(exps, **f64)
        self.cn = torch.tensor(cn, **f64)
        self.norms = torch.tensor([bf.norm for bf in bfs], **f64)

    def args(self):
        return (self.n, ptr(self.origin), ptr(self.powers), ptr(self.prim_off), ptr(self.exps), ptr(self.cn),
                ptr(self.norms))


def oneint(ft, atoms, ctx, stream=None):
    """S, T, V (n x n device tensors) for a FunctionTable and atoms."""
    n = ft.n
    if int(ft.powers_host.sum(axis=1).max(initial=0)) > 3:
        raise _lib.EngineError(_lib.PQB_E_CLASS, "one-electron integrals support up to f functions")
    dev = ft.origin.device
    S = torch.empty((n, n), dtype=torch.float64, device=dev)
    T = torch.empty_like(S)
    V = torch.empty_like(S)
    atoms = list(atoms or [])
    xyz = (ctypes.c_double * max(3 * len(atoms), 1))(*[c for a in atoms for c in a.pos()])
    z = (ctypes.c_double * max(len(atoms), 1))(*[float(a.atno) for a in atoms])
    ctx.check(ctx.lib.pqb_oneint(ctx.h, *ft.args(), len(atoms), xyz, z, ptr(S), ptr(T), ptr(V), stream_ptr(stream)))
    return S, T, V


def eri_functions(ft, quartets, ctx, engine=_lib.PQB_ENGINE_RYS, aux_m=0, stream=None):
    """Contracted ERIs for function quartets (host int array (nq, 4))."""
    q = np.ascontiguousarray(np.asarray(quartets, dtype=np.int32).reshape(-1, 4))
    L = ft.powers_host.sum(axis=1)
    if len(q):
        tot = L[q].sum(axis=1)
        if int(tot.max()) > 9:
            raise _lib.EngineError(_lib.PQB_E_CLASS, "total angular momentum %d > 9 (5 Rys roots)" % int(tot.max()))
        if engine == _lib.PQB_ENGINE_HGP and (int((L[q[:, 0]] + L[q[:, 1]]).max()) > 4 or
                                              int((L[q[:, 2]] + L[q[:, 3]]).max()) > 4 or int(tot.max()) + aux_m > 8):
            raise _lib.EngineError(_lib.PQB_E_CLASS, "HGP engine: |a|+|b| and |c|+|d| must be <= 4, total+m <= 8")
    dev = ft.origin.device
    qd = torch.from_numpy(q).to(dev)
    out = torch.empty(len(q), dtype=torch.float64, device=dev)
    ctx.check(ctx.lib.pqb_eri_functions(ctx.h, engine, aux_m, len(q), ptr(qd), *ft.args(), ptr(out),
                                        stream_ptr(stream)))
    return out


class BasisEngine:
    """A basis resident on one GPU, with the class-engine tables when the
    functions form complete s/p/d shells."""

    def __init__(self, bfs, device=None):
        self.bfs = list(bfs)
        self.nbf = len(self.bfs)
        if device is None:
            device = torch.cuda.current_device() if torch.cuda.is_available() else 0
        self.ctx = _lib.Context(device)
        self.device = torch.device("cuda", device)
        self.ft = FunctionTable(self.bfs, device)
        self.shells = detect_shells(self.bfs)
        self.Q = None
        self.plan_counts = None
        self._plan_key = None
        if self.shells is not None:
            s = self.shells
            ns = len(s["l"])
            I = ctypes.c_int
            D = ctypes.c_double
            self.ctx.check(self.ctx.lib.pqb_shells_upload(
                self.ctx.h, ns, (I * ns)(*s["l"]), (I * ns)(*s["nprim"]), (I * ns)(*s["off"]), (I * ns)(*s["f0"]),
                (D * (3 * ns))(*s["xyz"]), (D * len(s["exps"]))(*s["exps"]), (D * len(s["coefs"]))(*s["coefs"]),
                self.nbf, (D * self.nbf)(*s["fscale"])))
            from . import autotune
            autotune.apply(self)

    @property
    def has_shells(self):
        return self.shells is not None

    def _need_shells(self):
        if not self.has_shells:
            raise _lib.EngineError(_lib.PQB_E_CLASS,
                                   "the class engine needs complete s/p/d cartesian shells (use the per-function path)")

    def schwarz(self, stream=None):
        self._need_shells()
        if self.Q is None:
            np_ = self.ctx.lib.pqb_num_pairs(self.ctx.h)
            buf = (ctypes.c_double * np_)()
            self.ctx.check(self.ctx.lib.pqb_schwarz(self.ctx.h, buf, stream_ptr(stream)))
            self.Q = np.frombuffer(buf, dtype=np.float64).copy()
        return self.Q

    def plan(self, schwarz=1e-12, fp32_threshold=1e-5):
        """Screened quartet lists; returns the counts dict."""
        key = (float(schwarz), float(fp32_threshold))
        if self._plan_key != key:
            self.schwarz()
            c = (ctypes.c_int64 * 4)()
            self.ctx.check(self.ctx.lib.pqb_plan(self.ctx.h, key[0], key[1], c))
            self.plan_counts = dict(shell_quartets=c[0], fp64=c[1], fp32=c[2], dropped=c[3])
            self._plan_key = key
        return self.plan_counts

    def packed_len(self):
        P = self.nbf * (self.nbf + 1) // 2
        return P * (P + 1) // 2

    def eri_packed(self, out=None, stream=None):
        self._need_shells()
        Q = self.packed_len()
        if out is None:
            out = torch.empty(Q, dtype=torch.float64, device=self.device)
        self.ctx.check(self.ctx.lib.pqb_eri_packed(self.ctx.h, ptr(out), Q, stream_ptr(stream)))
        return out

    def jk(self, D, mode="fp64", schwarz=1e-12, fp32_threshold=1e-5, J=None, K=None, stream=None):
        """Integral-direct J and K for a symmetric density D (device tensor)."""
        self._need_shells()
        self.plan(schwarz, fp32_threshold)
        D = D.to(device=self.device, dtype=torch.float64).contiguous()
        if J is None:
            J = torch.empty_like(D)
        if K is None:
            K = torch.empty_like(D)
        m = _lib.PQB_MIXED if mode == "mixed" else _lib.PQB_FP64
        self.ctx.check(self.ctx.lib.pqb_jk_direct(self.ctx.h, ptr(D), ptr(J), ptr(K), m, stream_ptr(stream)))
        return J, K

    def j(self, D, mode="fp64", schwarz=1e-12, fp32_threshold=1e-5, J=None, stream=None):
        """Integral-direct Coulomb matrix alone (no exchange digestion)."""
        self._need_shells()
        self.plan(schwarz, fp32_threshold)
        D = D.to(device=self.device, dtype=torch.float64).contiguous()
        if J is None:
            J = torch.empty_like(D)
        m = _lib.PQB_MIXED if mode == "mixed" else _lib.PQB_FP64
        self.ctx.check(self.ctx.lib.pqb_jk_direct(self.ctx.h, ptr(D), ptr(J), None, m, stream_ptr(stream)))
        return J

    def get2jmk_host(self, D, G, mode="fp64", schwarz=1e-12, fp32_threshold=1e-5, stream=None):
        """G = 2J - K into the host array G for the host density D (CPU
        tensors or numpy arrays, float64, C-contiguous, nbf x nbf): one
        pqb_get2jmk_host call that copies D in, builds and copies G out on the
        stream; G is complete after a stream synchronisation."""
        self._need_shells()
        self.plan(schwarz, fp32_threshold)
        n = self.nbf
        for x in (D, G):
            if isinstance(x, torch.Tensor):
                ok = (not x.is_cuda) and x.dtype == torch.float64 and x.is_contiguous()
            else:
                ok = x.dtype == np.float64 and x.flags.c_contiguous
            if not ok or tuple(x.shape) != (n, n):
                raise ValueError("get2jmk_host: D and G must be C-contiguous float64 host arrays of shape (%d, %d)"
                                 % (n, n))
        m = _lib.PQB_MIXED if mode == "mixed" else _lib.PQB_FP64
        self.ctx.check(self.ctx.lib.pqb_get2jmk_host(self.ctx.h, _host_ptr(D), _host_ptr(G), m, stream_ptr(stream)))
        return G

    def jk2(self, Da, Db, mode="fp64", schwarz=1e-12, fp32_threshold=1e-5, stream=None):
        """J and K of two densities (UHF alpha and beta) from one pass over the
        integrals: (Ja, Ka, Jb, Kb)."""
        self._need_shells()
        self.plan(schwarz, fp32_threshold)
        Da = Da.to(device=self.device, dtype=torch.float64).contiguous()
        Db = Db.to(device=self.device, dtype=torch.float64).contiguous()
        out = [torch.empty_like(Da) for _ in range(4)]
        m = _lib.PQB_MIXED if mode == "mixed" else _lib.PQB_FP64
        self.ctx.check(self.ctx.lib.pqb_jk_direct2(self.ctx.h, ptr(Da), ptr(Db), *(ptr(x) for x in out), m,
                                                   stream_ptr(stream)))
        return tuple(out)

    def oneint(self, atoms, stream=None):
        return oneint(self.ft, atoms, self.ctx, stream)


def jk_packed(ints, D, ctx=None, stream=None):
    """J and K from stored packed integrals (device tensors)."""
    ctx = ctx or _lib.context(ints.device.index)
    n = D.shape[0]
    D = D.contiguous()
    J = torch.empty_like(D)
    K = torch.empty_like(D)
    ctx.check(ctx.lib.pqb_jk_packed(ctx.h, ptr(ints), ints.numel(), ptr(D), ptr(J), ptr(K), n, stream_ptr(stream)))
    return J, K
