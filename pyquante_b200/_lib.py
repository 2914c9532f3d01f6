"""ctypes binding of ``libpyquante_b200.so`` (the C ABI in include/pyquante_b200.h).

The library is built in-tree by ``pyquante_b200.csrc.build``.  There is no
CPU fallback: if the library or a CUDA device is missing, every entry point
raises ``EngineUnavailable``.
"""
import ctypes
import os
import threading

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libpyquante_b200.so")

PQB_OK, PQB_E_ARG, PQB_E_CLASS, PQB_E_NPRIM, PQB_E_SHAPE, PQB_E_CUDA, PQB_E_STATE, PQB_E_TIMEOUT, PQB_E_NOMEM = range(9)
PQB_FP64, PQB_MIXED = 0, 1
PQB_ENGINE_RYS, PQB_ENGINE_HGP = 0, 1
(PQB_PARAM_CHUNK, PQB_PARAM_STREAMS, PQB_PARAM_ORDER, PQB_PARAM_PACKED_KERNEL, PQB_PARAM_GRAPH,
 PQB_PARAM_THREADS) = 0, 1, 2, 3, 4, 5

_c_int_p = ctypes.POINTER(ctypes.c_int)
_c_dbl_p = ctypes.POINTER(ctypes.c_double)
_c_i64_p = ctypes.POINTER(ctypes.c_int64)
_vp = ctypes.c_void_p

# name -> (restype, argtypes); every symbol declared in include/pyquante_b200.h
SIGNATURES = {
    "pqb_version": (ctypes.c_int, []),
    "pqb_create": (ctypes.c_int, [ctypes.POINTER(_vp), ctypes.c_int]),
    "pqb_destroy": (None, [_vp]),
    "pqb_last_error": (ctypes.c_int, [_vp, ctypes.c_char_p, ctypes.c_size_t]),
    "pqb_shells_upload": (ctypes.c_int, [_vp, ctypes.c_int, _c_int_p, _c_int_p, _c_int_p, _c_int_p, _c_dbl_p,
                                         _c_dbl_p, _c_dbl_p, ctypes.c_int, _c_dbl_p]),
    "pqb_shells_upload_batch": (ctypes.c_int, [_vp, ctypes.c_int, _c_int_p, ctypes.c_int, _c_int_p, _c_int_p,
                                               _c_int_p, _c_int_p, _c_dbl_p, _c_dbl_p, _c_dbl_p, ctypes.c_int,
                                               _c_dbl_p]),
    "pqb_dense_len": (ctypes.c_int, [_vp, _c_i64_p]),
    "pqb_set_molecule_mask": (ctypes.c_int, [_vp, _vp]),
    "pqb_set_density_screen": (ctypes.c_int, [_vp, _vp, ctypes.c_double]),
    "pqb_shell_dmax": (ctypes.c_int, [_vp, _vp, _vp, _vp]),
    "pqb_purify_step": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _vp, _vp, _vp, _vp, _vp, ctypes.c_double, _vp]),
    "pqb_schwarz": (ctypes.c_int, [_vp, _c_dbl_p, _vp]),
    "pqb_num_pairs": (ctypes.c_int, [_vp]),
    "pqb_plan": (ctypes.c_int, [_vp, ctypes.c_double, ctypes.c_double, _c_i64_p]),
    "pqb_set_param": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "pqb_plan_stats": (ctypes.c_int, [_vp, _c_i64_p, _c_i64_p]),
    "pqb_plan_shard": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int]),
    "pqb_fp64_peak": (ctypes.c_int, [_vp, ctypes.c_int, _c_dbl_p]),
    "pqb_eri_packed": (ctypes.c_int, [_vp, _vp, ctypes.c_int64, _vp]),
    "pqb_jk_direct": (ctypes.c_int, [_vp, _vp, _vp, _vp, ctypes.c_int, _vp]),
    "pqb_get2jmk_host": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_int, _vp]),
    "pqb_jk_direct2": (ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, ctypes.c_int, _vp]),
    "pqb_jk_direct_class": (ctypes.c_int, [_vp, _vp, _vp, _vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp]),
    "pqb_jk_packed": (ctypes.c_int, [_vp, _vp, ctypes.c_int64, _vp, _vp, _vp, ctypes.c_int, _vp]),
    "pqb_eri_functions": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp, ctypes.c_int, _vp, _vp, _vp, _vp,
                                         _vp, _vp, _vp, _vp]),
    "pqb_oneint": (ctypes.c_int, [_vp, ctypes.c_int, _vp, _vp, _vp, _vp, _vp, _vp, ctypes.c_int, _c_dbl_p,
                                  _c_dbl_p, _vp, _vp, _vp, _vp]),
    "pqb_oneint_noalloc": (ctypes.c_int, [ctypes.c_int, _vp, _vp, _vp, _vp, _vp, _vp, ctypes.c_int, _vp, _vp,
                                          _vp, _vp, _vp, _vp]),
    "pqb_set_shell_atoms": (ctypes.c_int, [_vp, _c_int_p]),
    "pqb_grad_2e": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_int, _vp]),
    "pqb_grad_1e": (ctypes.c_int, [_vp, ctypes.c_int, _vp, _vp, _vp, _vp, _vp, _vp, _vp, ctypes.c_int, _c_dbl_p,
                                   _c_dbl_p, _vp, _vp, _vp, _vp]),
    "pqb_mo_unpack_rows": (ctypes.c_int, [_vp, ctypes.c_int64, ctypes.c_int, ctypes.c_int64, ctypes.c_int, _vp, _vp]),
    "pqb_mo_unpack_pairs": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int64, _vp, _vp]),
    "pqb_mo_pack": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, _vp, ctypes.c_int64, _vp]),
    "pqb_mp2_pairs": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, _vp, _vp, _vp, _vp]),
    "pqb_becke_weights": (ctypes.c_int, [ctypes.c_int, _vp, _vp, ctypes.c_int, _vp, _vp, _vp, _vp]),
    "pqb_grid_amps": (ctypes.c_int, [ctypes.c_int, _vp, _vp, _vp, _vp, _vp, _vp, ctypes.c_int, _vp, _vp, _vp]),
    "pqb_grid_rowdot": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _vp, _vp, _vp, _vp]),
    "pqb_xc_svwn": (ctypes.c_int, [ctypes.c_int, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "pqb_ijkl2intindex": (ctypes.c_int64, [ctypes.c_int64] * 4),
    "pqb_boys_eval": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, _vp, _vp, _vp]),
    "pqb_boys_rows_eval": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, _vp, _vp, _vp]),
    "pqb_rys_eval": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, _vp, _vp, _vp, _vp]),
}


class EngineUnavailable(RuntimeError):
    """The CUDA engine (library or device) is not available."""


class EngineError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("pyquante_b200 error %d: %s" % (code, msg))
        self.code = code


_lib = None
_lock = threading.Lock()


def load():
    """Load the shared library (no device needed). Raises EngineUnavailable."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise EngineUnavailable("%s not built; run python -m pyquante_b200.csrc.build" % LIB_PATH)
            lib = ctypes.CDLL(LIB_PATH)
            for name, (res, args) in SIGNATURES.items():
                fn = getattr(lib, name)
                fn.restype = res
                fn.argtypes = args
            _lib = lib
    return _lib


class Context:
    """Owns one ``pqb_ctx`` on one CUDA device."""

    def __init__(self, device=0):
        import torch
        if not torch.cuda.is_available():
            raise EngineUnavailable("no CUDA device: the engine has no CPU fallback")
        self.lib = load()
        self.device = device
        h = ctypes.c_void_p()
        rc = self.lib.pqb_create(ctypes.byref(h), device)
        if rc != PQB_OK:
            raise EngineError(rc, "pqb_create(device=%d) failed" % device)
        self.h = h

    def check(self, rc):
        if rc != PQB_OK:
            buf = ctypes.create_string_buffer(512)
            self.lib.pqb_last_error(self.h, buf, 512)
            raise EngineError(rc, buf.value.decode(errors="replace"))

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            try:
                self.lib.pqb_destroy(h)
            except Exception:
                pass
            self.h = None


_contexts = {}


def context(device=None):
    """Process-wide context for ``device`` (default: torch's current device)."""
    import torch
    if not torch.cuda.is_available():
        raise EngineUnavailable("no CUDA device: the engine has no CPU fallback")
    if device is None:
        device = torch.cuda.current_device()
    with _lock:
        ctx = _contexts.get(device)
    if ctx is None:
        ctx = Context(device)
        with _lock:
            _contexts[device] = ctx
    return ctx


def ptr(t):
    """Raw device pointer of a torch tensor (None -> NULL)."""
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def stream_ptr(stream=None):
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)
