"""ctypes binding of libhfg.so (include/hfg.h)."""
import ctypes
import os

import numpy as np

PKG_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(os.path.dirname(PKG_ROOT), "include", "hfg.h")

HFG_FP64, HFG_MIXED = 0, 1
STATUS = {0: "OK", 1: "INVALID_INPUT", 2: "INTEGRAL", 3: "SCF", 4: "OOM", 5: "TIMEOUT", 6: "CUDA", 7: "UNSUPPORTED"}


def library_path():
    return os.path.join(PKG_ROOT, "libhfg.so")


class HfgError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("%s: %s" % (STATUS.get(code, str(code)), msg))
        self.code = code


class HfgBasis(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int), ("center", ctypes.POINTER(ctypes.c_double)),
                ("lxyz", ctypes.POINTER(ctypes.c_int)), ("atom", ctypes.POINTER(ctypes.c_int)),
                ("prim_off", ctypes.POINTER(ctypes.c_int)), ("exps", ctypes.POINTER(ctypes.c_double)),
                ("coefs", ctypes.POINTER(ctypes.c_double))]


class JKOptions(ctypes.Structure):
    _fields_ = [("schwarz_threshold", ctypes.c_double), ("prim_threshold", ctypes.c_double),
                ("precision", ctypes.c_int), ("mixed_threshold", ctypes.c_double)]

    @classmethod
    def make(cls, schwarz=1e-12, prim=0.0, mixed=None):
        o = cls()
        o.schwarz_threshold = schwarz
        o.prim_threshold = prim
        o.precision = HFG_FP64 if mixed is None else HFG_MIXED
        o.mixed_threshold = 0.0 if mixed is None else mixed
        return o


class JKStats(ctypes.Structure):
    _fields_ = [("quartets_fp64", ctypes.c_double), ("quartets_fp32", ctypes.c_double),
                ("prim_quartets_fp64", ctypes.c_double), ("prim_quartets_fp32", ctypes.c_double),
                ("wmd_flops_fp64", ctypes.c_double), ("wmd_flops_fp32", ctypes.c_double),
                ("launches", ctypes.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_lib = None
DP = ctypes.POINTER(ctypes.c_double)
VP = ctypes.c_void_p


def _dp(a):
    return a.ctypes.data_as(DP)


def _ip(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


def load_library():
    """Load libhfg.so; raise if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    path = library_path()
    if not os.path.exists(path):
        raise HfgError(6, "libhfg.so not built (run __graft_entry__.build())")
    L = ctypes.CDLL(path)
    P = ctypes.POINTER
    L.hfg_jk_opts_default.argtypes = [P(JKOptions)]
    L.hfg_ctx_create.argtypes = [P(HfgBasis), ctypes.c_int, VP, P(VP)]
    L.hfg_ctx_destroy.argtypes = [VP]
    L.hfg_last_error.argtypes = [VP]
    L.hfg_last_error.restype = ctypes.c_char_p
    L.hfg_ctx_sizes.argtypes = [VP, P(ctypes.c_int), P(ctypes.c_int), P(ctypes.c_long)]
    L.hfg_schwarz.argtypes = [VP, DP, ctypes.c_long]
    L.hfg_shell_quartet.argtypes = [VP, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, DP]
    L.hfg_jk.argtypes = [VP, P(JKOptions), ctypes.c_int, DP, DP, DP, DP]
    L.hfg_jk_device.argtypes = [VP, P(JKOptions), ctypes.c_int, VP, VP, VP, VP]
    L.hfg_jk_device_noalloc.argtypes = [VP, P(JKOptions), ctypes.c_int, VP, VP, VP, VP]
    L.hfg_fock_rhf.argtypes = [VP, P(JKOptions), DP, DP, DP]
    L.hfg_fock_uhf.argtypes = [VP, P(JKOptions), DP, DP, DP, DP, DP]
    L.hfg_jk_last_stats.argtypes = [VP, P(JKStats)]
    L.hfg_fma_peak.argtypes = [ctypes.c_int, ctypes.c_int, DP]
    _lib = L
    return L


def exported_functions():
    """Function names declared in include/hfg.h."""
    import re
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|void|const char\*)\s+(hfg_\w+)\s*\(", txt, re.M)))


def fma_peak_tflops(device=0, fp32=False):
    """Measured FP64 (or FP32) FMA-pipe peak of the device (hfg_fma_peak)."""
    L = load_library()
    out = ctypes.c_double()
    rc = L.hfg_fma_peak(device, 1 if fp32 else 0, ctypes.byref(out))
    if rc != 0:
        raise HfgError(rc, "hfg_fma_peak failed")
    return out.value


class Context:
    """One basis on one device (hfg_ctx)."""

    def __init__(self, basis, device=0, stream=None):
        self.lib = load_library()
        self.basis = basis
        self._keep = basis
        self._b = HfgBasis(basis.n, _dp(basis.center), _ip(basis.lxyz), _ip(basis.atom), _ip(basis.prim_off),
                           _dp(basis.exps), _dp(basis.coefs))
        h = VP()
        if stream == 0:
            raise HfgError(1, "pass a non-default CUDA stream (or None for a context-owned stream)")
        rc = self.lib.hfg_ctx_create(ctypes.byref(self._b), device, stream, ctypes.byref(h))
        self.h = h
        if rc != 0:
            msg = self.lib.hfg_last_error(h).decode() if h.value else "context creation failed"
            self.close()
            raise HfgError(rc, msg)
        self.n = basis.n

    def _check(self, rc):
        if rc != 0:
            raise HfgError(rc, self.lib.hfg_last_error(self.h).decode())

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            self.lib.hfg_ctx_destroy(self.h)
            self.h = VP()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def sizes(self):
        a, s, p = ctypes.c_int(), ctypes.c_int(), ctypes.c_long()
        self._check(self.lib.hfg_ctx_sizes(self.h, ctypes.byref(a), ctypes.byref(s), ctypes.byref(p)))
        return a.value, s.value, p.value

    def schwarz(self):
        _, _, npair = self.sizes()
        out = np.zeros(npair)
        self._check(self.lib.hfg_schwarz(self.h, _dp(out), npair))
        return out

    def shell_quartet(self, a, b, c, d, dims):
        out = np.zeros(int(np.prod(dims)))
        self._check(self.lib.hfg_shell_quartet(self.h, a, b, c, d, _dp(out)))
        return out

    def jk(self, P_total, P_spin=None, opts=None):
        """J and K (list) from host densities (hfg_jk)."""
        n = self.n
        pt = np.ascontiguousarray(P_total, dtype=np.float64)
        spins = [pt] if P_spin is None else list(P_spin)
        ps = np.ascontiguousarray(np.stack(spins), dtype=np.float64)
        J = np.zeros((n, n))
        K = np.zeros((len(spins), n, n))
        o = opts or JKOptions.make()
        self._check(self.lib.hfg_jk(self.h, ctypes.byref(o), len(spins), _dp(pt), _dp(ps), _dp(J), _dp(K)))
        return J, K

    def jk_device(self, d_total, d_spin, d_J, d_K, nspin=1, opts=None):
        """Device-pointer form (integers); runs on the context stream."""
        o = opts or JKOptions.make()
        self._check(self.lib.hfg_jk_device(self.h, ctypes.byref(o), nspin, d_total, d_spin, d_J, d_K))

    def fock_rhf(self, H, P, opts=None):
        n = self.n
        F = np.zeros((n, n))
        o = opts or JKOptions.make()
        self._check(self.lib.hfg_fock_rhf(self.h, ctypes.byref(o), _dp(np.ascontiguousarray(H)),
                                          _dp(np.ascontiguousarray(P)), _dp(F)))
        return F

    def fock_uhf(self, H, Pa, Pb, opts=None):
        n = self.n
        Fa, Fb = np.zeros((n, n)), np.zeros((n, n))
        o = opts or JKOptions.make()
        self._check(self.lib.hfg_fock_uhf(self.h, ctypes.byref(o), _dp(np.ascontiguousarray(H)),
                                          _dp(np.ascontiguousarray(Pa)), _dp(np.ascontiguousarray(Pb)),
                                          _dp(Fa), _dp(Fb)))
        return Fa, Fb

    def last_stats(self):
        s = JKStats()
        self._check(self.lib.hfg_jk_last_stats(self.h, ctypes.byref(s)))
        return s.as_dict()
