"""ctypes binding of libhfg.so (include/hfg.h)."""
import ctypes
import os

import numpy as np

PKG_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(os.path.dirname(PKG_ROOT), "include", "hfg.h")

HFG_FP64, HFG_MIXED = 0, 1
STATUS = {0: "OK", 1: "INVALID_INPUT", 2: "INTEGRAL", 3: "SCF", 4: "OOM", 5: "TIMEOUT", 6: "CUDA", 7: "UNSUPPORTED"}


def library_path():
    """The in-tree libhfg.so, or the build named by HFG_LIBRARY (a tuning
    build of the same sources)."""
    return os.environ.get("HFG_LIBRARY") or os.path.join(PKG_ROOT, "libhfg.so")


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
                ("precision", ctypes.c_int), ("deterministic", ctypes.c_int), ("mixed_threshold", ctypes.c_double),
                ("tile", ctypes.c_int)]

    @classmethod
    def make(cls, schwarz=1e-12, prim=0.0, mixed=None, deterministic=False, tile=0):
        o = cls()
        o.schwarz_threshold = schwarz
        o.prim_threshold = prim
        o.precision = HFG_FP64 if mixed is None else HFG_MIXED
        o.deterministic = int(bool(deterministic))
        o.mixed_threshold = 0.0 if mixed is None else mixed
        o.tile = tile
        return o

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class SCFOptions(ctypes.Structure):
    _fields_ = [("natom", ctypes.c_int), ("positions", ctypes.POINTER(ctypes.c_double)),
                ("charges", ctypes.POINTER(ctypes.c_double)), ("charge", ctypes.c_int),
                ("multiplicity", ctypes.c_int), ("uhf", ctypes.c_int), ("spherical", ctypes.c_int),
                ("max_iter", ctypes.c_int), ("energy_tol", ctypes.c_double), ("residual_tol", ctypes.c_double),
                ("density_tol", ctypes.c_double), ("jk", JKOptions), ("refine_iters", ctypes.c_int),
                ("diis_size", ctypes.c_int), ("verbose", ctypes.c_int), ("guess", ctypes.c_int),
                ("incremental_tol", ctypes.c_double), ("rebuild_every", ctypes.c_int),
                ("refine_at", ctypes.c_double)]


class SCFResult(ctypes.Structure):
    _fields_ = [("energy", ctypes.c_double), ("electronic", ctypes.c_double), ("nuclear", ctypes.c_double),
                ("energy_before_refinement", ctypes.c_double), ("s2", ctypes.c_double),
                ("iterations", ctypes.c_int), ("converged", ctypes.c_int), ("n_mo", ctypes.c_int),
                ("fock_builds_fp64", ctypes.c_int), ("fock_builds_mixed", ctypes.c_int), ("time_ms", ctypes.c_double),
                ("fock_builds_incremental", ctypes.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


def convergence_from_tol(tol):
    """Residual and density tolerances hf-rs derives from an energy tolerance
    (src/scf.rs:393-399)."""
    import math
    return tol, max(math.sqrt(tol) * 1e-2, 1e-11), min(max(math.sqrt(tol) * 0.1, 1e-12), 1e-10)


class Job(ctypes.Structure):
    _fields_ = [("basis", HfgBasis), ("natom", ctypes.c_int), ("positions", ctypes.POINTER(ctypes.c_double)),
                ("charges", ctypes.POINTER(ctypes.c_double)), ("charge", ctypes.c_int),
                ("multiplicity", ctypes.c_int), ("uhf", ctypes.c_int), ("spherical", ctypes.c_int),
                ("max_iter", ctypes.c_int), ("energy_tol", ctypes.c_double), ("residual_tol", ctypes.c_double),
                ("density_tol", ctypes.c_double), ("jk", JKOptions), ("tag", ctypes.c_longlong)]


class JobResult(ctypes.Structure):
    _fields_ = [("tag", ctypes.c_longlong), ("status", ctypes.c_int), ("iterations", ctypes.c_int),
                ("converged", ctypes.c_int), ("n_ao", ctypes.c_int), ("energy", ctypes.c_double),
                ("energy_before_refinement", ctypes.c_double), ("submit_ms", ctypes.c_double),
                ("start_ms", ctypes.c_double), ("end_ms", ctypes.c_double), ("footprint_bytes", ctypes.c_longlong)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class JKStats(ctypes.Structure):
    _fields_ = [("quartets_fp64", ctypes.c_double), ("quartets_fp32", ctypes.c_double),
                ("prim_quartets_fp64", ctypes.c_double), ("prim_quartets_fp32", ctypes.c_double),
                ("wmd_flops_fp64", ctypes.c_double), ("wmd_flops_fp32", ctypes.c_double),
                ("launches", ctypes.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class AutotuneOptions(ctypes.Structure):
    _fields_ = [("fp32_thresholds", ctypes.c_double * 8), ("n_fp32", ctypes.c_int),
                ("prim_thresholds", ctypes.c_double * 8), ("n_prim", ctypes.c_int),
                ("max_energy_error", ctypes.c_double), ("repeats", ctypes.c_int),
                ("tiles", ctypes.c_int * 4), ("n_tile", ctypes.c_int)]


class AutotuneResult(ctypes.Structure):
    _fields_ = [("best", JKOptions), ("found", ctypes.c_int), ("best_ms", ctypes.c_double),
                ("best_energy_error", ctypes.c_double), ("fp64_ms", ctypes.c_double), ("evaluated", ctypes.c_int),
                ("ms", ctypes.c_double * 64), ("energy_error", ctypes.c_double * 64)]


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
    L.hfg_eri_packed.argtypes = [VP, ctypes.c_double, DP, ctypes.c_size_t]
    L.hfg_eri_packed_device.argtypes = [VP, ctypes.c_double, VP, ctypes.c_size_t]
    L.hfg_jk.argtypes = [VP, P(JKOptions), ctypes.c_int, DP, DP, DP, DP]
    L.hfg_jk_device.argtypes = [VP, P(JKOptions), ctypes.c_int, VP, VP, VP, VP]
    L.hfg_jk_device_shard.argtypes = [VP, P(JKOptions), ctypes.c_int, VP, VP, VP, VP, ctypes.c_int, ctypes.c_int]
    L.hfg_jk_device_noalloc.argtypes = [VP, P(JKOptions), ctypes.c_int, VP, VP, VP, VP]
    L.hfg_jk_device_batch.argtypes = [P(VP), ctypes.c_int, P(JKOptions), P(VP), P(VP), P(VP), VP]
    L.hfg_eri_gradient.argtypes = [VP, ctypes.c_double, ctypes.c_int, DP, DP, ctypes.c_int, DP]
    L.hfg_gradient.argtypes = [VP, ctypes.c_int, DP, DP, ctypes.c_int, DP, DP, DP, ctypes.c_double, DP]
    L.hfg_fock_rhf.argtypes = [VP, P(JKOptions), DP, DP, DP]
    L.hfg_fock_uhf.argtypes = [VP, P(JKOptions), DP, DP, DP, DP, DP]
    L.hfg_jk_last_stats.argtypes = [VP, P(JKStats)]
    L.hfg_autotune_opts_default.argtypes = [P(AutotuneOptions)]
    L.hfg_jk_autotune.argtypes = [VP, P(JKOptions), ctypes.c_int, VP, VP, P(AutotuneOptions), P(AutotuneResult)]
    L.hfg_fma_peak.argtypes = [ctypes.c_int, ctypes.c_int, DP]
    L.hfg_scf_opts_default.argtypes = [P(SCFOptions)]
    L.hfg_df_build.argtypes = [VP, P(HfgBasis), ctypes.c_double, ctypes.c_double, ctypes.c_int, P(VP)]
    L.hfg_df_build_shard.argtypes = [VP, P(HfgBasis), ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                     ctypes.c_int, P(VP)]
    L.hfg_df_destroy.argtypes = [VP]
    L.hfg_df_sizes.argtypes = [VP, P(ctypes.c_int), P(ctypes.c_int), P(ctypes.c_longlong)]
    L.hfg_df_metric.argtypes = [VP, DP]
    L.hfg_df_three_center.argtypes = [VP, P(HfgBasis), DP, ctypes.c_size_t]
    L.hfg_df_jk.argtypes = [VP, DP, ctypes.c_int, DP, DP, ctypes.c_int]
    L.hfg_df_last_stats.argtypes = [VP, DP, DP, DP]
    L.hfg_df_jk_shard.argtypes = [VP, DP, ctypes.c_int, DP, DP, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    L.hfg_df_jk_device_shard.argtypes = [VP, VP, ctypes.c_int, VP, VP, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    L.hfg_df_transform.argtypes = [VP, DP, ctypes.c_int, DP, ctypes.c_size_t]
    L.hfg_df_mp2.argtypes = [VP, DP, DP, ctypes.c_int, ctypes.c_int, ctypes.c_int, DP]
    L.hfg_cholesky_eri.argtypes = [VP, ctypes.c_double, ctypes.c_size_t, P(VP), DP, P(ctypes.c_longlong), ctypes.c_int,
                                   P(ctypes.c_int)]
    L.hfg_scf_df.argtypes = [VP, VP, ctypes.c_int, P(SCFOptions), P(SCFResult), DP, DP, DP, DP]
    L.hfg_server_create.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_longlong, P(VP)]
    L.hfg_server_submit.argtypes = [VP, P(Job)]
    L.hfg_server_poll.argtypes = [VP, P(JobResult), ctypes.c_int, P(ctypes.c_int), ctypes.c_int]
    L.hfg_server_stats.argtypes = [VP, P(ctypes.c_int), P(ctypes.c_int), P(ctypes.c_longlong)]
    L.hfg_server_set_mixed_min_ao.argtypes = [VP, ctypes.c_int]
    L.hfg_server_set_batching.argtypes = [VP, ctypes.c_int, ctypes.c_double]
    L.hfg_server_batch_stats.argtypes = [VP, P(ctypes.c_longlong), P(ctypes.c_longlong)]
    L.hfg_server_destroy.argtypes = [VP]
    L.hfg_scf.argtypes = [VP, P(SCFOptions), P(SCFResult), DP, DP, DP, DP]
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
        """Destroy the context; DF tensors built on it are destroyed first
        (each holds a pointer into the context)."""
        for child in list(getattr(self, "_children", ())):
            child.close()
        if getattr(self, "h", None) is not None and self.h.value:
            self.lib.hfg_ctx_destroy(self.h)
            self.h = VP()

    def _adopt(self, child):
        import weakref
        if not hasattr(self, "_children"):
            self._children = weakref.WeakSet()
        self._children.add(child)

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

    def eri_packed(self, threshold=1e-12, length=None):
        """Packed 8-fold ERI tensor (hfg_eri_packed), hf-rs's compute_eri_tensor
        layout."""
        n = self.n
        npair = n * (n + 1) // 2
        length = npair * (npair + 1) // 2 if length is None else length
        out = np.zeros(length)
        self._check(self.lib.hfg_eri_packed(self.h, threshold, _dp(out), length))
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

    def jk_device_shard(self, d_total, d_spin, d_J, d_K, shard, nshards, nspin=1, opts=None):
        """One cost-balanced shard of the device build (hfg_jk_device_shard)."""
        o = opts or JKOptions.make()
        self._check(self.lib.hfg_jk_device_shard(self.h, ctypes.byref(o), nspin, d_total, d_spin, d_J, d_K, shard,
                                                 nshards))

    def jk_device(self, d_total, d_spin, d_J, d_K, nspin=1, opts=None):
        """Device-pointer form (integers); runs on the context stream."""
        o = opts or JKOptions.make()
        self._check(self.lib.hfg_jk_device(self.h, ctypes.byref(o), nspin, d_total, d_spin, d_J, d_K))

    def eri_gradient(self, P_total, P_spin=None, schwarz=1e-12):
        """Two-electron part of the nuclear gradient (hfg_eri_gradient):
        (natom, 3) array of dE2/dR for the context's basis; P_spin None for
        a closed shell, else the two spin densities."""
        pt = np.ascontiguousarray(P_total, dtype=np.float64)
        spins = [pt] if P_spin is None else list(P_spin)
        ps = np.ascontiguousarray(np.stack(spins), dtype=np.float64)
        natom = int(np.max(self.basis.atom)) + 1
        g = np.zeros((natom, 3))
        self._check(self.lib.hfg_eri_gradient(self.h, schwarz, len(spins), _dp(pt), _dp(ps), natom, _dp(g)))
        return g

    def gradient(self, P_total, W, P_spin=None, schwarz=1e-12):
        """Analytic nuclear gradient (hfg_gradient), (natom, 3) in hartree/bohr,
        from the SCF's total density, energy-weighted density W and (open
        shell) spin densities, all in the Cartesian basis."""
        b = self.basis
        pos = np.ascontiguousarray(b.positions())
        chg = np.ascontiguousarray(b.nuclear_charges())
        pt = np.ascontiguousarray(P_total, dtype=np.float64)
        spins = [pt] if P_spin is None else list(P_spin)
        ps = np.ascontiguousarray(np.stack(spins), dtype=np.float64)
        w = np.ascontiguousarray(W, dtype=np.float64)
        g = np.zeros((len(chg), 3))
        self._check(self.lib.hfg_gradient(self.h, len(chg), _dp(pos), _dp(chg), len(spins), _dp(pt), _dp(ps), _dp(w),
                                          schwarz, _dp(g)))
        return g

    def scf_gradient(self, charge=0, multiplicity=1, uhf=False, spherical=False, tol=1e-10, max_iter=100):
        """SCF (hfg_scf) and its analytic gradient: returns (result dict,
        (natom, 3) gradient).  W = sum over occupied orbitals of eps C C^T
        per spin (x 2 for a closed shell)."""
        r = self.scf(charge=charge, multiplicity=multiplicity, uhf=uhf, spherical=spherical, tol=tol,
                     max_iter=max_iter, want=("P", "C", "eps"))
        nel = int(round(float(np.sum(self.basis.nuclear_charges())))) - charge
        if uhf:
            na = (nel + multiplicity - 1) // 2
            occ = [na, nel - na]
            W = sum(r["C"][s][:, :occ[s]] @ np.diag(r["eps"][s][:occ[s]]) @ r["C"][s][:, :occ[s]].T for s in range(2))
            g = self.gradient(r["P"][0] + r["P"][1], W, P_spin=[r["P"][0], r["P"][1]])
        else:
            no = nel // 2
            C = r["C"][0][:, :no]
            W = 2.0 * C @ np.diag(r["eps"][0][:no]) @ C.T
            g = self.gradient(r["P"][0], W)
        return r, g

    @staticmethod
    def jk_device_batch(contexts, d_P, d_J, d_K, opts=None, stream=None):
        """RHF J and K of several molecules in one pass (hfg_jk_device_batch):
        one context per molecule, device-pointer lists (integers).  Runs on
        `stream` (None: the first context's stream) and does not synchronise."""
        m = len(contexts)
        if not (len(d_P) == len(d_J) == len(d_K) == m) or m == 0:
            raise ValueError("one density, J and K per context")
        arr = lambda xs: (VP * m)(*[VP(int(x)) for x in xs])
        hs = (VP * m)(*[c.h for c in contexts])
        o = opts or JKOptions.make()
        c0 = contexts[0]
        c0._check(c0.lib.hfg_jk_device_batch(hs, m, ctypes.byref(o), arr(d_P), arr(d_J), arr(d_K),
                                             VP(int(stream) if stream else 0)))

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

    def scf(self, charge=0, multiplicity=1, uhf=False, spherical=False, tol=1e-10, max_iter=100, jk=None,
            refine_iters=2, verbose=False, want=("P", "F"), guess="sad", incremental=1e-12, rebuild_every=8,
            refine_at=10.0):
        """Device SCF (hfg_scf) for the context's molecule; returns a dict.
        `incremental` (mixed J/K only): screening tolerance of the builds from
        density changes, 0 for a full build every iteration."""
        b = self.basis
        o = SCFOptions()
        self.lib.hfg_scf_opts_default(ctypes.byref(o))
        pos = np.ascontiguousarray(b.positions())
        chg = np.ascontiguousarray(b.nuclear_charges())
        o.natom = len(chg)
        o.positions = _dp(pos)
        o.charges = _dp(chg)
        o.charge, o.multiplicity, o.uhf, o.spherical = charge, multiplicity, int(uhf), int(spherical)
        o.max_iter = max_iter
        o.energy_tol, o.residual_tol, o.density_tol = convergence_from_tol(tol)
        o.jk = jk or JKOptions.make()
        o.refine_iters = refine_iters
        o.verbose = int(verbose)
        o.guess = 0 if guess == "sad" else 1
        o.incremental_tol = incremental
        o.rebuild_every = rebuild_every
        o.refine_at = refine_at
        n = self.n
        ns = 2 if uhf else 1
        P = np.zeros((ns, n, n)) if "P" in want else None
        F = np.zeros((ns, n, n)) if "F" in want else None
        C = np.zeros((ns, n, n)) if "C" in want else None
        eps = np.zeros((ns, n)) if "eps" in want else None
        r = SCFResult()
        rc = self.lib.hfg_scf(self.h, ctypes.byref(o), ctypes.byref(r), _dp(P) if P is not None else None,
                              _dp(F) if F is not None else None, _dp(C) if C is not None else None,
                              _dp(eps) if eps is not None else None)
        if rc not in (0, 3):
            self._check(rc)
        out = r.as_dict()
        m = r.n_mo
        out.update({"P": P, "F": F, "C": None if C is None else C.reshape(ns, -1)[:, :n * m].reshape(ns, n, m),
                    "eps": None if eps is None else eps[:, :m], "status": rc})
        return out

    def _scf_opts(self, charge, multiplicity, uhf, spherical, tol, max_iter, jk, refine_iters, verbose, keep):
        b = self.basis
        o = SCFOptions()
        self.lib.hfg_scf_opts_default(ctypes.byref(o))
        pos = np.ascontiguousarray(b.positions())
        chg = np.ascontiguousarray(b.nuclear_charges())
        keep.extend([pos, chg])
        o.natom = len(chg)
        o.positions = _dp(pos)
        o.charges = _dp(chg)
        o.charge, o.multiplicity, o.uhf, o.spherical = charge, multiplicity, int(uhf), int(spherical)
        o.max_iter = max_iter
        if isinstance(tol, tuple):
            o.energy_tol, o.residual_tol, o.density_tol = tol
        else:
            o.energy_tol, o.residual_tol, o.density_tol = convergence_from_tol(tol)
        o.jk = jk or JKOptions.make()
        o.refine_iters = refine_iters
        o.verbose = int(verbose)
        return o

    def scf_df(self, df, mma=0, charge=0, spherical=False, tol=(1e-12, 1e-10, 1e-10), max_iter=100, verbose=False,
               guess="core"):
        """DF-RHF (hfg_scf_df) with a DFTensor built on this context; guess
        "core" as run_factorized_rhf, or "sad"."""
        keep = []
        o = self._scf_opts(charge, 1, False, spherical, tol, max_iter, None, 0, verbose, keep)
        o.guess = 0 if guess == "sad" else 1
        n = self.n
        P, F, J, K = (np.zeros((n, n)) for _ in range(4))
        r = SCFResult()
        rc = self.lib.hfg_scf_df(self.h, df.h, mma, ctypes.byref(o), ctypes.byref(r), _dp(P), _dp(F), _dp(J), _dp(K))
        if rc not in (0, 3):
            self._check(rc)
        out = r.as_dict()
        out.update({"P": P, "F": F, "J": J, "K": K, "status": rc})
        return out

    def df_three_center(self, aux):
        """(P|mu nu) for every auxiliary function and AO pair mu >= nu
        (hfg_df_three_center): naux x n (n + 1) / 2, packed columns."""
        b = HfgBasis(aux.n, _dp(aux.center), _ip(aux.lxyz), _ip(aux.atom), _ip(aux.prim_off), _dp(aux.exps),
                     _dp(aux.coefs))
        np_ = self.n * (self.n + 1) // 2
        out = np.zeros((aux.n, np_))
        self._check(self.lib.hfg_df_three_center(self.h, ctypes.byref(b), _dp(out), out.size))
        return out

    def last_stats(self):
        s = JKStats()
        self._check(self.lib.hfg_jk_last_stats(self.h, ctypes.byref(s)))
        return s.as_dict()

    def autotune(self, d_total, d_spin, nspin=1, base=None, fp32=(), prim=(), max_energy_error=None, repeats=None,
                 tiles=None):
        """hfg_jk_autotune on device densities (integer pointers): returns the
        chosen JKOptions and a report of every candidate.  tiles: quartet
        tiles tried on the best threshold pair (None: the library's)."""
        o = AutotuneOptions()
        self.lib.hfg_autotune_opts_default(ctypes.byref(o))
        if tiles is not None:
            o.n_tile = len(tiles)
            for i, v in enumerate(tiles):
                o.tiles[i] = v
        if fp32:
            o.n_fp32 = len(fp32)
            for i, v in enumerate(fp32):
                o.fp32_thresholds[i] = v
        if prim:
            o.n_prim = len(prim)
            for i, v in enumerate(prim):
                o.prim_thresholds[i] = v
        if max_energy_error is not None:
            o.max_energy_error = max_energy_error
        if repeats is not None:
            o.repeats = repeats
        r = AutotuneResult()
        b = base or JKOptions.make()
        self._check(self.lib.hfg_jk_autotune(self.h, ctypes.byref(b), nspin, d_total, d_spin, ctypes.byref(o),
                                             ctypes.byref(r)))
        fl = [o.fp32_thresholds[i] for i in range(o.n_fp32)]
        pl = [o.prim_thresholds[i] for i in range(o.n_prim)]
        cands = [{"fp32_threshold": f, "prim_threshold": p, "ms": r.ms[k], "energy_error": r.energy_error[k]}
                 for k, (f, p) in enumerate((f, p) for f in fl for p in pl)]
        k0 = len(cands)
        for i in range(r.evaluated - k0):
            cands.append({"tile": o.tiles[i], "ms": r.ms[k0 + i], "energy_error": r.energy_error[k0 + i]})
        best = JKOptions()
        ctypes.memmove(ctypes.byref(best), ctypes.byref(r.best), ctypes.sizeof(JKOptions))
        return best, {"found": bool(r.found), "best_ms": r.best_ms, "best_energy_error": r.best_energy_error,
                      "fp64_ms": r.fp64_ms, "max_energy_error": o.max_energy_error, "candidates": cands,
                      "best": best.as_dict()}


HFG_DF_FP64, HFG_DF_FP32, HFG_DF_BF16 = 0, 1, 2


class DFTensor:
    """hfg_df: the DF factor B = X^T (P|mn) of an auxiliary basis on a context."""

    def __init__(self, ctx, aux, metric_cutoff=1e-10, pair_threshold=0.0, storage=HFG_DF_FP64, shard=0, nshards=1):
        """shard/nshards: hold only that share of the whitened auxiliary
        functions (hfg_df_build_shard), one rank's factor of a multi-GPU
        build; its J/K are the rank's partial sums."""
        self.ctx = ctx
        self.lib = ctx.lib
        self.aux = aux
        self._b = HfgBasis(aux.n, _dp(aux.center), _ip(aux.lxyz), _ip(aux.atom), _ip(aux.prim_off), _dp(aux.exps),
                           _dp(aux.coefs))
        h = VP()
        rc = self.lib.hfg_df_build_shard(ctx.h, ctypes.byref(self._b), metric_cutoff, pair_threshold, storage, shard,
                                         nshards, ctypes.byref(h))
        ctx._check(rc)
        self.h = h
        ctx._adopt(self)

    def sizes(self):
        a, r, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_longlong()
        self.ctx._check(self.lib.hfg_df_sizes(self.h, ctypes.byref(a), ctypes.byref(r), ctypes.byref(c)))
        return a.value, r.value, c.value

    def metric(self):
        naux = self.sizes()[0]
        M = np.zeros((naux, naux))
        self.ctx._check(self.lib.hfg_df_metric(self.h, _dp(M)))
        return M

    def jk(self, C_occ, mma=HFG_DF_FP64):
        n = self.ctx.n
        C = np.ascontiguousarray(C_occ, dtype=np.float64)
        J, K = np.zeros((n, n)), np.zeros((n, n))
        self.ctx._check(self.lib.hfg_df_jk(self.h, _dp(C), C.shape[1], _dp(J), _dp(K), mma))
        return J, K

    def transform(self, C):
        """The factor in the MO basis C (n x m): rank x m (m + 1) / 2 packed
        (hfg_df_transform, DfTensor::transform)."""
        C = np.ascontiguousarray(C, dtype=np.float64)
        m = C.shape[1]
        rank = self.sizes()[1]
        out = np.zeros((rank, m * (m + 1) // 2))
        self.ctx._check(self.lib.hfg_df_transform(self.h, _dp(C), m, _dp(out), out.size))
        return out

    def mp2_energy(self, C, eps, n_occ, n_frozen=0):
        """RI-MP2 correlation energy (hfg_df_mp2, DfTensor::mp2_energy)."""
        C = np.ascontiguousarray(C, dtype=np.float64)
        e = np.ascontiguousarray(eps, dtype=np.float64)
        out = ctypes.c_double()
        self.ctx._check(self.lib.hfg_df_mp2(self.h, _dp(C), _dp(e), C.shape[1], n_occ, n_frozen, ctypes.byref(out)))
        return out.value

    def jk_shard(self, C_occ, shard, nshards, mma=HFG_DF_FP64):
        """Partial J, K over the shard's auxiliary functions (hfg_df_jk_shard)."""
        n = self.ctx.n
        C = np.ascontiguousarray(C_occ, dtype=np.float64)
        J, K = np.zeros((n, n)), np.zeros((n, n))
        self.ctx._check(self.lib.hfg_df_jk_shard(self.h, _dp(C), C.shape[1], _dp(J), _dp(K), mma, shard, nshards))
        return J, K

    def jk_device_shard(self, d_C, nocc, d_J, d_K, shard, nshards, mma=HFG_DF_FP64):
        """Device form (integer pointers; C column-major n x nocc)."""
        self.ctx._check(self.lib.hfg_df_jk_device_shard(self.h, d_C, nocc, d_J, d_K, mma, shard, nshards))

    def last_stats(self):
        """Device time (ms), executed tensor-core flops and non-zero tile share
        of the last tensor-core exchange (hfg_df_last_stats)."""
        ms, fl, tf = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        self.ctx._check(self.lib.hfg_df_last_stats(self.h, ctypes.byref(ms), ctypes.byref(fl), ctypes.byref(tf)))
        return {"k_ms": ms.value, "k_flops": fl.value, "tiles_fraction": tf.value}

    @classmethod
    def cholesky(cls, ctx, threshold, budget=512 * 1024 * 1024):
        """Pivoted Cholesky vectors of the AO ERIs as a factor
        (hfg_cholesky_eri, pivoted_cholesky_eri); returns (factor, pivots,
        largest residual diagonal)."""
        self = cls.__new__(cls)
        self.ctx, self.lib, self.aux = ctx, ctx.lib, None
        h = VP()
        npair = ctx.n * (ctx.n + 1) // 2
        piv = (ctypes.c_longlong * npair)()
        cnt, mres = ctypes.c_int(), ctypes.c_double()
        ctx._check(self.lib.hfg_cholesky_eri(ctx.h, threshold, budget, ctypes.byref(h), ctypes.byref(mres), piv, npair,
                                             ctypes.byref(cnt)))
        self.h = h
        ctx._adopt(self)
        return self, [int(piv[k]) for k in range(cnt.value)], mres.value

    def close(self):
        # a context that is already gone took its DF tensors with it
        if getattr(self, "h", None) is not None and self.h.value and self.ctx.h.value:
            self.lib.hfg_df_destroy(self.h)
        self.h = VP()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """hfg_server: continuous admission of SCF jobs onto worker slots."""

    def __init__(self, device=0, slots=8, hbm_budget_bytes=64 << 30, mixed_min_ao=None, batch_max_ao=None,
                 batch_window_us=300.0):
        """batch_max_ao: RHF jobs below this many functions batch their Fock
        builds across jobs (0 turns batching off; None keeps the default)."""
        self.lib = load_library()
        h = VP()
        rc = self.lib.hfg_server_create(device, slots, hbm_budget_bytes, ctypes.byref(h))
        if rc != 0:
            raise HfgError(rc, "hfg_server_create failed")
        self.h = h
        if mixed_min_ao is not None:
            self.lib.hfg_server_set_mixed_min_ao(h, mixed_min_ao)
        if batch_max_ao is not None:
            rc = self.lib.hfg_server_set_batching(h, batch_max_ao, batch_window_us)
            if rc != 0:
                raise HfgError(rc, "hfg_server_set_batching failed")

    def batch_stats(self):
        """Fock builds that went through cross-job batches, and batch count."""
        b, n = ctypes.c_longlong(), ctypes.c_longlong()
        self.lib.hfg_server_batch_stats(self.h, ctypes.byref(b), ctypes.byref(n))
        return {"batched_builds": b.value, "batches": n.value}

    def submit(self, basis, charge=0, multiplicity=1, uhf=False, spherical=False, tol=1e-10, max_iter=100,
               jk=None, tag=0):
        pos = np.ascontiguousarray(basis.positions())
        chg = np.ascontiguousarray(basis.nuclear_charges())
        j = Job()
        j.basis = HfgBasis(basis.n, _dp(basis.center), _ip(basis.lxyz), _ip(basis.atom), _ip(basis.prim_off),
                           _dp(basis.exps), _dp(basis.coefs))
        j.natom = len(chg)
        j.positions, j.charges = _dp(pos), _dp(chg)
        j.charge, j.multiplicity, j.uhf, j.spherical = charge, multiplicity, int(uhf), int(spherical)
        j.max_iter = max_iter
        j.energy_tol, j.residual_tol, j.density_tol = convergence_from_tol(tol)
        j.jk = jk or JKOptions.make()
        j.tag = tag
        rc = self.lib.hfg_server_submit(self.h, ctypes.byref(j))  # inputs copied before return
        if rc != 0:
            raise HfgError(rc, "hfg_server_submit failed")

    def poll(self, wait=False, max_results=256):
        buf = (JobResult * max_results)()
        n = ctypes.c_int()
        rc = self.lib.hfg_server_poll(self.h, buf, max_results, ctypes.byref(n), int(wait))
        if rc != 0:
            raise HfgError(rc, "hfg_server_poll failed")
        return [buf[i].as_dict() for i in range(n.value)]

    def stats(self):
        p, r, b = ctypes.c_int(), ctypes.c_int(), ctypes.c_longlong()
        self.lib.hfg_server_stats(self.h, ctypes.byref(p), ctypes.byref(r), ctypes.byref(b))
        return {"pending": p.value, "running": r.value, "in_use_bytes": b.value}

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            self.lib.hfg_server_destroy(self.h)
            self.h = VP()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
