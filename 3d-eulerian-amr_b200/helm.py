"""Python mirror of the reference Helmholtz EOS calls (helmholtz/helmholtz.h).

ctypes binding of the batched C ABI in include/helm_b200.h.  Every call runs
the CUDA kernels of lib/libamr_b200.so; there is no CPU path.

    h = Helm(table_path)            # read_helm_table (helmeos.cpp:73-130)
    h.set_cgs_units(cm, g, s, K)    # helmholtz_set_cgs_units
    h.eos(rho, T, abar, zbar)       # helmholtz_eos, arrays
    h.invert_T(rho, e, abar, zbar, T_guess)   # helmholtz_compute_T, arrays
    h.ztwd(zbar, rho)               # helmholtz_ztwd, arrays
"""

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libamr_b200.so")

STATUS = {0: "ok", 1: "outside the table", 2: "cv < 0", 3: "cs^2 < 0", 4: "Newton did not converge",
          5: "temperature below the table floor"}

_lib = None


def load_library(path=LIB_PATH):
    global _lib
    if _lib is None:
        if not os.path.exists(path):
            raise ImportError("libamr_b200.so not built (run 3d-eulerian-amr_b200/build.py): %s" % path)
        lib = ctypes.CDLL(path)
        P, L, I, D = ctypes.c_void_p, ctypes.c_longlong, ctypes.c_int, ctypes.c_double
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int)
        lib.helm_create.argtypes = [ctypes.c_char_p, ctypes.POINTER(P)]
        lib.helm_destroy.argtypes = [P]
        lib.helm_last_error.argtypes = [P]
        lib.helm_last_error.restype = ctypes.c_char_p
        lib.helm_set_cgs_units.argtypes = [P, D, D, D, D]
        lib.helm_eos_batch.argtypes = [P, L] + [dp] * 4 + [dp] * 6 + [ip]
        lib.helm_eos_device.argtypes = [P, L] + [P] * 4 + [P] * 6 + [P, P]
        lib.helm_invert_T_batch.argtypes = [P, L] + [dp] * 4 + [I] + [dp] * 6 + [ip, ip]
        lib.helm_invert_T_device.argtypes = [P, L] + [P] * 4 + [I] + [P] * 6 + [P, P, P]
        lib.helm_ztwd_batch.argtypes = [P, L, dp, dp, dp, dp]
        _lib = lib
    return _lib


def _d(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) if a is not None else None


def _i(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int)) if a is not None else None


def _arr(x, n):
    return np.ascontiguousarray(np.broadcast_to(np.asarray(x, np.float64), (n,)))


class HelmError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("helm error %d: %s" % (code, msg))
        self.code = code


class Helm:
    def __init__(self, table_path, lib_path=LIB_PATH):
        self.lib = load_library(lib_path)
        self.ctx = ctypes.c_void_p()
        rc = self.lib.helm_create(os.fsencode(table_path), ctypes.byref(self.ctx))
        if rc != 0:
            raise HelmError(rc, "cannot create the Helmholtz context from %s" % table_path)

    def close(self):
        if self.ctx:
            self.lib.helm_destroy(self.ctx)
            self.ctx = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc, raise_on_error):
        if rc != 0 and raise_on_error:
            raise HelmError(rc, self.lib.helm_last_error(self.ctx).decode(errors="replace"))
        return rc

    def set_cgs_units(self, cm, g, s, K):
        self._check(self.lib.helm_set_cgs_units(self.ctx, cm, g, s, K), True)

    def eos(self, rho, T, abar, zbar, raise_on_error=False):
        rho = np.ascontiguousarray(rho, np.float64).reshape(-1)
        n = rho.size
        T, abar, zbar = _arr(T, n), _arr(abar, n), _arr(zbar, n)
        out = {k: np.zeros(n) for k in ("p", "e", "cs", "cv", "s", "dsdt")}
        out["status"] = np.zeros(n, np.int32)
        rc = self.lib.helm_eos_batch(self.ctx, n, _d(rho), _d(T), _d(abar), _d(zbar), _d(out["p"]), _d(out["e"]),
                                     _d(out["cs"]), _d(out["cv"]), _d(out["s"]), _d(out["dsdt"]),
                                     _i(out["status"]))
        self._check(rc, raise_on_error)
        out["rc"] = rc
        return out

    def invert_T(self, rho, target, abar, zbar, T_guess, from_entropy=False, raise_on_error=False):
        rho = np.ascontiguousarray(rho, np.float64).reshape(-1)
        n = rho.size
        target, abar, zbar = _arr(target, n), _arr(abar, n), _arr(zbar, n)
        T = _arr(T_guess, n).copy()
        out = {k: np.zeros(n) for k in ("p", "e", "cs", "cv", "s")}
        out["iters"] = np.zeros(n, np.int32)
        out["status"] = np.zeros(n, np.int32)
        rc = self.lib.helm_invert_T_batch(self.ctx, n, _d(rho), _d(target), _d(abar), _d(zbar),
                                          1 if from_entropy else 0, _d(T), _d(out["p"]), _d(out["e"]),
                                          _d(out["cs"]), _d(out["cv"]), _d(out["s"]), _i(out["iters"]),
                                          _i(out["status"]))
        self._check(rc, raise_on_error)
        out["T"] = T
        out["rc"] = rc
        return out

    def ztwd(self, zbar, rho):
        rho = np.ascontiguousarray(rho, np.float64).reshape(-1)
        n = rho.size
        zbar = _arr(zbar, n)
        p, e = np.zeros(n), np.zeros(n)
        self._check(self.lib.helm_ztwd_batch(self.ctx, n, _d(zbar), _d(rho), _d(p), _d(e)), True)
        return p, e

    # device arrays (torch CUDA tensors, float64 / int32), asynchronous on `stream`
    def eos_device(self, rho, T, abar, zbar, p, e, cs, status, cv=None, s=None, dsdt=None, stream=None):
        ptr = lambda t: ctypes.c_void_p(t.data_ptr()) if t is not None else None
        rc = self.lib.helm_eos_device(self.ctx, rho.numel(), ptr(rho), ptr(T), ptr(abar), ptr(zbar), ptr(p), ptr(e),
                                      ptr(cs), ptr(cv), ptr(s), ptr(dsdt), ptr(status),
                                      ctypes.c_void_p(stream or 0))
        self._check(rc, True)

    def invert_T_device(self, rho, target, abar, zbar, T, status, iters=None, p=None, e=None, cs=None, cv=None,
                        s=None, from_entropy=False, stream=None):
        ptr = lambda t: ctypes.c_void_p(t.data_ptr()) if t is not None else None
        rc = self.lib.helm_invert_T_device(self.ctx, rho.numel(), ptr(rho), ptr(target), ptr(abar), ptr(zbar),
                                           1 if from_entropy else 0, ptr(T), ptr(p), ptr(e), ptr(cs), ptr(cv),
                                           ptr(s), ptr(iters), ptr(status), ctypes.c_void_p(stream or 0))
        self._check(rc, True)
