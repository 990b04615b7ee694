"""ctypes binding of liblsmoke_oracle.so -- test infrastructure only.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
module, as the checker; the product path never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liblsmoke_oracle.so")
NCOUNT = 8
COUNTER_NAMES = ("steps", "rhs", "jacobians", "factorizations", "solves",
                 "error_failures", "convergence_failures", "jacobian_rhs")


class OrcOptions(C.Structure):
    _fields_ = [("rtol", C.c_double), ("atol", C.c_double), ("tmin_chem", C.c_double),
                ("y_min_T", C.c_double), ("y_max_T", C.c_double),
                ("max_steps", C.c_int), ("full_pivoting", C.c_int), ("energy", C.c_int),
                ("alfa2_4", C.c_double), ("alfa2_5", C.c_double),
                ("maximum_order", C.c_int), ("sequential_state", C.c_int)]


def build() -> str:
    subprocess.check_call(["make", "-s", "-C", HERE])
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = C.CDLL(LIB)
        L.orc_mech_load.restype = C.c_void_p
        L.orc_mech_load.argtypes = [C.c_void_p, C.c_size_t]
        L.orc_mech_free.argtypes = [C.c_void_p]
        L.orc_rhs.argtypes = [C.c_void_p, C.c_double, C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_fd_jacobian.argtypes = [C.c_void_p, C.c_double, C.c_void_p, C.c_double, C.c_double,
                                      C.c_double, C.c_double, C.c_void_p]
        L.orc_reaction_step.argtypes = [C.c_void_p, C.POINTER(OrcOptions), C.c_int, C.c_void_p, C.c_void_p,
                                        C.c_double, C.c_double, C.c_void_p, C.c_double, C.c_void_p,
                                        C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]
        L.orc_reaction_step.restype = C.c_int
        L.orc_compact_sources.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                          C.c_double, C.c_void_p, C.c_double, C.c_int, C.c_void_p, C.c_void_p]
        L.orc_formation_rates.argtypes = [C.c_void_p, C.c_double, C.c_void_p, C.c_void_p]
        L.orc_steady_sources.argtypes = [C.c_void_p, C.c_double, C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_steady_sources_sparse.argtypes = [C.c_void_p, C.c_double, C.c_void_p, C.c_void_p, C.c_void_p,
                                                C.c_int, C.c_int]
        L.orc_reaction_step_drg.argtypes = [C.c_void_p, C.POINTER(OrcOptions), C.POINTER(OrcDrgOptions), C.c_int,
                                            C.c_void_p, C.c_void_p, C.c_double, C.c_double, C.c_void_p, C.c_double,
                                            C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_drg_analysis.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_void_p, C.c_double, C.c_void_p,
                                       C.c_int, C.c_void_p, C.POINTER(C.c_int), C.c_void_p, C.POINTER(C.c_int)]
        _lib = L
    return _lib


class OrcDrgOptions(C.Structure):
    _fields_ = [("key", C.c_void_p), ("nkey", C.c_int), ("band_T", C.c_void_p), ("band_eps", C.c_void_p),
                ("nbands", C.c_int), ("epsilon0", C.c_double), ("min_T", C.c_double),
                ("first_cell_options_only", C.c_int)]


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


class OracleMechanism:
    def __init__(self, blob: bytes):
        self._buf = (C.c_ubyte * len(blob)).from_buffer_copy(blob)
        self.h = lib().orc_mech_load(C.cast(self._buf, C.c_void_p), len(blob))
        if not self.h:
            raise ValueError("oracle: bad mechanism blob")
        from laminarsmoke_b200.mech import blob as _blob
        dims = _blob.unpack(blob)[0]["dims"]
        self.n_species, self.n_reactions = int(dims[0]), int(dims[1])

    def __del__(self):
        try:
            if self.h:
                lib().orc_mech_free(self.h)
        except Exception:
            pass

    def rhs(self, y: np.ndarray, p: float = 101325.0):
        y = np.ascontiguousarray(y, dtype=np.float64)
        dy = np.zeros_like(y)
        q = np.zeros(1)
        lib().orc_rhs(self.h, p, _ptr(y), _ptr(dy), _ptr(q))
        return dy, float(q[0])

    def compact_sources(self, Y0, T0, Yf, Tf, dt, p=101325.0, energy=True):
        """Cell-major Y0/Yf [ncells, NC]; returns (RR [ncells, NC], RT [ncells])."""
        Y0 = np.ascontiguousarray(Y0, dtype=np.float64)
        Yf = np.ascontiguousarray(Yf, dtype=np.float64)
        T0 = np.ascontiguousarray(T0, dtype=np.float64)
        Tf = np.ascontiguousarray(Tf, dtype=np.float64)
        n = T0.size
        dt_arr = None if np.ndim(dt) == 0 else np.ascontiguousarray(dt, dtype=np.float64)
        RR = np.zeros_like(Y0)
        RT = np.zeros(n)
        lib().orc_compact_sources(self.h, n, _ptr(Y0), _ptr(T0), _ptr(Yf), _ptr(Tf), p, _ptr(dt_arr),
                                  0.0 if dt_arr is not None else float(dt), int(energy), _ptr(RR), _ptr(RT))
        return RR, RT

    def formation_rates(self, y, p=101325.0):
        """R_i MW_i [kg/m3/s] at y = [Y_1..Y_NC, T]."""
        y = np.ascontiguousarray(y, dtype=np.float64)
        out = np.zeros(y.size - 1)
        lib().orc_formation_rates(self.h, p, _ptr(y), _ptr(out))
        return out

    def steady_sources(self, y, p=101325.0):
        """(S_implicit, S_explicit) [NC + 1] of the steady solvers at y = [Y_1..Y_NC, T]."""
        y = np.ascontiguousarray(y, dtype=np.float64)
        si = np.zeros(y.size)
        se = np.zeros(y.size)
        lib().orc_steady_sources(self.h, p, _ptr(y), _ptr(si), _ptr(se))
        return si, se

    def steady_sources_sparse(self, y, p=101325.0, species=True, energy=True):
        """(S_implicit, S_explicit) [NC + 1] with the steady solvers' default analytic species diagonal
        (sparseJacobian true)."""
        y = np.ascontiguousarray(y, dtype=np.float64)
        si = np.zeros(y.size)
        se = np.zeros(y.size)
        lib().orc_steady_sources_sparse(self.h, p, _ptr(y), _ptr(si), _ptr(se), int(species), int(energy))
        return si, se

    def fd_jacobian(self, y, h, rtol=1e-7, atol=1e-12, p=101325.0, y_max_T=6000.0):
        y = np.ascontiguousarray(y, dtype=np.float64)
        n = y.size
        J = np.zeros(n * n)
        lib().orc_fd_jacobian(self.h, p, _ptr(y), h, rtol, atol, y_max_T, _ptr(J))
        return J.reshape(n, n).T.copy()  # stored column-major

    def reaction_step(self, Y, T, dt, p=101325.0, t0=0.0, rtol=1e-7, atol=1e-12, tmin_chem=0.0,
                      max_steps=500000, energy=True, alfa2_4=0.8, alfa2_5=0.8, maximum_order=5,
                      sequential_state=False, nthreads=0, y_min_T=200.0, y_max_T=6000.0, rho=None):
        """Cell-major Y[ncells, NC], T[ncells]; returns (Y, T, Q, status, counters).  rho [ncells]:
        constant-volume reactor of those densities (p is then unused)."""
        Y = np.array(Y, dtype=np.float64, order="C", copy=True)
        T = np.array(T, dtype=np.float64, copy=True)
        n = T.size
        dt_arr = None
        dt_s = 0.0
        if np.ndim(dt) == 0:
            dt_s = float(dt)
        else:
            dt_arr = np.ascontiguousarray(dt, dtype=np.float64)
        Q = np.zeros(n)
        st = np.zeros(n, dtype=np.int32)
        cnt = np.zeros((n, NCOUNT), dtype=np.int64)
        o = OrcOptions(rtol, atol, tmin_chem, y_min_T, y_max_T, max_steps, 0, int(energy),
                       alfa2_4, alfa2_5, maximum_order, int(sequential_state))
        lib().orc_reaction_step(self.h, C.byref(o), n, _ptr(Y), _ptr(T), p, t0, _ptr(dt_arr), dt_s,
                                _ptr(Q), _ptr(st), _ptr(cnt), nthreads,
                                _ptr(None if rho is None else np.ascontiguousarray(rho, dtype=np.float64)))
        return Y, T, Q, st, cnt

    def drg_analysis(self, T, P, c, eps, key):
        """DRG analysis at one state (concentrations c [NC]): (important species, dropped reactions)."""
        c = np.ascontiguousarray(c, dtype=np.float64)
        k = np.ascontiguousarray(key, dtype=np.int32)
        nc = c.size
        imp = np.zeros(nc, np.int32)
        drop = np.zeros(max(self.n_reactions, 1), np.int32)
        ni, nd = C.c_int(), C.c_int()
        lib().orc_drg_analysis(self.h, T, P, _ptr(c), eps, _ptr(k), k.size, _ptr(imp), C.byref(ni), _ptr(drop),
                               C.byref(nd))
        return imp[:ni.value].tolist(), drop[:nd.value].tolist()

    def reaction_step_drg(self, Y, T, dt, key, bands=((1.e6, 1.e-2),), epsilon0=1.e-2, min_T=300.0,
                          first_cell_options_only=True, p=101325.0, t0=0.0, rtol=1e-7, atol=1e-12, energy=True):
        """DRG-reduced step of cell-major Y[ncells, NC], T[ncells] (chemistry_DRG.H): key species
        indices, (temperature, epsilon) bands.  Returns (Y, T, Q, status, counters, n_species,
        n_reactions)."""
        Y = np.array(Y, dtype=np.float64, order="C", copy=True)
        T = np.array(T, dtype=np.float64, copy=True)
        n = T.size
        dt_arr, dt_s = (None, float(dt)) if np.ndim(dt) == 0 else (np.ascontiguousarray(dt, dtype=np.float64), 0.)
        Q = np.zeros(n)
        st = np.zeros(n, dtype=np.int32)
        cnt = np.zeros((n, NCOUNT), dtype=np.int64)
        nsp = np.zeros(n, dtype=np.int32)
        nrx = np.zeros(n, dtype=np.int32)
        k = np.ascontiguousarray(key, dtype=np.int32)
        bt = np.ascontiguousarray([b[0] for b in bands], dtype=np.float64)
        be = np.ascontiguousarray([b[1] for b in bands], dtype=np.float64)
        o = OrcOptions(rtol, atol, 0.0, 200.0, 6000.0, 500000, 0, int(energy), 0.8, 0.8, 5, 1)
        d = OrcDrgOptions(_ptr(k), k.size, _ptr(bt), _ptr(be), bt.size, epsilon0, min_T, int(first_cell_options_only))
        lib().orc_reaction_step_drg(self.h, C.byref(o), C.byref(d), n, _ptr(Y), _ptr(T), p, t0, _ptr(dt_arr), dt_s,
                                    _ptr(Q), _ptr(st), _ptr(cnt), _ptr(nsp), _ptr(nrx))
        return Y, T, Q, st, cnt, nsp, nrx


# ----------------------------------------------------------------------------
# The reference's own integrator (oracle/refpin): the class templates of
# math/native-ode-solvers/{MultiValueSolver,MethodGear,KernelDense}.hpp compiled
# unchanged from the reference checkout, driving the oracle's right-hand side.
# Built into oracle/_ref/ by oracle/refpin/Makefile where the reference sources
# are present; used by tests/test_refpin.py to pin the oracle's integrator.
REFPIN = os.path.join(HERE, "_ref", "liblsmoke_refpin.so")
_refpin = None


def refpin_available() -> bool:
    return os.path.exists(REFPIN)


def refpin_lib():
    global _refpin
    if _refpin is None:
        L = C.CDLL(REFPIN)
        L.orc_mech_load.restype = C.c_void_p
        L.orc_mech_load.argtypes = [C.c_void_p, C.c_size_t]
        L.orc_mech_free.argtypes = [C.c_void_p]
        L.ref_reaction_step.argtypes = [C.c_void_p, C.POINTER(OrcOptions), C.c_int, C.c_void_p, C.c_void_p,
                                        C.c_double, C.c_double, C.c_void_p, C.c_double, C.c_void_p,
                                        C.c_void_p, C.c_void_p, C.c_int]
        L.ref_reaction_step.restype = C.c_int
        _refpin = L
    return _refpin


class ReferenceIntegrator:
    """The reference's MultiValueSolver<MethodGear<KernelDense<...>>> on the oracle's RHS, with the
    per-cell calls of chemistry_DI.H:92-169 (a fresh solver object per cell)."""

    def __init__(self, blob: bytes):
        self._buf = (C.c_ubyte * len(blob)).from_buffer_copy(blob)
        self.h = refpin_lib().orc_mech_load(C.cast(self._buf, C.c_void_p), len(blob))
        if not self.h:
            raise ValueError("refpin: bad mechanism blob")

    def __del__(self):
        try:
            if self.h:
                refpin_lib().orc_mech_free(self.h)
        except Exception:
            pass

    def reaction_step(self, Y, T, dt, p=101325.0, t0=0.0, rtol=1e-7, atol=1e-12, tmin_chem=0.0,
                      max_steps=500000, energy=True, nthreads=0, y_min_T=200.0, y_max_T=6000.0):
        """Cell-major Y[ncells, NC], T[ncells]; returns (Y, T, Q, status, counters) as
        OracleMechanism.reaction_step does."""
        Y = np.array(Y, dtype=np.float64, order="C", copy=True)
        T = np.array(T, dtype=np.float64, copy=True)
        n = T.size
        dt_arr = None
        dt_s = 0.0
        if np.ndim(dt) == 0:
            dt_s = float(dt)
        else:
            dt_arr = np.ascontiguousarray(dt, dtype=np.float64)
        Q = np.zeros(n)
        st = np.zeros(n, dtype=np.int32)
        cnt = np.zeros((n, NCOUNT), dtype=np.int64)
        o = OrcOptions(rtol, atol, tmin_chem, y_min_T, y_max_T, max_steps, 0, int(energy), 0.8, 0.8, 5, 0)
        refpin_lib().ref_reaction_step(self.h, C.byref(o), n, _ptr(Y), _ptr(T), p, t0, _ptr(dt_arr), dt_s,
                                       _ptr(Q), _ptr(st), _ptr(cnt), nthreads)
        return Y, T, Q, st, cnt
