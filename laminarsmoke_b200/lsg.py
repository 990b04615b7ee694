"""Python binding of the C ABI (include/lsmoke_gpu.h) over ctypes.

This is the harness the tests and the benchmark drive the library through; it
adds no computation of its own.  The shared library must have been built
(``python -m laminarsmoke_b200.csrc.build`` or ``__graft_entry__.build()``);
importing this module without it raises, there is no fallback path.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liblsmoke_gpu.so")

LSG_PRECISION_FP64 = 0
LSG_PRECISION_MIXED = 1
LSG_JACOBIAN_FD, LSG_JACOBIAN_ANALYTIC = 0, 1
LSG_TILE_AUTO, LSG_TILE_WARP, LSG_TILE_LANE, LSG_TILE_PERSISTENT, LSG_TILE_BLOCK, LSG_TILE_GROUP = 0, 1, 2, 3, 4, 5
LSG_ERR_SCRATCH = -8
NOALLOC_SCRATCH_BYTES = 16 << 20
NCOUNTERS = 8
COUNTER_NAMES = ("steps", "rhs", "jacobians", "factorizations", "solves",
                 "error_failures", "convergence_failures", "jacobian_rhs")


class LsgError(RuntimeError):
    def __init__(self, msg: str, code: int = 0):
        super().__init__(msg)
        self.code = code


class Options(C.Structure):
    _fields_ = [("rtol", C.c_double), ("atol", C.c_double), ("tmin_chem", C.c_double),
                ("y_min_T", C.c_double), ("y_max_T", C.c_double),
                ("max_steps", C.c_int), ("full_pivoting", C.c_int), ("energy", C.c_int),
                ("precision", C.c_int),
                ("alfa2_4", C.c_double), ("alfa2_5", C.c_double), ("maximum_order", C.c_int),
                ("tile", C.c_int), ("kernel_timing", C.c_int), ("autotune", C.c_int), ("jacobian", C.c_int),
                ("reserved", C.c_int * 3)]


EXPORTS = (
    "lsg_options_default", "lsg_mech_load_blob", "lsg_mech_load_file", "lsg_mech_info",
    "lsg_mech_destroy", "lsg_ctx_create", "lsg_ctx_set_options", "lsg_ctx_destroy",
    "lsg_reaction_step", "lsg_reaction_step_device", "lsg_ctx_check", "lsg_rhs_device",
    "lsg_strerror", "lsg_abi_version", "lsg_ctx_stream", "lsg_ctx_launches",
    "lsg_reaction_step_device_noalloc", "lsg_ctx_kernel_times", "lsg_ctx_tuning",
    "lsg_compact_sources_device", "lsg_formation_rates_device",
    "lsg_reaction_step_cv", "lsg_reaction_step_cv_device", "lsg_steady_sources_device",
    "lsg_mech_transport_info", "lsg_properties_device", "lsg_properties", "lsg_build_and_invert_g_device",
    "lsg_reaction_step_sequence_device", "lsg_jacobian_device", "lsg_steady_sources_sparse_device",
    "lsg_reaction_step_drg_device", "lsg_reaction_step_drg",
)

class DrgOptions(C.Structure):
    """lsg_drg_options."""
    _fields_ = [("key", C.c_void_p), ("nkey", C.c_int), ("band_T", C.c_void_p), ("band_eps", C.c_void_p),
                ("nbands", C.c_int), ("epsilon0", C.c_double), ("min_T", C.c_double),
                ("first_cell_options_only", C.c_int)]


# lsg_property_fields, in declaration order: species rows (nc), scalars, light-species rows
PROPERTY_FIELDS = ("X", "cTot", "psi", "mu", "lambda", "cp", "cv", "h", "MWmix", "cp_species", "Dmix", "Dsoret")


class PropertyFields(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in PROPERTY_FIELDS]


class PropertyOptions(C.Structure):
    _fields_ = [("energy", C.c_int), ("simplified_transport", C.c_int), ("lewis", C.c_void_p)]

_lib = None


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise LsgError(f"{LIB_PATH} is not built; run __graft_entry__.build()")
    L = C.CDLL(LIB_PATH)
    vp, i, d, l = C.c_void_p, C.c_int, C.c_double, C.c_long
    L.lsg_options_default.argtypes = [C.POINTER(Options)]
    L.lsg_options_default.restype = None
    L.lsg_mech_load_blob.argtypes = [vp, C.c_size_t, i, C.POINTER(vp)]
    L.lsg_mech_load_file.argtypes = [C.c_char_p, i, C.POINTER(vp)]
    L.lsg_mech_info.argtypes = [vp, C.POINTER(i), C.POINTER(i)]
    L.lsg_mech_destroy.argtypes = [vp]
    L.lsg_ctx_create.argtypes = [vp, C.POINTER(Options), i, C.POINTER(vp)]
    L.lsg_ctx_set_options.argtypes = [vp, C.POINTER(Options)]
    L.lsg_ctx_destroy.argtypes = [vp]
    L.lsg_reaction_step.argtypes = [vp, i, i, C.POINTER(vp), vp, d, d, vp, d, vp, vp, vp]
    L.lsg_reaction_step_device.argtypes = [vp, i, i, vp, l, vp, d, d, vp, d, vp, vp, vp, vp, vp]
    L.lsg_ctx_check.argtypes = [vp, C.POINTER(i)]
    L.lsg_rhs_device.argtypes = [vp, i, vp, vp, l, d, vp, vp]
    L.lsg_build_and_invert_g_device.argtypes = [vp, i, i, vp, vp, vp, vp]
    L.lsg_reaction_step_sequence_device.argtypes = [vp, i, i, i, vp, l, vp, d, d, d, vp, vp, C.POINTER(i), vp]
    L.lsg_jacobian_device.argtypes = [vp, i, vp, l, d, vp, vp]
    L.lsg_steady_sources_sparse_device.argtypes = [vp, i, i, vp, vp, l, vp, d, i, i, vp, vp, l, vp]
    L.lsg_reaction_step_drg_device.argtypes = [vp, i, i, vp, l, vp, d, d, vp, d, C.POINTER(DrgOptions), vp, vp, vp,
                                               vp, vp, vp]
    L.lsg_reaction_step_drg.argtypes = [vp, i, i, C.POINTER(vp), vp, d, d, vp, d, C.POINTER(DrgOptions), vp, vp, vp,
                                        vp]
    L.lsg_strerror.argtypes = [i]
    L.lsg_strerror.restype = C.c_char_p
    L.lsg_abi_version.restype = i
    L.lsg_ctx_stream.argtypes = [vp]
    L.lsg_ctx_stream.restype = vp
    L.lsg_reaction_step_device_noalloc.argtypes = [vp, C.POINTER(Options), i, i, vp, l, vp, d, d, vp, d, vp,
                                                   vp, vp, vp, vp]
    L.lsg_ctx_kernel_times.argtypes = [vp, vp, vp, i, i]
    L.lsg_ctx_tuning.argtypes = [vp, C.POINTER(i), C.POINTER(i), vp]
    L.lsg_ctx_launches.argtypes = [vp]
    L.lsg_ctx_launches.restype = C.c_longlong
    L.lsg_reaction_step_cv.argtypes = [vp, i, i, C.POINTER(vp), vp, vp, d, vp, d, vp, vp, vp]
    L.lsg_reaction_step_cv_device.argtypes = [vp, i, i, vp, l, vp, vp, d, vp, d, vp, vp, vp, vp, vp]
    L.lsg_steady_sources_device.argtypes = [vp, i, i, vp, vp, l, vp, d, vp, vp, l, vp]
    L.lsg_compact_sources_device.argtypes = [vp, i, i, vp, vp, vp, vp, l, d, vp, d, vp, vp, vp]
    L.lsg_formation_rates_device.argtypes = [vp, i, i, vp, vp, l, d, vp, l, vp]
    L.lsg_mech_transport_info.argtypes = [vp, C.POINTER(i), C.POINTER(i), vp]
    L.lsg_properties_device.argtypes = [vp, i, i, vp, vp, l, vp, d, C.POINTER(PropertyOptions),
                                        C.POINTER(PropertyFields), l, vp]
    L.lsg_properties.argtypes = [vp, i, i, vp, vp, vp, d, C.POINTER(PropertyOptions), C.POINTER(PropertyFields)]
    _lib = L
    return L


def _check(rc: int, what: str):
    if rc != 0:
        raise LsgError(f"{what}: {lib().lsg_strerror(rc).decode()} ({rc})", rc)


def default_options(**kw) -> Options:
    o = Options()
    lib().lsg_options_default(C.byref(o))
    for k, v in kw.items():
        if not hasattr(o, k):
            raise KeyError(k)
        setattr(o, k, v)
    return o


class Mechanism:
    """Device-resident mechanism tables (lsg_mech)."""

    def __init__(self, blob: bytes, device: int = 0):
        self.device = device
        self.h = C.c_void_p()
        buf = (C.c_ubyte * len(blob)).from_buffer_copy(blob)
        _check(lib().lsg_mech_load_blob(C.cast(buf, C.c_void_p), len(blob), device, C.byref(self.h)),
               "lsg_mech_load_blob")
        ns, nr = C.c_int(), C.c_int()
        _check(lib().lsg_mech_info(self.h, C.byref(ns), C.byref(nr)), "lsg_mech_info")
        self.n_species, self.n_reactions = ns.value, nr.value

    def transport_info(self):
        """(has transport data, species indices of the light species with Soret terms)."""
        has, nt = C.c_int(), C.c_int()
        idx = (C.c_int * max(self.n_species, 1))()
        _check(lib().lsg_mech_transport_info(self.h, C.byref(has), C.byref(nt), C.cast(idx, C.c_void_p)),
               "lsg_mech_transport_info")
        return bool(has.value), [idx[k] for k in range(nt.value)]

    def close(self):
        if self.h:
            lib().lsg_mech_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _require_layout(*tensors):
    for t in tensors:
        if t is None:
            continue
        if not t.is_cuda or not t.is_contiguous():
            raise TypeError("device arrays must be contiguous CUDA tensors (species-major [rows, ld])")


def _stream_handle(stream):
    """The caller's stream for device calls: torch's current stream unless one is given."""
    import torch
    if stream is None:
        stream = torch.cuda.current_stream()
    return stream.cuda_stream


class ReactionStep:
    """A context (lsg_ctx): options + stream + staging buffers."""

    def __init__(self, mech: Mechanism, options: Optional[Options] = None, **kw):
        self.mech = mech
        self.options = options if options is not None else default_options(**kw)
        self.h = C.c_void_p()
        _check(lib().lsg_ctx_create(mech.h, C.byref(self.options), mech.device, C.byref(self.h)),
               "lsg_ctx_create")

    def set_options(self, **kw):
        for k, v in kw.items():
            setattr(self.options, k, v)
        _check(lib().lsg_ctx_set_options(self.h, C.byref(self.options)), "lsg_ctx_set_options")

    def close(self):
        if self.h:
            lib().lsg_ctx_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- host arrays (the OpenFOAM-facing call) ----
    def step(self, Y_species: np.ndarray, T: np.ndarray, dt, p: float = 101325.0, t0: float = 0.0,
             want_q: bool = True):
        """Y_species: [NC, ncells] float64 (updated in place), T: [ncells] (in place)."""
        Y = Y_species
        if Y.dtype != np.float64 or not Y.flags.c_contiguous or T.dtype != np.float64:
            raise TypeError("Y_species and T must be C-contiguous float64")
        nc, n = Y.shape
        ptrs = (C.c_void_p * nc)(*[Y[i].ctypes.data for i in range(nc)])
        dt_arr = None
        dt_s = 0.0
        if np.ndim(dt) == 0:
            dt_s = float(dt)
        else:
            dt_arr = np.ascontiguousarray(dt, dtype=np.float64)
        Q = np.zeros(n) if want_q else None
        st = np.zeros(n, dtype=np.int32)
        ns = np.zeros(n, dtype=np.int32)
        _check(lib().lsg_reaction_step(self.h, n, nc, ptrs, T.ctypes.data, p, t0,
                                       None if dt_arr is None else dt_arr.ctypes.data, dt_s,
                                       None if Q is None else Q.ctypes.data, st.ctypes.data, ns.ctypes.data),
               "lsg_reaction_step")
        return Q, st, ns

    def step_cv(self, Y_species: np.ndarray, T: np.ndarray, rho: np.ndarray, dt, t0: float = 0.0,
                want_q: bool = True):
        """Constant-volume reactor (lsg_reaction_step_cv): as step(), with the
        per-cell density rho [ncells] instead of a pressure."""
        Y = Y_species
        if Y.dtype != np.float64 or not Y.flags.c_contiguous or T.dtype != np.float64:
            raise TypeError("Y_species and T must be C-contiguous float64")
        nc, n = Y.shape
        rho = np.ascontiguousarray(rho, dtype=np.float64)
        if rho.shape != (n,):
            raise ValueError("rho must have one value per cell")
        ptrs = (C.c_void_p * nc)(*[Y[i].ctypes.data for i in range(nc)])
        dt_arr = None
        dt_s = 0.0
        if np.ndim(dt) == 0:
            dt_s = float(dt)
        else:
            dt_arr = np.ascontiguousarray(dt, dtype=np.float64)
        Q = np.zeros(n) if want_q else None
        st = np.zeros(n, dtype=np.int32)
        ns = np.zeros(n, dtype=np.int32)
        _check(lib().lsg_reaction_step_cv(self.h, n, nc, ptrs, T.ctypes.data, rho.ctypes.data, t0,
                                          None if dt_arr is None else dt_arr.ctypes.data, dt_s,
                                          None if Q is None else Q.ctypes.data, st.ctypes.data, ns.ctypes.data),
               "lsg_reaction_step_cv")
        return Q, st, ns

    # ---- device arrays (torch tensors) ----
    def step_device(self, Y, T, dt=1e-5, p: float = 101325.0, t0: float = 0.0, Q=None, status=None,
                    nsteps=None, counters=None, stream=None):
        """Y: cuda float64 [NC, ld] species-major, T: [ncells]; in place."""
        _require_layout(Y, T, Q, status, nsteps, counters, dt if hasattr(dt, "data_ptr") else None)
        nc, ld = Y.shape
        n = T.shape[0]
        dtp, dts = (None, float(dt)) if not hasattr(dt, "data_ptr") else (dt.data_ptr(), 0.0)
        _check(lib().lsg_reaction_step_device(
            self.h, n, nc, Y.data_ptr(), ld, T.data_ptr(), p, t0, dtp, dts,
            None if Q is None else Q.data_ptr(), None if status is None else status.data_ptr(),
            None if nsteps is None else nsteps.data_ptr(), None if counters is None else counters.data_ptr(),
            _stream_handle(stream)), "lsg_reaction_step_device")

    def step_cv_device(self, Y, T, rho, dt=1e-5, t0: float = 0.0, Q=None, status=None, nsteps=None,
                       counters=None, stream=None):
        """Constant-volume reactor on device arrays (lsg_reaction_step_cv_device)."""
        _require_layout(Y, T, rho, Q, status, nsteps, counters, dt if hasattr(dt, "data_ptr") else None)
        nc, ld = Y.shape
        n = T.shape[0]
        dtp, dts = (None, float(dt)) if not hasattr(dt, "data_ptr") else (dt.data_ptr(), 0.0)
        _check(lib().lsg_reaction_step_cv_device(
            self.h, n, nc, Y.data_ptr(), ld, T.data_ptr(), rho.data_ptr(), t0, dtp, dts,
            None if Q is None else Q.data_ptr(), None if status is None else status.data_ptr(),
            None if nsteps is None else nsteps.data_ptr(), None if counters is None else counters.data_ptr(),
            _stream_handle(stream)), "lsg_reaction_step_cv_device")

    def step_sequence_device(self, Y, T, dt, nsteps: int, p: float = 101325.0, t0: float = 0.0, Q=None,
                             status=None, stream=None):
        """`nsteps` successive reaction steps on the same device arrays, the
        start time advancing by dt each step (a CFD run's chemistry calls with
        the state kept resident).  `dt` is a scalar.  Q and status, when given,
        hold the last step's heat release and ODE codes; returns the number of
        cells that reported a failure (status < 0) in any step."""
        import torch
        n = T.shape[0]
        st = status if status is not None else torch.empty(n, dtype=torch.int32, device=T.device)
        bad = torch.zeros(n, dtype=torch.bool, device=T.device)
        for k in range(nsteps):
            self.step_device(Y, T, dt, p=p, t0=t0 + k * float(dt), Q=Q, status=st, stream=stream)
            bad |= st < 0
        return int(bad.sum().item())

    def step_drg_device(self, Y, T, dt, key, bands=((1.e6, 1.e-2),), epsilon0: float = 1.e-2, min_T: float = 300.0,
                        first_cell_options_only: bool = True, p: float = 101325.0, t0: float = 0.0, Q=None,
                        status=None, n_species=None, n_reactions=None, counters=None, stream=None):
        """lsg_reaction_step_drg_device: the DRG-reduced step (chemistry_DRG.H) of device arrays Y [NC, ld]
        and T [ncells], in place.  key: key species indices; bands: (temperature, epsilon) pairs."""
        _require_layout(Y, T, Q, status, n_species, n_reactions, counters,
                        dt if hasattr(dt, "data_ptr") else None)
        nc, ld = Y.shape
        n = T.shape[0]
        k = (C.c_int * len(key))(*[int(x) for x in key])
        bt = (C.c_double * len(bands))(*[float(b[0]) for b in bands])
        be = (C.c_double * len(bands))(*[float(b[1]) for b in bands])
        o = DrgOptions(C.cast(k, C.c_void_p), len(key), C.cast(bt, C.c_void_p), C.cast(be, C.c_void_p), len(bands),
                       float(epsilon0), float(min_T), int(bool(first_cell_options_only)))
        dtp, dts = (None, float(dt)) if not hasattr(dt, "data_ptr") else (dt.data_ptr(), 0.0)
        ptr = (lambda x: None if x is None else x.data_ptr())
        _check(lib().lsg_reaction_step_drg_device(
            self.h, n, nc, Y.data_ptr(), ld, T.data_ptr(), p, t0, dtp, dts, C.byref(o), ptr(Q), ptr(status),
            ptr(n_species), ptr(n_reactions), ptr(counters), _stream_handle(stream)), "lsg_reaction_step_drg_device")

    def step_drg(self, Y_species: np.ndarray, T: np.ndarray, dt, key, bands=((1.e6, 1.e-2),), epsilon0: float = 1.e-2,
                 min_T: float = 300.0, first_cell_options_only: bool = True, p: float = 101325.0, t0: float = 0.0):
        """lsg_reaction_step_drg from host arrays: Y_species [NC, ncells] (C-contiguous float64) and T
        [ncells], updated in place.  Returns (Q, status, n_species, n_reactions)."""
        nc, n = Y_species.shape
        if Y_species.dtype != np.float64 or not Y_species.flags.c_contiguous or T.dtype != np.float64:
            raise TypeError("Y_species [NC, ncells] and T must be C-contiguous float64")
        rows = (C.c_void_p * nc)(*[Y_species[i].ctypes.data for i in range(nc)])
        k = (C.c_int * len(key))(*[int(x) for x in key])
        bt = (C.c_double * len(bands))(*[float(b[0]) for b in bands])
        be = (C.c_double * len(bands))(*[float(b[1]) for b in bands])
        o = DrgOptions(C.cast(k, C.c_void_p), len(key), C.cast(bt, C.c_void_p), C.cast(be, C.c_void_p), len(bands),
                       float(epsilon0), float(min_T), int(bool(first_cell_options_only)))
        dt_arr = None if np.ndim(dt) == 0 else np.ascontiguousarray(dt, dtype=np.float64)
        Q = np.zeros(n)
        st = np.zeros(n, dtype=np.int32)
        nsp = np.zeros(n, dtype=np.int32)
        nrx = np.zeros(n, dtype=np.int32)
        _check(lib().lsg_reaction_step_drg(
            self.h, n, nc, C.cast(rows, C.POINTER(C.c_void_p)), T.ctypes.data, p, t0,
            None if dt_arr is None else dt_arr.ctypes.data, 0.0 if dt_arr is not None else float(dt), C.byref(o),
            Q.ctypes.data, st.ctypes.data, nsp.ctypes.data, nrx.ctypes.data), "lsg_reaction_step_drg")
        return Q, st, nsp, nrx

    def step_sequence_graph(self, Y, T, dt: float, nsteps: int, p: float = 101325.0, t0: float = 0.0, Q=None,
                            status=None, stream=None) -> bool:
        """lsg_reaction_step_sequence_device: `nsteps` successive steps of the device-resident cells,
        captured once into a CUDA graph by the library and replayed (the round scheme runs them one by
        one).  Returns True when the graph ran."""
        _require_layout(Y, T, Q, status)
        nc, ld = Y.shape
        n = T.shape[0]
        used = C.c_int(0)
        _check(lib().lsg_reaction_step_sequence_device(
            self.h, int(nsteps), n, nc, Y.data_ptr(), ld, T.data_ptr(), p, t0, float(dt),
            None if Q is None else Q.data_ptr(), None if status is None else status.data_ptr(), C.byref(used),
            _stream_handle(stream)), "lsg_reaction_step_sequence_device")
        return bool(used.value)

    def compact_sources_device(self, Y0, T0, Yf, Tf, dt, RR, RT=None, p: float = 101325.0, stream=None):
        """Source terms of the compact Strang scheme (lsg_compact_sources_device):
        RR [NC, ld] and RT [ncells] from the fields before (Y0, T0) and after
        (Yf, Tf) a step of length dt (scalar or a per-cell tensor)."""
        _require_layout(Y0, T0, Yf, Tf, RR, RT, dt if hasattr(dt, "data_ptr") else None)
        nc, ld = Y0.shape
        n = T0.shape[0]
        if Yf.shape != Y0.shape or RR.shape != Y0.shape:
            raise ValueError("Y0, Yf and RR must have the same shape")
        dtp, dts = (None, float(dt)) if not hasattr(dt, "data_ptr") else (dt.data_ptr(), 0.0)
        _check(lib().lsg_compact_sources_device(
            self.h, n, nc, Y0.data_ptr(), T0.data_ptr(), Yf.data_ptr(), Tf.data_ptr(), ld, p, dtp, dts,
            RR.data_ptr(), None if RT is None else RT.data_ptr(), _stream_handle(stream)),
            "lsg_compact_sources_device")

    def steady_sources_device(self, Y, T, S_implicit, S_explicit, p=101325.0, stream=None):
        """Linearised source terms of the steady solvers (lsg_steady_sources_device): S_implicit and
        S_explicit [NC + 1, lds]; p a scalar or a per-cell tensor."""
        _require_layout(Y, T, S_implicit, S_explicit, p if hasattr(p, "data_ptr") else None)
        nc, ld = Y.shape
        pp, ps = (p.data_ptr(), 0.0) if hasattr(p, "data_ptr") else (None, float(p))
        _check(lib().lsg_steady_sources_device(self.h, T.shape[0], nc, Y.data_ptr(), T.data_ptr(), ld, pp, ps,
                                               S_implicit.data_ptr(), S_explicit.data_ptr(), S_implicit.shape[1],
                                               _stream_handle(stream)), "lsg_steady_sources_device")

    def steady_sources_sparse_device(self, Y, T, S_implicit, S_explicit, p=101325.0, species=True, energy=True,
                                     stream=None):
        """The steady solvers' default linearisation, sparseJacobian true (lsg_steady_sources_sparse_device):
        as steady_sources_device with the analytic species diagonal."""
        _require_layout(Y, T, S_implicit, S_explicit, p if hasattr(p, "data_ptr") else None)
        nc, ld = Y.shape
        pp, ps = (p.data_ptr(), 0.0) if hasattr(p, "data_ptr") else (None, float(p))
        _check(lib().lsg_steady_sources_sparse_device(
            self.h, T.shape[0], nc, Y.data_ptr(), T.data_ptr(), ld, pp, ps, int(species), int(energy),
            S_implicit.data_ptr(), S_explicit.data_ptr(), S_implicit.shape[1], _stream_handle(stream)),
            "lsg_steady_sources_sparse_device")

    def formation_rates_device(self, Y, T, out, p: float = 101325.0, stream=None):
        """R_i MW_i [kg/m3/s] of every species at the states (Y [NC, ld], T) into out [NC, ld_out]."""
        _require_layout(Y, T, out)
        nc, ld = Y.shape
        _check(lib().lsg_formation_rates_device(self.h, T.shape[0], nc, Y.data_ptr(), T.data_ptr(), ld, p,
                                                out.data_ptr(), out.shape[1], _stream_handle(stream)),
               "lsg_formation_rates_device")

    def _property_request(self, soret: bool, fields, thermal: bool):
        nt = len(self.mech.transport_info()[1])
        want = set(PROPERTY_FIELDS if fields is None else fields)
        if not soret:
            want.discard("Dsoret")
        if not thermal:   # evaluated only with the energy equation or Lewis numbers
            want -= {"lambda", "cp", "cv", "cp_species"}
        if "Dsoret" in want:
            want.add("Dmix")
        rows = {"X": self.mech.n_species, "cp_species": self.mech.n_species, "Dmix": self.mech.n_species,
                "Dsoret": nt}
        return [f for f in PROPERTY_FIELDS if f in want], rows

    def properties_device(self, Y, T, p=None, p_scalar: float = 101325.0, energy: bool = True, lewis=None,
                          simplified: bool = False, soret: bool = False, fields=None, stream=None) -> dict:
        """Property update of the cells (Y [NC, ld], T [ncells], p [ncells] or p_scalar) on the
        device: a dict of new CUDA tensors, species fields [rows, ncells]; lewis a CUDA tensor
        of NC Lewis numbers or None (mixture-averaged diffusivities)."""
        import torch
        _require_layout(Y, T, p, lewis)
        nc, ld = Y.shape
        n = T.shape[0]
        names, rows = self._property_request(soret, fields, energy or lewis is not None)
        out = {f: torch.empty((rows[f], n) if f in rows else (n,), dtype=torch.float64, device=Y.device)
               for f in names}
        fd = PropertyFields(**{f: out[f].data_ptr() for f in names})
        opt = PropertyOptions(int(energy), int(simplified), None if lewis is None else lewis.data_ptr())
        _check(lib().lsg_properties_device(self.h, n, nc, Y.data_ptr(), T.data_ptr(), ld,
                                           None if p is None else p.data_ptr(), p_scalar, C.byref(opt),
                                           C.byref(fd), n, _stream_handle(stream)), "lsg_properties_device")
        return out

    def properties(self, Y, T, p=None, p_scalar: float = 101325.0, energy: bool = True, lewis=None,
                   simplified: bool = False, soret: bool = False, fields=None) -> dict:
        """The same from host arrays (Y [NC, ncells] species-major, float64): numpy fields."""
        Y = np.ascontiguousarray(Y, dtype=np.float64)
        T = np.ascontiguousarray(T, dtype=np.float64)
        nc, n = Y.shape
        names, rows = self._property_request(soret, fields, energy or lewis is not None)
        out = {f: np.empty((rows[f], n) if f in rows else (n,)) for f in names}
        fd = PropertyFields(**{f: out[f].ctypes.data for f in names})
        le = None if lewis is None else np.ascontiguousarray(lewis, dtype=np.float64)
        pp = None if p is None else np.ascontiguousarray(p, dtype=np.float64)
        opt = PropertyOptions(int(energy), int(simplified), None if le is None else le.ctypes.data)
        _check(lib().lsg_properties(self.h, n, nc, Y.ctypes.data, T.ctypes.data,
                                    None if pp is None else pp.ctypes.data, p_scalar, C.byref(opt), C.byref(fd)),
               "lsg_properties")
        return out

    def rhs_device(self, y, dy, p: float = 101325.0, qr=None, stream=None):
        _require_layout(y, dy, qr)
        n1, ld = y.shape
        n = ld if qr is None else qr.shape[0]
        _check(lib().lsg_rhs_device(self.h, n, y.data_ptr(), dy.data_ptr(), ld, p,
                                    None if qr is None else qr.data_ptr(),
                                    _stream_handle(stream)), "lsg_rhs_device")

    def build_and_invert_g_device(self, J, hr0, inv, stream=None):
        """lsg_build_and_invert_g_device: G^-1 (FP32) of G = I - hr0 J for a batch of Jacobians.
        J: cuda float64 [nmat, n, n] holding each Jacobian column-major (J[m].T is the matrix, i.e.
        J[m][j][i] = J_ij); hr0: float64 [nmat]; inv: float32 [nmat, n, n], written the same way."""
        _require_layout(J, hr0, inv)
        nmat, n, n2 = J.shape
        if n != n2 or tuple(inv.shape) != (nmat, n, n) or hr0.shape[0] != nmat:
            raise ValueError("J, hr0 and inv shapes disagree")
        _check(lib().lsg_build_and_invert_g_device(self.h, nmat, n, J.data_ptr(), hr0.data_ptr(), inv.data_ptr(),
                                                   _stream_handle(stream)), "lsg_build_and_invert_g_device")

    def jacobian_device(self, y, J, p: float = 101325.0, stream=None):
        """lsg_jacobian_device: y cuda float64 [n, ld] (species-major, row n-1 = T); J float64
        [ncells, n, n] receives df/dy row-major per state."""
        _require_layout(y, J)
        n, ld = y.shape
        ncells = J.shape[0]
        if tuple(J.shape) != (ncells, n, n):
            raise ValueError("J must be [ncells, n, n]")
        _check(lib().lsg_jacobian_device(self.h, ncells, y.data_ptr(), ld, p, J.data_ptr(), _stream_handle(stream)),
               "lsg_jacobian_device")

    def launches(self) -> int:
        """Kernels this context has enqueued so far."""
        return int(lib().lsg_ctx_launches(self.h))

    KERNEL_KINDS = ("rhs", "advance", "compact", "init", "plain", "persistent", "block", "group")

    def kernel_times(self, reset: bool = False) -> dict:
        """{kind: (total ms, timed launches)} from the CUDA events recorded when
        the context was created with kernel_timing=1."""
        nk = len(self.KERNEL_KINDS)
        ms = (C.c_double * nk)()
        nl = (C.c_longlong * nk)()
        _check(lib().lsg_ctx_kernel_times(self.h, C.cast(ms, C.c_void_p), C.cast(nl, C.c_void_p), nk, int(reset)),
               "lsg_ctx_kernel_times")
        return {k: (ms[i], nl[i]) for i, k in enumerate(self.KERNEL_KINDS)}

    TUNE_CANDIDATES = ("rounds16", "rounds32", "plain_warp", "persistent", "group_4", "group_2")
    # mechanisms above 31 species, mixed precision: the block form's factorisation
    TUNE_CANDIDATES_LARGE = ("block_fp64_lu", "block_tc_inverse")

    def tuning(self):
        """(tile, width, {candidate: cells/s}) chosen by the autotuner, or None before it ran."""
        tile, width = C.c_int(), C.c_int()
        rates = (C.c_double * len(self.TUNE_CANDIDATES))()
        rc = lib().lsg_ctx_tuning(self.h, C.byref(tile), C.byref(width), C.cast(rates, C.c_void_p))
        if rc != 0:
            return None
        names = self.TUNE_CANDIDATES_LARGE if tile.value == LSG_TILE_BLOCK else self.TUNE_CANDIDATES
        return tile.value, width.value, {k: rates[i] for i, k in enumerate(names)}

    def check(self):
        f = C.c_int()
        rc = lib().lsg_ctx_check(self.h, C.byref(f))
        if rc != 0:
            raise LsgError(f"device error flags 0x{f.value:x}: {lib().lsg_strerror(rc).decode()}")


def step_device_noalloc(mech: Mechanism, Y, T, dt=1e-5, p: float = 101325.0, t0: float = 0.0,
                        options: Optional[Options] = None, Q=None, status=None, nsteps=None, counters=None,
                        stream=None):
    """lsg_reaction_step_device_noalloc: the reaction step without any device
    allocation, for callers that cannot allocate while they advance the
    chemistry (see include/lsmoke_gpu.h).  Same array layout as
    ReactionStep.step_device; synchronous; calls must not overlap on the GPU."""
    _require_layout(Y, T, Q, status, nsteps, counters, dt if hasattr(dt, "data_ptr") else None)
    nc, ld = Y.shape
    n = T.shape[0]
    dtp, dts = (None, float(dt)) if not hasattr(dt, "data_ptr") else (dt.data_ptr(), 0.0)
    opt = None if options is None else C.byref(options)
    _check(lib().lsg_reaction_step_device_noalloc(
        mech.h, opt, n, nc, Y.data_ptr(), ld, T.data_ptr(), p, t0, dtp, dts,
        None if Q is None else Q.data_ptr(), None if status is None else status.data_ptr(),
        None if nsteps is None else nsteps.data_ptr(), None if counters is None else counters.data_ptr(),
        _stream_handle(stream)), "lsg_reaction_step_device_noalloc")
