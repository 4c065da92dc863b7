"""freeshearlayer_b200 -- B200 (sm_100a) explicit time step of freeShearLayer.

Python view of the C ABI in ``include/fsl_gpu.h`` (libfsl_gpu.so, built
in-tree by ``make -C freeshearlayer_b200``).  One :class:`Domain` is one
device-resident domain; its methods carry the reference's phase names
(src/layer2.c:141-185) so a driver reads like the reference's main loop::

    d = Domain(params)                 # Initialize()  (src/initialize.c:14)
    d.upload_state(state)
    d.checkCoNum()                     # src/helpers.c:23
    d.draw_disturbance()               # src/layer2.c:152-162
    for stage in (1, 2, 3):
        d.BounCondInGhostCells()       # src/boundCondInGhostCells.c:10
        d.Reconstruction()             # src/reconstruction.c:26
        d.BounCondOnInterfaces()       # src/bounCondOnInterfaces.c:11
        d.Fluxes()                     # src/fluxes.c:12 (includes DynamicSmagorinsky)
        d.Evolution(3, stage)          # src/evolution.c:15

or, fused and asynchronous, ``d.step(n)``.  There is no CPU path: loading
fails with :class:`FslError` when the library is missing, and creating a
domain fails when no sm_100 device is present.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

__all__ = ["Params", "Domain", "FslError", "lib", "LIB_PATH", "default_params",
           "params_from_ini", "params_from_bin", "initial_state", "temporal_state",
           "SETUP_SPATIAL", "SETUP_TEMPORAL", "CFL_STREAMWISE", "CFL_ACOUSTIC",
           "PREC_FP64", "PREC_FP32", "SGS_DYNAMIC", "SGS_LEARNED", "SGS_STATIC", "SGS_NONE", "RECON_CHARMINMOD",
           "RECON_PPM", "Trainer", "Ensemble", "closure_weights", "shear_statistics", "favre_from_probes",
           "favre_profiles", "debug_bounds",
           "tecplot_write"]

HERE = os.path.dirname(os.path.abspath(__file__))
# FSL_GPU_LIB=checked loads the bounds-checked debug build (libfsl_gpu_checked.so)
LIB_PATH = os.path.join(HERE, "libfsl_gpu_checked.so" if os.environ.get("FSL_GPU_LIB") == "checked"
                        else "libfsl_gpu.so")

FSL_OK = 0
ERRORS = {-1: "FSL_ERR_ARG", -2: "FSL_ERR_NOMEM", -3: "FSL_ERR_CUDA", -4: "FSL_ERR_NONFINITE",
          -5: "FSL_ERR_TIMEOUT", -6: "FSL_ERR_IO", -7: "FSL_ERR_UNSUPPORTED", -8: "FSL_ERR_NODEVICE",
          -9: "FSL_ERR_TOO_LARGE"}
SETUP_SPATIAL, SETUP_TEMPORAL = 0, 1
CFL_STREAMWISE, CFL_ACOUSTIC = 0, 1
PREC_FP64, PREC_FP32 = 0, 1
SGS_DYNAMIC, SGS_LEARNED, SGS_STATIC, SGS_NONE = 0, 1, 2, 3
RECON_CHARMINMOD, RECON_PPM = 0, 1


class FslError(RuntimeError):
    def __init__(self, code: int, what: str = ""):
        self.code = code
        super().__init__("%s (%d)%s" % (ERRORS.get(code, "FSL_ERR"), code, (": " + what) if what else ""))


class Params(C.Structure):
    """fsl_params: the 22 layer2.ini values in file order, then the options."""

    _fields_ = [("LEN", C.c_int), ("HIG", C.c_int), ("DEP", C.c_int),
                ("deltaX", C.c_double), ("deltaY", C.c_double), ("deltaZ", C.c_double),
                ("deltaT", C.c_double), ("Answer", C.c_int), ("numstep", C.c_int),
                ("mu_L", C.c_double), ("Pr_L", C.c_double), ("Pr_T", C.c_double),
                ("Cs", C.c_double), ("BL_HIG", C.c_int), ("Ua", C.c_double),
                ("Va", C.c_double), ("Wa", C.c_double), ("Ns_min", C.c_int),
                ("Nst", C.c_int), ("f_step", C.c_int), ("nStages", C.c_int),
                ("maxCoNum", C.c_double), ("setup", C.c_int), ("cfl_mode", C.c_int),
                ("seed_X", C.c_double), ("precision", C.c_int), ("sgs", C.c_int),
                ("recon", C.c_int), ("reserved", C.c_int * 8)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}


class Info(C.Structure):
    _fields_ = [("deltaT", C.c_double), ("deltaT_X", C.c_double), ("deltaT_Y", C.c_double),
                ("deltaT_Z", C.c_double), ("maxCo", C.c_double), ("X", C.c_double),
                ("Ud", C.c_double), ("Vd", C.c_double), ("Wd", C.c_double),
                ("k_min", C.c_uint), ("k_max", C.c_uint), ("step", C.c_uint),
                ("counter", C.c_int), ("cur", C.c_int), ("DD", C.c_double),
                ("lambda_L", C.c_double), ("cp_Pr_T", C.c_double),
                ("device_bytes", C.c_ulonglong)]


K_CLASSES = ["stage", "recon", "flux", "sgs", "evol", "bc", "cfl", "other"]
CLOSURE_NPARAMS = 9473


class ClosureStats(C.Structure):
    _fields_ = [("profile_err", C.c_double), ("cell_err", C.c_double), ("mu_profile_err", C.c_double),
                ("visc_err", C.c_double), ("judgements", C.c_int),
                ("fallbacks", C.c_int), ("using_dynamic", C.c_int), ("last_step", C.c_uint),
                ("mu_active_err", C.c_double), ("dyn_ratio", C.c_double), ("active_rows", C.c_int),
                ("dynamic_steps", C.c_int)]


class BoundsReport(C.Structure):
    _fields_ = [("hits", C.c_ulonglong), ("unit", C.c_int), ("line", C.c_int), ("index", C.c_longlong),
                ("extent", C.c_longlong)]


class KTimes(C.Structure):
    _fields_ = [("ms", C.c_double * 8), ("launches", C.c_ulonglong * 8)]

    def as_dict(self) -> dict:
        return {n: (self.ms[i], self.launches[i]) for i, n in enumerate(K_CLASSES)}


_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_lib = None


def lib():
    """Load libfsl_gpu.so (raises FslError if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FslError(-8, "%s not built: run `make -C %s%s`"
                           % (os.path.basename(LIB_PATH), HERE, " checked" if "checked" in LIB_PATH else ""))
        L = C.CDLL(LIB_PATH)
        vp, i, d, u = C.c_void_p, C.c_int, C.c_double, C.c_uint
        P = C.POINTER(Params)
        sig = {
            "fsl_params_default": [P], "fsl_params_from_ini": [C.c_char_p, P],
            "fsl_params_from_bin": [C.c_char_p, P], "fsl_params_check": [P],
            "fsl_initial_state": [P, _dp],
            "fsl_temporal_state": [P, d, d, d, C.c_ulonglong, _dp, C.POINTER(C.c_double)],
            "fsl_init": [P, C.POINTER(C.c_void_p)], "fsl_destroy": [vp],
            "fsl_get_info": [vp, C.POINTER(Info)], "fsl_sync": [vp],
            "fsl_upload_state": [vp, _dp], "fsl_download_state": [vp, _dp],
            "fsl_set_time": [vp, u, d],
            "fsl_check_courant": [vp, C.POINTER(C.c_double), C.POINTER(C.c_double)],
            "fsl_draw_disturbance": [vp], "fsl_set_disturbance": [vp, u, u, d, d, d],
            "fsl_ghost_bc": [vp], "fsl_reconstruct": [vp], "fsl_interface_bc": [vp],
            "fsl_dynamic_smagorinsky": [vp], "fsl_fluxes": [vp], "fsl_evolution": [vp, i],
            "fsl_step": [vp, i], "fsl_step_phased": [vp, i], "fsl_step_stage": [vp],
            "fsl_get_cells": [vp, i, i, _dp], "fsl_set_cells": [vp, i, i, _dp],
            "fsl_get_faces": [vp, i, i, i, _dp], "fsl_set_faces": [vp, i, i, i, _dp],
            "fsl_set_cur": [vp, i], "fsl_sums": [vp, _dp], "fsl_plane_sums": [vp, _dp],
        }
        fp = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
        ll = C.c_longlong
        sig.update({
            "fsl_closure_set_scales": [vp, d, d], "fsl_closure_set_weights": [vp, fp],
            "fsl_closure_get_weights": [vp, fp], "fsl_closure_judge": [vp, i, d],
            "fsl_closure_judge_active": [vp, d, d],
            "fsl_closure_get_stats": [vp, C.POINTER(ClosureStats)],
            "fsl_closure_compare": [vp, C.c_void_p, C.c_void_p, C.POINTER(ClosureStats)],
            "fsl_trainer_create": [ll, C.c_ulonglong, C.POINTER(C.c_void_p)],
            "fsl_trainer_destroy": [vp], "fsl_trainer_harvest": [vp, vp, i],
            "fsl_trainer_get_samples": [vp, fp, fp, ll], "fsl_trainer_set_samples": [vp, fp, fp, ll],
            "fsl_trainer_get_weights": [vp, fp], "fsl_trainer_set_weights": [vp, fp],
            "fsl_trainer_gradient": [vp, ll, fp, C.POINTER(C.c_double)], "fsl_trainer_set_loss": [vp, i],
            "fsl_trainer_train": [vp, i, ll, d, C.POINTER(C.c_double)],
        })
        sig.update({
            "fsl_ensemble_create": [C.POINTER(C.c_void_p), i, C.POINTER(C.c_void_p)],
            "fsl_ensemble_destroy": [vp], "fsl_ensemble_set_chunk": [vp, i], "fsl_ensemble_step": [vp, i],
            "fsl_ensemble_sync": [vp], "fsl_ensemble_persistent": [vp],
            "fsl_ensemble_set_barrier_limit": [vp, C.c_uint],
            "fsl_ensemble_tune": [vp, i, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_double)],
        })
        cs = C.c_char_p
        sig.update({
            "fsl_write_backup": [vp, cs, i], "fsl_read_backup": [vp, cs, i], "fsl_probe_rows": [vp, _dp],
            "fsl_write_probes": [vp, cs, i], "fsl_favre_reset": [vp], "fsl_favre_accumulate": [vp],
            "fsl_favre_read": [vp, _dp, C.POINTER(C.c_int)],
            "fsl_favre_from_probes": [cs, i, i, i, i, _dp, C.POINTER(C.c_int)],
            "fsl_favre_profiles": [cs, i, i, i, cs, C.POINTER(C.c_int)],
            "fsl_output_fields": [vp, _dp], "fsl_write_tecplot": [vp, cs],
            "fsl_tecplot_write": [cs, i, i, i, _dp],
        })
        sig.update({
            "fsl_get_planes": [vp, i, i, vp], "fsl_set_planes": [vp, i, i, vp],
            "fsl_get_planes_async": [vp, i, i, vp], "fsl_set_planes_async": [vp, i, i, vp],
            "fsl_set_courant_range": [vp, i, i], "fsl_courant_prepare": [vp],
            "fsl_upload_state_async": [vp, _dp], "fsl_download_state_async": [vp, _dp], "fsl_transfer_wait": [vp],
            "fsl_get_courant_max": [vp, C.POINTER(C.c_double)], "fsl_set_courant_max": [vp, d],
        })
        sig["fsl_tune"] = [vp, i, i]
        sig["fsl_debug_bounds"] = [C.POINTER(BoundsReport), i]
        sig["fsl_profile"] = [vp, i]
        sig["fsl_profile_read"] = [vp, C.POINTER(KTimes)]
        for name, args in sig.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = C.c_int
        L.fsl_last_error.argtypes = [vp]
        L.fsl_last_error.restype = C.c_char_p
        L.fsl_stream.argtypes = [vp]
        L.fsl_stream.restype = C.c_void_p
        L.fsl_ensemble_last_error.argtypes = [vp]
        L.fsl_ensemble_last_error.restype = C.c_char_p
        L.fsl_ensemble_stream.argtypes = [vp]
        L.fsl_ensemble_stream.restype = C.c_void_p
        L.fsl_courant_bits.argtypes = [vp]
        L.fsl_courant_bits.restype = C.c_void_p
        L.fsl_trainer_size.argtypes = [vp]
        L.fsl_trainer_size.restype = C.c_longlong
        _lib = L
    return _lib


def _check(rc: int, h=None):
    if rc != FSL_OK:
        what = lib().fsl_last_error(h).decode() if h else ""
        raise FslError(rc, what)


def debug_bounds(clear: bool = False) -> dict:
    """The bounds-checked build's report (FSL_GPU_LIB=checked): offending
    global-memory accesses since the last clear and the first one's file
    (1 fsl_fused.cu, 2 fsl_fused32.cu, 3 fsl_mlp.cu, 4 fsl_phase.cu,
    5 fsl_dyn32.cu, 6 fsl_io.cu), line, index and extent.  Raises FslError (FSL_ERR_UNSUPPORTED) in the product
    build."""
    r = BoundsReport()
    _check(lib().fsl_debug_bounds(C.byref(r), 1 if clear else 0))
    return {"hits": int(r.hits), "unit": r.unit, "line": r.line, "index": r.index, "extent": r.extent}


def default_params(**kw) -> Params:
    p = Params()
    _check(lib().fsl_params_default(C.byref(p)))
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def params_from_ini(path: str, **kw) -> Params:
    p = default_params()
    _check(lib().fsl_params_from_ini(path.encode(), C.byref(p)))
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def params_from_bin(path: str, **kw) -> Params:
    p = default_params()
    _check(lib().fsl_params_from_bin(path.encode(), C.byref(p)))
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def _as_params(p) -> Params:
    if isinstance(p, Params):
        return p
    q = default_params()
    for k, v in dict(p).items():
        if hasattr(q, k):
            setattr(q, k, v)
    return q


def state_size(p) -> int:
    return p.LEN * p.HIG * 5 * p.DEP


def initial_state(p) -> np.ndarray:
    p = _as_params(p)
    out = np.empty(state_size(p), np.float64)
    _check(lib().fsl_initial_state(C.byref(p), out))
    return out


def temporal_state(p, Mc: float, delta_w0: float = 1.0, amp: float = 1e-3,
                   seed: int = 20251203):
    p = _as_params(p)
    out = np.empty(state_size(p), np.float64)
    dU = C.c_double()
    _check(lib().fsl_temporal_state(C.byref(p), Mc, delta_w0, amp, seed, out, C.byref(dU)))
    return out, dU.value


def _buffer_ptr(buf, n: int) -> int:
    """Address of a contiguous float64 buffer of at least n values (numpy
    array or torch tensor, host or CUDA)."""
    if isinstance(buf, np.ndarray):
        if buf.dtype != np.float64 or not buf.flags.c_contiguous or buf.size < n:
            raise FslError(-1, "buffer: contiguous float64 with %d values expected" % n)
        return buf.ctypes.data
    if hasattr(buf, "data_ptr"):
        import torch
        if buf.dtype != torch.float64 or not buf.is_contiguous() or buf.numel() < n:
            raise FslError(-1, "buffer: contiguous float64 with %d values expected" % n)
        return buf.data_ptr()
    raise FslError(-1, "buffer: numpy array or torch tensor expected")


class Domain:
    """One device-resident domain (an fsl_ctx) on the current CUDA device."""

    def __init__(self, params):
        self.p = _as_params(params)
        h = C.c_void_p()
        _check(lib().fsl_init(C.byref(self.p), C.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            lib().fsl_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _c(self, rc):
        _check(rc, self.h)

    # --- shapes -------------------------------------------------------------
    @property
    def padded_shape(self):
        return (self.p.LEN + 2, self.p.HIG + 2, self.p.DEP + 2)

    def face_shape(self, d: int):
        return (self.p.LEN + (d == 0), self.p.HIG + (d == 1), self.p.DEP + (d == 2))

    # --- state ----------------------------------------------------------------
    def upload_state(self, state: np.ndarray):
        self._c(lib().fsl_upload_state(self.h, np.ascontiguousarray(state, np.float64).ravel()))

    def download_state(self, out: np.ndarray | None = None) -> np.ndarray:
        """U^n into `out` (a contiguous float64 array, e.g. over pinned memory)
        or into a new array."""
        if out is None:
            out = np.empty(state_size(self.p), np.float64)
        elif out.dtype != np.float64 or not out.flags.c_contiguous or out.size != state_size(self.p):
            raise FslError(-1, "download_state: out must be contiguous float64 of the state size")
        self._c(lib().fsl_download_state(self.h, out))
        return out

    def set_time(self, step: int, dt: float):
        self._c(lib().fsl_set_time(self.h, step, dt))

    def upload_state_async(self, state: np.ndarray):
        """Queue U^n <- state (a contiguous float64 array, pinned for overlap);
        the array must stay untouched until transfer_wait()."""
        if state.dtype != np.float64 or not state.flags.c_contiguous or state.size != state_size(self.p):
            raise FslError(-1, "upload_state_async: contiguous float64 of the state size expected")
        self._c(lib().fsl_upload_state_async(self.h, state.reshape(-1)))
        self._pending = getattr(self, "_pending", []) + [state]

    def download_state_async(self, out: np.ndarray):
        """Queue out <- U^n (contiguous float64, pinned for overlap); valid
        after transfer_wait()."""
        if out.dtype != np.float64 or not out.flags.c_contiguous or out.size != state_size(self.p):
            raise FslError(-1, "download_state_async: contiguous float64 of the state size expected")
        self._c(lib().fsl_download_state_async(self.h, out.reshape(-1)))
        self._pending = getattr(self, "_pending", []) + [out]

    def transfer_wait(self):
        self._c(lib().fsl_transfer_wait(self.h))
        self._pending = []

    # --- x-slabs ------------------------------------------------------------------
    def plane_size(self) -> int:
        return self.p.HIG * 5 * self.p.DEP

    def get_planes(self, i0: int, n: int, out):
        """Planes i0..i0+n-1 (1-based) of U^n into `out`: a contiguous float64
        numpy array or CUDA tensor of at least n * plane_size() values."""
        self._c(lib().fsl_get_planes(self.h, i0, n, _buffer_ptr(out, n * self.plane_size())))
        return out

    def set_planes(self, i0: int, n: int, buf):
        self._c(lib().fsl_set_planes(self.h, i0, n, _buffer_ptr(buf, n * self.plane_size())))

    def get_planes_async(self, i0: int, n: int, out):
        """get_planes queued on the domain's stream without waiting (`out`: a
        CUDA tensor, or pinned host memory)."""
        self._c(lib().fsl_get_planes_async(self.h, i0, n, _buffer_ptr(out, n * self.plane_size())))
        return out

    def set_planes_async(self, i0: int, n: int, buf):
        self._c(lib().fsl_set_planes_async(self.h, i0, n, _buffer_ptr(buf, n * self.plane_size())))

    def set_courant_range(self, i0: int, i1: int):
        self._c(lib().fsl_set_courant_range(self.h, i0, i1))

    def courant_prepare(self):
        self._c(lib().fsl_courant_prepare(self.h))

    def get_courant_max(self) -> float:
        m = C.c_double()
        self._c(lib().fsl_get_courant_max(self.h, C.byref(m)))
        return m.value

    def set_courant_max(self, m: float):
        self._c(lib().fsl_set_courant_max(self.h, m))

    def courant_bits_ptr(self) -> int:
        """Device address of the Courant maximum's bit pattern (uint64)."""
        return lib().fsl_courant_bits(self.h)

    def info(self) -> Info:
        i = Info()
        self._c(lib().fsl_get_info(self.h, C.byref(i)))
        return i

    def sync(self):
        self._c(lib().fsl_sync(self.h))

    # --- driver scalar work -----------------------------------------------------
    def check_courant(self):
        mc, dt = C.c_double(), C.c_double()
        self._c(lib().fsl_check_courant(self.h, C.byref(mc), C.byref(dt)))
        return mc.value, dt.value

    def draw_disturbance(self):
        self._c(lib().fsl_draw_disturbance(self.h))

    def set_disturbance(self, k_min, k_max, Ud, Vd, Wd):
        self._c(lib().fsl_set_disturbance(self.h, k_min, k_max, Ud, Vd, Wd))

    # --- phases -------------------------------------------------------------------
    def ghost_bc(self): self._c(lib().fsl_ghost_bc(self.h))
    def reconstruct(self): self._c(lib().fsl_reconstruct(self.h))
    def interface_bc(self): self._c(lib().fsl_interface_bc(self.h))
    def dynamic_smagorinsky(self): self._c(lib().fsl_dynamic_smagorinsky(self.h))
    def fluxes(self): self._c(lib().fsl_fluxes(self.h))
    def evolution(self, stage: int): self._c(lib().fsl_evolution(self.h, stage))
    def step(self, n: int = 1): self._c(lib().fsl_step(self.h, n))
    def step_phased(self, n: int = 1): self._c(lib().fsl_step_phased(self.h, n))
    def step_stage(self): self._c(lib().fsl_step_stage(self.h))

    # reference names (src/layer2.c:147-176)
    def checkCoNum(self): return self.check_courant()
    def BounCondInGhostCells(self): self.ghost_bc()
    def Reconstruction(self): self.reconstruct()
    def BounCondOnInterfaces(self): self.interface_bc()
    def DynamicSmagorinsky(self): self.dynamic_smagorinsky()

    def Fluxes(self):
        """Fluxes() including its DynamicSmagorinsky(U1..U4) call (src/fluxes.c:52-54)."""
        self.dynamic_smagorinsky()
        self.fluxes()

    def Evolution(self, nStages: int, Stage: int):
        if nStages != self.p.nStages:
            raise FslError(-1, "nStages is fixed at domain creation (%d)" % self.p.nStages)
        self.evolution(Stage)

    # --- debug access -------------------------------------------------------------
    def cells(self, which: int, var: int = 0) -> np.ndarray:
        out = np.empty(self.padded_shape, np.float64)
        self._c(lib().fsl_get_cells(self.h, which, var, out))
        return out

    def set_cells(self, which: int, var: int, a: np.ndarray):
        self._c(lib().fsl_set_cells(self.h, which, var, np.ascontiguousarray(a, np.float64)))

    def faces(self, d: int, side: int, var: int) -> np.ndarray:
        out = np.empty(self.face_shape(d), np.float64)
        self._c(lib().fsl_get_faces(self.h, d, side, var, out))
        return out

    def set_faces(self, d: int, side: int, var: int, a: np.ndarray):
        self._c(lib().fsl_set_faces(self.h, d, side, var, np.ascontiguousarray(a, np.float64)))

    def set_cur(self, which: int):
        self._c(lib().fsl_set_cur(self.h, which))

    # --- learned closure ----------------------------------------------------------
    def closure_set_scales(self, t_ref: float, len_ref: float):
        self._c(lib().fsl_closure_set_scales(self.h, t_ref, len_ref))

    def closure_set_weights(self, params: np.ndarray):
        self._c(lib().fsl_closure_set_weights(self.h, np.ascontiguousarray(params, np.float32)))

    def closure_get_weights(self) -> np.ndarray:
        out = np.empty(CLOSURE_NPARAMS, np.float32)
        self._c(lib().fsl_closure_get_weights(self.h, out))
        return out

    def closure_judge(self, every: int, threshold: float):
        self._c(lib().fsl_closure_judge(self.h, every, threshold))

    def closure_judge_active(self, floor: float, threshold: float):
        """Rows whose dynamic SGS viscosity is at least floor * mu_L are judged
        on the SGS viscosity profile itself against `threshold`."""
        self._c(lib().fsl_closure_judge_active(self.h, floor, threshold))

    def closure_stats(self) -> ClosureStats:
        s = ClosureStats()
        self._c(lib().fsl_closure_get_stats(self.h, C.byref(s)))
        return s

    def closure_compare(self, fields: bool = False):
        """One judgement on U^n: a ClosureStats whose profile_err, cell_err,
        mu_profile_err and visc_err compare the MLP with the dynamic procedure
        (with fields=True also the padded Cs^2 arrays: (stats, cs2_mlp, cs2_dyn))."""
        st = ClosureStats()
        a = np.empty(self.padded_shape, np.float32) if fields else None
        b = np.empty(self.padded_shape, np.float32) if fields else None
        self._c(lib().fsl_closure_compare(self.h, a.ctypes.data if fields else None,
                                          b.ctypes.data if fields else None, C.byref(st)))
        return (st, a, b) if fields else st

    TUNE_STAGE_ROWS, TUNE_STAGE_SEG, TUNE_CLOSURE_POLY = 1, 2, 3

    def tune(self, key: int, value: int):
        """Launch-shape knob of the fused kernels (results do not depend on it)."""
        self._c(lib().fsl_tune(self.h, key, value))

    # --- profiling ------------------------------------------------------------------
    def profile(self, on: bool = True):
        self._c(lib().fsl_profile(self.h, 1 if on else 0))

    def profile_read(self) -> KTimes:
        t = KTimes()
        self._c(lib().fsl_profile_read(self.h, C.byref(t)))
        return t

    @property
    def stream(self) -> int:
        """cudaStream_t of the domain (for torch.cuda.ExternalStream)."""
        return lib().fsl_stream(self.h)

    # --- diagnostics ----------------------------------------------------------------
    def sums(self) -> np.ndarray:
        out = np.empty(5, np.float64)
        self._c(lib().fsl_sums(self.h, out))
        return out

    def plane_sums(self) -> np.ndarray:
        out = np.empty(8 * self.p.HIG, np.float64)
        self._c(lib().fsl_plane_sums(self.h, out))
        return out.reshape(self.p.HIG, 8)

    # --- driver files (real_bytes 4: the reference's float build, 8: FP64) -----------
    def write_backup(self, path: str, real_bytes: int = 8):
        """backup.dat as Finalize() writes it (src/finalize.c:14-35)."""
        self._c(lib().fsl_write_backup(self.h, os.fsencode(path), real_bytes))

    def read_backup(self, path: str, real_bytes: int = 8):
        """Restore state, deltaT and step from a backup.dat (src/initialize.c:133-158)."""
        self._c(lib().fsl_read_backup(self.h, os.fsencode(path), real_bytes))

    def probe_rows(self) -> np.ndarray:
        """rho and rho u at the three probe stations of src/probes.c: (3, 2, HIG)."""
        out = np.empty(6 * self.p.HIG, np.float64)
        self._c(lib().fsl_probe_rows(self.h, out))
        return out.reshape(3, 2, self.p.HIG)

    def write_probes(self, path: str, real_bytes: int = 8):
        """Append one Probes() record (src/probes.c:13-44)."""
        self._c(lib().fsl_write_probes(self.h, os.fsencode(path), real_bytes))

    def output_fields(self) -> np.ndarray:
        """Output()'s 12 values per cell (src/output.c): (DEP, HIG, LEN, 12)."""
        p = self.p
        out = np.empty(12 * p.LEN * p.HIG * p.DEP, np.float64)
        self._c(lib().fsl_output_fields(self.h, out))
        return out.reshape(p.DEP, p.HIG, p.LEN, 12)

    def write_tecplot(self, path: str):
        """The ASCII Tecplot frame Output() writes (src/output.c)."""
        self._c(lib().fsl_write_tecplot(self.h, os.fsencode(path)))

    def favre_reset(self):
        self._c(lib().fsl_favre_reset(self.h))

    def favre_accumulate(self):
        self._c(lib().fsl_favre_accumulate(self.h))

    def favre_read(self):
        """Favre-averaged u at the probe stations, (3, HIG), and the record count."""
        out = np.empty(3 * self.p.HIG, np.float64)
        n = C.c_int()
        self._c(lib().fsl_favre_read(self.h, out, C.byref(n)))
        return out.reshape(3, self.p.HIG), n.value


class Trainer:
    """Training of the learned closure on (features, dynamic Cs^2) samples
    harvested on the GPU; forward and backward run on the tensor cores."""

    def __init__(self, capacity: int, seed: int = 1):
        h = C.c_void_p()
        _check(lib().fsl_trainer_create(capacity, seed, C.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            lib().fsl_trainer_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def size(self) -> int:
        return lib().fsl_trainer_size(self.h)

    def harvest(self, domain: "Domain", stride: int = 1):
        _check(lib().fsl_trainer_harvest(self.h, domain.h, stride), domain.h)

    def samples(self, n: int | None = None):
        n = self.size if n is None else n
        X = np.empty((n, 8), np.float32)
        Y = np.empty(n, np.float32)
        _check(lib().fsl_trainer_get_samples(self.h, X, Y, n))
        return X, Y

    def set_samples(self, X: np.ndarray, Y: np.ndarray):
        X = np.ascontiguousarray(X, np.float32)
        Y = np.ascontiguousarray(Y, np.float32)
        _check(lib().fsl_trainer_set_samples(self.h, X, Y, len(Y)))

    def weights(self) -> np.ndarray:
        out = np.empty(CLOSURE_NPARAMS, np.float32)
        _check(lib().fsl_trainer_get_weights(self.h, out))
        return out

    def set_weights(self, p: np.ndarray):
        _check(lib().fsl_trainer_set_weights(self.h, np.ascontiguousarray(p, np.float32)))

    def set_loss(self, mode: int):
        """0: MSE of Cs^2; 1: squared error of mu_SGS (samples weighted by (rho |S| t_ref)^2)."""
        _check(lib().fsl_trainer_set_loss(self.h, mode))

    def gradient(self, n: int | None = None):
        n = self.size if n is None else n
        g = np.empty(CLOSURE_NPARAMS, np.float32)
        loss = C.c_double()
        _check(lib().fsl_trainer_gradient(self.h, n, g, C.byref(loss)))
        return g, loss.value

    def train(self, epochs: int, batch: int = 65536, lr: float = 1e-3) -> float:
        loss = C.c_double()
        _check(lib().fsl_trainer_train(self.h, epochs, batch, lr, C.byref(loss)))
        return loss.value


class Ensemble:
    """Independent temporal shear layers (each a :class:`Domain`) advanced
    together: chunks of steps of all members are captured into one CUDA graph
    and replayed (members on their own streams, so their kernels share the
    SMs).  Results are bit-identical to stepping each member alone."""

    def __init__(self, members):
        self.members = list(members)
        arr = (C.c_void_p * len(self.members))(*[m.h for m in self.members])
        h = C.c_void_p()
        _check(lib().fsl_ensemble_create(arr, len(self.members), C.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            lib().fsl_ensemble_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _c(self, rc):
        if rc != FSL_OK:
            raise FslError(rc, lib().fsl_ensemble_last_error(self.h).decode())

    @property
    def stream(self) -> int:
        return lib().fsl_ensemble_stream(self.h)

    def set_chunk(self, steps: int):
        self._c(lib().fsl_ensemble_set_chunk(self.h, steps))

    def step(self, n: int = 1):
        self._c(lib().fsl_ensemble_step(self.h, n))

    def sync(self):
        self._c(lib().fsl_ensemble_sync(self.h))

    def persistent(self) -> int:
        """1 when a step's stages run as one cooperative launch for all members."""
        return lib().fsl_ensemble_persistent(self.h)

    def set_barrier_limit(self, polls: int):
        """Polls a grid barrier of the persistent launch waits before giving up."""
        self._c(lib().fsl_ensemble_set_barrier_limit(self.h, polls))

    def tune(self, trial_steps: int = 5):
        """Autotune the fused-stage tile shape; returns (rows, seg, ms per step)."""
        r, s, ms = C.c_int(), C.c_int(), C.c_double()
        self._c(lib().fsl_ensemble_tune(self.h, trial_steps, C.byref(r), C.byref(s), C.byref(ms)))
        return r.value, s.value, ms.value


def tecplot_write(path: str, fields: np.ndarray):
    """Write Output()-style values, shape (DEP, HIG, LEN, 12), as the ASCII
    Tecplot file of src/output.c (host only)."""
    f = np.ascontiguousarray(fields, np.float64)
    D, H, L, _ = f.shape
    _check(lib().fsl_tecplot_write(os.fsencode(path), L, H, D, f.ravel()))


def favre_from_probes(path: str, HIG: int, real_bytes: int = 4, step_start: int = 0, step_end: int = 2**31 - 1):
    """The reference's Favre post-processor over a probes.dat file
    (favre-average-src/layer2_p.c:59-112; host only): u~ per station and row,
    (3, HIG), and the number of records averaged."""
    out = np.empty(3 * HIG, np.float64)
    n = C.c_int()
    _check(lib().fsl_favre_from_probes(os.fsencode(path), HIG, real_bytes, step_start, step_end, out, C.byref(n)))
    return out.reshape(3, HIG), n.value


def favre_profiles(path: str, HIG: int, step_start: int, step_end: int, out_dir: str) -> int:
    """The reference's post-processor (favre-average-src/layer2_p.c) on a
    float probes file: writes out_dir/probe1.dat .. probe3.dat (float sums,
    its text format); returns the number of records summed (host only)."""
    n = C.c_int()
    _check(lib().fsl_favre_profiles(os.fsencode(path), HIG, step_start, step_end, os.fsencode(out_dir),
                                    C.byref(n)))
    return n.value


# --- shear-layer statistics ----------------------------------------------------------
CLOSURE_WEIGHTS = os.path.join(HERE, "closure_weights.f32")


def closure_weights(path: str | None = None) -> np.ndarray:
    """The trained closure parameters shipped with the package (FSL_CLOSURE_NPARAMS
    little-endian float32, written by ``python -m freeshearlayer_b200.train_closure``)."""
    w = np.fromfile(path or CLOSURE_WEIGHTS, dtype="<f4")
    if w.size != CLOSURE_NPARAMS:
        raise ValueError("closure weights: expected %d float32 values, found %d" % (CLOSURE_NPARAMS, w.size))
    return w


def shear_statistics(rows: np.ndarray, cells_per_row: int, dU: float, dy: float, rho0: float = 1.0) -> dict:
    """Favre statistics of a temporal shear layer from :meth:`Domain.plane_sums`
    rows (per y row: sums of rho, rho u, rho v, rho w, rho uu, rho vv, rho ww,
    rho uv over the cells_per_row = LEN * DEP cells of the x-z plane).

    Returns the momentum thickness theta = (1 / (rho0 dU^2)) int rho_bar
    (dU/2 - u~)(u~ + dU/2) dy, the Favre mean velocity u~ and the Favre
    Reynolds stresses R_ij = {rho u_i u_j}/{rho} - u~_i u~_j per row."""
    r = np.asarray(rows, np.float64)
    rho = r[:, 0]
    u, v, w = r[:, 1] / rho, r[:, 2] / rho, r[:, 3] / rho
    R11 = r[:, 4] / rho - u * u
    R22 = r[:, 5] / rho - v * v
    R33 = r[:, 6] / rho - w * w
    R12 = r[:, 7] / rho - u * v
    rho_bar = rho / cells_per_row
    return {"theta": float(np.sum(rho_bar * (0.5 * dU - u) * (u + 0.5 * dU)) * dy / (rho0 * dU * dU)),
            "rho": rho_bar, "u": u, "R11": R11, "R22": R22, "R33": R33, "R12": R12}
