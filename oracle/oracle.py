"""ctypes access to the two CPU oracles.  TEST INFRASTRUCTURE ONLY.

* ``Oracle``   -- this project's C restatement (oracle/fsl_oracle.c, liboracle.so).
* ``RefOracle`` -- the reference's own serial solver compiled in place with the
  FP64 + zero-fill patch (oracle/_ref/libfslref.so, built by ``make ref``).

Only tests, the smoke check and the CPU-baseline leg of bench.py import this
module; the product never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_ORACLE = os.path.join(HERE, "liboracle.so")
LIB_REF = os.path.join(HERE, "_ref", "libfslref.so")

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")

# layer2.ini line order (src/initialize.c:25-58)
INI_KEYS = ["LEN", "HIG", "DEP", "deltaX", "deltaY", "deltaZ", "deltaT", "Answer",
            "numstep", "mu_L", "Pr_L", "Pr_T", "Cs", "BL_HIG", "Ua", "Va", "Wa",
            "Ns_min", "Nst", "f_step", "nStages", "maxCoNum"]
INT_KEYS = {"LEN", "HIG", "DEP", "Answer", "numstep", "BL_HIG", "Ns_min", "Nst",
            "f_step", "nStages"}


class OrcParams(C.Structure):
    _fields_ = [("LEN", C.c_int), ("HIG", C.c_int), ("DEP", C.c_int),
                ("deltaX", C.c_double), ("deltaY", C.c_double), ("deltaZ", C.c_double),
                ("deltaT", C.c_double), ("Answer", C.c_int), ("numstep", C.c_int),
                ("mu_L", C.c_double), ("Pr_L", C.c_double), ("Pr_T", C.c_double),
                ("Cs", C.c_double), ("BL_HIG", C.c_int), ("Ua", C.c_double),
                ("Va", C.c_double), ("Wa", C.c_double), ("Ns_min", C.c_int),
                ("Nst", C.c_int), ("f_step", C.c_int), ("nStages", C.c_int),
                ("maxCoNum", C.c_double), ("setup", C.c_int), ("cfl_mode", C.c_int),
                ("seed_X", C.c_double), ("recon", C.c_int), ("sgs", C.c_int)]


def build(ref: bool = False) -> None:
    """Build liboracle.so (and, with ref=True and the reference sources present
    -- FSL_REF_SRC, or a `reference` checkout beside the repository -- _ref)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    if ref:
        subprocess.run(["make", "-s", "-C", HERE, "ref-if-present"], check=True)


def ref_available() -> bool:
    return os.path.exists(LIB_REF)


def default_params(**kw) -> dict:
    """The reference's shipped layer2.ini physics with nStages=3 and a small grid."""
    p = dict(LEN=16, HIG=8, DEP=8, deltaX=1.6666667, deltaY=1.0, deltaZ=1.5,
             deltaT=0.0007, Answer=0, numstep=10, mu_L=0.253358, Pr_L=0.72, Pr_T=0.8,
             Cs=0.01, BL_HIG=2, Ua=35.0, Va=35.0, Wa=35.0, Ns_min=10, Nst=50,
             f_step=50, nStages=3, maxCoNum=0.1, setup=0, cfl_mode=0,
             seed_X=0.317391239817)
    p.update(kw)
    return p


def ini_text(p: dict) -> str:
    lines = []
    for key in INI_KEYS:
        v = p[key]
        lines.append(("%d" % int(v)) if key in INT_KEYS else ("%.17g" % float(v)))
    return "\n".join(lines) + "\n"


def padded_shape(p: dict):
    return (p["LEN"] + 2, p["HIG"] + 2, p["DEP"] + 2)


def face_shape(p: dict, d: int):
    return (p["LEN"] + (d == 0), p["HIG"] + (d == 1), p["DEP"] + (d == 2))


def _setup_common(lib):
    lib_cells = [C.c_void_p, C.c_int, C.c_int, _dp, C.c_int]
    return lib_cells


class Oracle:
    """This project's CPU restatement (one instance = one domain)."""

    _lib = None

    @classmethod
    def lib(cls):
        if cls._lib is None:
            if not os.path.exists(LIB_ORACLE):
                build()
            lib = C.CDLL(LIB_ORACLE)
            lib.orc_create.restype = C.c_void_p
            lib.orc_create.argtypes = [C.POINTER(OrcParams)]
            lib.orc_destroy.argtypes = [C.c_void_p]
            lib.orc_cells.argtypes = [C.c_void_p, C.c_int, C.c_int, _dp, C.c_int]
            lib.orc_faces.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, _dp, C.c_int]
            lib.orc_state.argtypes = [C.c_void_p, _dp, C.c_int]
            lib.orc_set_cur.argtypes = [C.c_void_p, C.c_int]
            lib.orc_get_cur.argtypes = [C.c_void_p]
            lib.orc_get_scalars.argtypes = [C.c_void_p, _dp]
            lib.orc_set_dt.argtypes = [C.c_void_p, C.c_double]
            lib.orc_set_disturbance.argtypes = [C.c_void_p, C.c_uint, C.c_uint, C.c_double,
                                                C.c_double, C.c_double]
            for name in ["orc_ghost_bc", "orc_reconstruct", "orc_interface_bc",
                         "orc_dynamic_smagorinsky", "orc_fluxes_only", "orc_fluxes",
                         "orc_disturb"]:
                getattr(lib, name).argtypes = [C.c_void_p]
            lib.orc_evolution.argtypes = [C.c_void_p, C.c_int, C.c_int]
            lib.orc_check_courant.argtypes = [C.c_void_p]
            lib.orc_check_courant.restype = C.c_double
            lib.orc_step.argtypes = [C.c_void_p, C.c_int]
            lib.orc_step_ref_sgs.argtypes = [C.c_void_p, C.c_int]
            lib.orc_filter.argtypes = [C.POINTER(OrcParams), _dp, _dp]
            lib.orc_minmod.argtypes = [C.c_double, C.c_double]
            lib.orc_minmod.restype = C.c_double
            lib.orc_random.argtypes = [C.c_double]
            lib.orc_random.restype = C.c_double
            lib.orc_temporal_state.argtypes = [C.POINTER(OrcParams), C.c_double, C.c_double,
                                               C.c_double, C.c_ulonglong, _dp,
                                               C.POINTER(C.c_double)]
            lib.orc_sums.argtypes = [C.c_void_p, _dp]
            lib.orc_plane_sums.argtypes = [C.c_void_p, _dp]
            lib.orc_output_fields.argtypes = [C.c_void_p, _dp]
            cls._lib = lib
        return cls._lib

    def __init__(self, p: dict):
        self.p = dict(p)
        self.cp = OrcParams(**{k: self.p.get(k, 0) for k, _ in OrcParams._fields_})
        self.h = self.lib().orc_create(C.byref(self.cp))
        if not self.h:
            raise MemoryError("orc_create failed")

    def __del__(self):
        if getattr(self, "h", None):
            self.lib().orc_destroy(self.h)
            self.h = None

    # --- arrays ---------------------------------------------------------
    def cells(self, which: int, var: int = 0) -> np.ndarray:
        a = np.empty(padded_shape(self.p), np.float64)
        self.lib().orc_cells(self.h, which, var, a, 0)
        return a

    def set_cells(self, which: int, var: int, a: np.ndarray) -> None:
        self.lib().orc_cells(self.h, which, var, np.ascontiguousarray(a, np.float64), 1)

    def faces(self, d: int, side: int, var: int) -> np.ndarray:
        a = np.empty(face_shape(self.p, d), np.float64)
        self.lib().orc_faces(self.h, d, side, var, a, 0)
        return a

    def set_faces(self, d: int, side: int, var: int, a: np.ndarray) -> None:
        self.lib().orc_faces(self.h, d, side, var, np.ascontiguousarray(a, np.float64), 1)

    def state(self) -> np.ndarray:
        a = np.empty(self.p["LEN"] * self.p["HIG"] * 5 * self.p["DEP"], np.float64)
        self.lib().orc_state(self.h, a, 0)
        return a

    def set_state(self, a: np.ndarray) -> None:
        self.lib().orc_state(self.h, np.ascontiguousarray(a, np.float64).ravel(), 1)

    def scalars(self) -> np.ndarray:
        a = np.empty(17, np.float64)
        self.lib().orc_get_scalars(self.h, a)
        return a

    def set_dt(self, dt: float) -> None:
        self.lib().orc_set_dt(self.h, dt)

    def set_disturbance(self, kmin, kmax, ud, vd, wd) -> None:
        self.lib().orc_set_disturbance(self.h, kmin, kmax, ud, vd, wd)

    def set_cur(self, which: int) -> None:
        self.lib().orc_set_cur(self.h, which)

    # --- phases ---------------------------------------------------------
    def ghost(self): self.lib().orc_ghost_bc(self.h)
    def recon(self): self.lib().orc_reconstruct(self.h)
    def ifbc(self): self.lib().orc_interface_bc(self.h)
    def dynsmag(self): self.lib().orc_dynamic_smagorinsky(self.h)
    def fluxes_only(self): self.lib().orc_fluxes_only(self.h)
    def fluxes(self): self.lib().orc_fluxes(self.h)
    def evolution(self, nst, stage): self.lib().orc_evolution(self.h, nst, stage)
    def check_courant(self) -> float: return self.lib().orc_check_courant(self.h)
    def disturb(self): self.lib().orc_disturb(self.h)
    def step(self, n=1): self.lib().orc_step(self.h, n)
    def step_ref_sgs(self, n=1): self.lib().orc_step_ref_sgs(self.h, n)

    def sums(self) -> np.ndarray:
        a = np.empty(5, np.float64)
        self.lib().orc_sums(self.h, a)
        return a

    def plane_sums(self) -> np.ndarray:
        a = np.empty(8 * self.p["HIG"], np.float64)
        self.lib().orc_plane_sums(self.h, a)
        return a.reshape(self.p["HIG"], 8)

    def output_fields(self) -> np.ndarray:
        """Output()'s 12 values per cell (src/output.c), (DEP, HIG, LEN, 12)."""
        p = self.p
        a = np.empty(12 * p["LEN"] * p["HIG"] * p["DEP"], np.float64)
        self.lib().orc_output_fields(self.h, a)
        return a.reshape(p["DEP"], p["HIG"], p["LEN"], 12)

    # --- standalone -----------------------------------------------------
    @classmethod
    def filter(cls, p: dict, a: np.ndarray) -> np.ndarray:
        cp = OrcParams(**{k: p.get(k, 0) for k, _ in OrcParams._fields_})
        out = np.empty_like(a)
        cls.lib().orc_filter(C.byref(cp), np.ascontiguousarray(a), out)
        return out

    @classmethod
    def temporal_state(cls, p: dict, Mc: float, delta_w0: float = 1.0, amp: float = 1e-3,
                       seed: int = 20251203):
        cp = OrcParams(**{k: p.get(k, 0) for k, _ in OrcParams._fields_})
        out = np.empty(p["LEN"] * p["HIG"] * 5 * p["DEP"], np.float64)
        dU = C.c_double()
        rc = cls.lib().orc_temporal_state(C.byref(cp), Mc, delta_w0, amp, seed, out, C.byref(dU))
        if rc != 0:
            raise RuntimeError("orc_temporal_state failed")
        return out, dU.value


class RefOracle:
    """The reference's own serial solver (FP64 + zero-fill), one per process.

    The reference keeps its whole state in globals, so every instance shares
    it; ``__init__`` re-runs Initialize() on a generated layer2.ini.
    """

    _lib = None

    @classmethod
    def lib(cls):
        if cls._lib is None:
            if not os.path.exists(LIB_REF):
                raise FileNotFoundError(LIB_REF)
            lib = C.CDLL(LIB_REF)
            lib.refh_init.argtypes = [C.c_char_p]
            lib.refh_seed.argtypes = [C.c_double]
            lib.refh_step.argtypes = [C.c_int]
            lib.refh_evolution.argtypes = [C.c_int, C.c_int]
            lib.refh_cells.argtypes = [C.c_int, C.c_int, _dp, C.c_int]
            lib.refh_faces.argtypes = [C.c_int, C.c_int, C.c_int, _dp, C.c_int]
            lib.refh_set_cur.argtypes = [C.c_int]
            lib.refh_get_scalars.argtypes = [_dp]
            lib.refh_set_dt.argtypes = [C.c_double]
            lib.refh_set_disturbance.argtypes = [C.c_uint, C.c_uint, C.c_double, C.c_double,
                                                 C.c_double]
            lib.refh_filter.argtypes = [_dp, _dp]
            lib.refh_minmod.argtypes = [C.c_double, C.c_double]
            lib.refh_minmod.restype = C.c_double
            lib.refh_random.argtypes = [C.c_double]
            lib.refh_random.restype = C.c_double
            lib.refh_output.argtypes = [C.c_char_p]
            lib.refh_set_static.argtypes = [C.c_int]
            cls._lib = lib
        return cls._lib

    def __init__(self, p: dict):
        if p.get("setup", 0) != 0:
            raise ValueError("the reference implements only the spatial setup")
        self.p = dict(p)
        with tempfile.TemporaryDirectory() as d:
            with open(os.path.join(d, "layer2.ini"), "w") as f:
                f.write(ini_text(p))
            rc = self.lib().refh_init(d.encode())
        if rc != 0:
            raise RuntimeError("refh_init failed: %d" % rc)
        self.lib().refh_seed(p["seed_X"])
        # the SGS model: the dynamic procedure (src/def.h:47) or, with
        # sgs = 2, the static Smagorinsky branch of src/fluxes.c
        self.lib().refh_set_static(1 if p.get("sgs", 0) == 2 else 0)

    def cells(self, which: int, var: int = 0) -> np.ndarray:
        a = np.empty(padded_shape(self.p), np.float64)
        self.lib().refh_cells(which, var, a, 0)
        return a

    def set_cells(self, which: int, var: int, a: np.ndarray) -> None:
        self.lib().refh_cells(which, var, np.ascontiguousarray(a, np.float64), 1)

    def faces(self, d: int, side: int, var: int) -> np.ndarray:
        a = np.empty(face_shape(self.p, d), np.float64)
        self.lib().refh_faces(d, side, var, a, 0)
        return a

    def set_faces(self, d: int, side: int, var: int, a: np.ndarray) -> None:
        self.lib().refh_faces(d, side, var, np.ascontiguousarray(a, np.float64), 1)

    def state(self) -> np.ndarray:
        L, H, D = self.p["LEN"], self.p["HIG"], self.p["DEP"]
        out = np.empty((L, H, 5, D))
        for v in range(5):
            out[:, :, v, :] = self.cells(0, v)[1:L + 1, 1:H + 1, 1:D + 1]
        return out.ravel()

    def set_state(self, a: np.ndarray) -> None:
        L, H, D = self.p["LEN"], self.p["HIG"], self.p["DEP"]
        a = np.asarray(a, np.float64).reshape(L, H, 5, D)
        for v in range(5):
            c = self.cells(0, v)
            c[1:L + 1, 1:H + 1, 1:D + 1] = a[:, :, v, :]
            self.set_cells(0, v, c)

    def scalars(self) -> np.ndarray:
        a = np.empty(16, np.float64)
        self.lib().refh_get_scalars(a)
        return a

    def set_dt(self, dt): self.lib().refh_set_dt(dt)
    def set_disturbance(self, kmin, kmax, ud, vd, wd):
        self.lib().refh_set_disturbance(kmin, kmax, ud, vd, wd)
    def set_cur(self, which): self.lib().refh_set_cur(which)
    def ghost(self): self.lib().refh_ghost()
    def recon(self): self.lib().refh_recon()
    def ifbc(self): self.lib().refh_ifbc()
    def dynsmag(self): self.lib().refh_dynsmag()
    def fluxes(self): self.lib().refh_fluxes()
    def fluxes_static(self): self.lib().refh_fluxes_static()
    def evolution(self, nst, stage): self.lib().refh_evolution(nst, stage)
    def check_courant(self): self.lib().refh_checkco()
    def output(self, dir: str) -> int: return self.lib().refh_output(os.fsencode(dir))
    def disturb(self): self.lib().refh_disturb()
    def step(self, n=1): self.lib().refh_step(n)

    def filter(self, a: np.ndarray) -> np.ndarray:
        out = np.empty_like(a)
        self.lib().refh_filter(np.ascontiguousarray(a), out)
        return out


def spatial_initial_state(p: dict) -> np.ndarray:
    """The reference's fresh-start initial condition, src/initialize.c:159-187,
    in the backup.dat layout (for i, for j: DEP values of U1..U5)."""
    L, H, D = p["LEN"], p["HIG"], p["DEP"]
    s = np.empty((L, H, 5, D))
    P, R = 100000.0, 1.0
    for j in range(1, H + 1):
        U = 76.4 if j <= H // 2 else 200.0
        s[:, j - 1, 0, :] = R
        s[:, j - 1, 1, :] = R * U
        s[:, j - 1, 2, :] = 0.0
        s[:, j - 1, 3, :] = 0.0
        s[:, j - 1, 4, :] = P / 0.4 + 0.5 * R * (U * U)
    return s.ravel()
