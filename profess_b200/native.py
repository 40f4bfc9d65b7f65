"""ctypes binding of the C ABI declared in ``include/profess_b200.h``.

``Engine`` mirrors the reference's density-solve entry points
(``CalculatePotentialPlus``, Source/CalPotential.f90:41, and
``ProjNormRhoMinimization``, Source/RhoOptN.f90:60) on top of the library's
slots.  Arrays cross the boundary as Fortran-ordered float64 (x fastest), the
layout the reference holds ``rho(n1,n2,n3)`` in.  Errors raise ``OfdftError``
carrying the library's status code and message.

The default library is the in-tree CUDA build; there is no CPU fallback: if
it is missing or no GPU is present, ``load_library`` raises.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_LIB = os.path.join(HERE, "_lib", "libprofess_b200.so")

KEDF_WT = 4
KEDF_WGC = 5
FP64 = 0
FP32 = 1
CONV_ENE = 0
CONV_POT = 1
CONV_BOTH = 2


class OfdftError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("ofdft error %d: %s" % (code, msg))
        self.code = code


class CellDesc(ctypes.Structure):
    _fields_ = [("n1", ctypes.c_int), ("n2", ctypes.c_int), ("n3", ctypes.c_int),
                ("lattice", ctypes.c_double * 9), ("kinetic", ctypes.c_int),
                ("lambda_", ctypes.c_double), ("mu", ctypes.c_double),
                ("alpha", ctypes.c_double), ("beta", ctypes.c_double), ("gamma", ctypes.c_double),
                ("rho0", ctypes.c_double), ("rho_s", ctypes.c_double),
                ("ion_ion_energy", ctypes.c_double), ("precision", ctypes.c_int)]


class NtnOptions(ctypes.Structure):
    _fields_ = [("max_iter", ctypes.c_int), ("conv_check", ctypes.c_int),
                ("pot_tol", ctypes.c_double), ("tole", ctypes.c_double),
                ("max_line", ctypes.c_int), ("max_ticks", ctypes.c_int)]


class NtnStats(ctypes.Structure):
    _fields_ = [("outcome", ctypes.c_int), ("iterations", ctypes.c_int), ("num_evals", ctypes.c_int),
                ("num_cg", ctypes.c_int), ("num_line", ctypes.c_int), ("history_len", ctypes.c_int),
                ("pot_norm", ctypes.c_double), ("error", ctypes.c_int), ("ticks", ctypes.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_vp = ctypes.c_void_p

# name -> argtypes (all functions return int status unless listed otherwise)
SIGNATURES = {
    "ofdft_version": [],
    "ofdft_engine_create": [ctypes.POINTER(_vp)],
    "ofdft_engine_destroy": [_vp],
    "ofdft_slot_create": [_vp, ctypes.POINTER(CellDesc), _ip],
    "ofdft_slot_destroy": [_vp, ctypes.c_int],
    "ofdft_slot_set_kernel": [_vp, ctypes.c_int, _dp, ctypes.c_int],
    "ofdft_slot_set_ion_potential": [_vp, ctypes.c_int, _dp],
    "ofdft_slot_build_wt_kernel": [_vp, ctypes.c_int],
    "ofdft_slot_build_wgc_kernel": [_vp, ctypes.c_int, ctypes.c_int, _dp, _dp, _dp, _dp],
    "ofdft_slot_build_ion_potential": [_vp, ctypes.c_int, ctypes.c_int, _dp, _ip, ctypes.c_int, _ip,
                                       _dp, _dp, _dp, _dp, _dp],
    "ofdft_calculate_potential_plus": [_vp, ctypes.c_int, _dp, ctypes.c_int, _dp, _dp],
    "ofdft_proj_norm_rho_minimization": [_vp, ctypes.c_int, _dp, _dp, ctypes.POINTER(NtnOptions),
                                         ctypes.POINTER(NtnStats)],
    "ofdft_slot_start_solve": [_vp, ctypes.c_int, _dp, ctypes.POINTER(NtnOptions)],
    "ofdft_slot_start_solve_from_slot": [_vp, ctypes.c_int, ctypes.c_int, ctypes.POINTER(NtnOptions)],
    "ofdft_slot_start_eval": [_vp, ctypes.c_int, _dp, ctypes.c_int, ctypes.c_int],
    "ofdft_engine_run": [_vp, ctypes.c_int, _ip],
    "ofdft_slot_poll": [_vp, ctypes.c_int, _ip],
    "ofdft_slot_result": [_vp, ctypes.c_int, _dp, _dp, ctypes.POINTER(NtnStats)],
    "ofdft_slot_history": [_vp, ctypes.c_int, ctypes.c_int, _dp, _dp, _dp, _ip, _ip, _ip],
    "ofdft_slot_download": [_vp, ctypes.c_int, ctypes.c_int, _dp],
}

_LIBS = {}


def load_library(path: str | None = None) -> ctypes.CDLL:
    """Load the engine library (the in-tree CUDA build by default)."""
    path = path or DEFAULT_LIB
    if path in _LIBS:
        return _LIBS[path]
    if not os.path.exists(path):
        raise OfdftError(-1, "engine library not built: %s (run python -m profess_b200.build)" % path)
    lib = ctypes.CDLL(path)
    for name, args in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = ctypes.c_int
    lib.ofdft_last_error.argtypes = []
    lib.ofdft_last_error.restype = ctypes.c_char_p
    _LIBS[path] = lib
    return lib


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_dp)


def _fortran(a, shape=None) -> np.ndarray:
    a = np.asarray(a, dtype=np.float64)
    if shape is not None and a.shape != tuple(shape):
        a = a.reshape(shape, order="F")
    return np.asfortranarray(a)


def ntn_options(max_iter=500, conv_check=CONV_ENE, pot_tol=1.0e-5, tole=1.0e-6, max_line=200, max_ticks=0):
    """RhoOptimizers defaults (Source/RhoOptimizers.f90:44-101)."""
    return NtnOptions(max_iter, conv_check, pot_tol, tole, max_line, max_ticks)


class Engine:
    """An engine holding up to 64 slots (cells) on the current GPU."""

    def __init__(self, lib: ctypes.CDLL | str | None = None):
        self.lib = lib if isinstance(lib, ctypes.CDLL) else load_library(lib)
        h = _vp()
        self._check(self.lib.ofdft_engine_create(ctypes.byref(h)))
        self.h = h
        self.shapes = {}

    def _check(self, rc):
        if rc != 0:
            raise OfdftError(rc, self.lib.ofdft_last_error().decode())

    def close(self):
        if getattr(self, "h", None):
            self.lib.ofdft_engine_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -------------------------------------------------------------- slots
    def slot_create(self, n, lattice, kinetic=KEDF_WT, lam=1.0, mu=1.0, alpha=5.0 / 6.0, beta=5.0 / 6.0,
                    gamma=2.7, rho0=0.0, rho_s=0.0, ion_ion=0.0, precision=FP64) -> int:
        """``lattice``: (3,3) bohr with lattice vector i in column i (cellReal)."""
        lat = np.asarray(lattice, float)
        d = CellDesc(int(n[0]), int(n[1]), int(n[2]), (ctypes.c_double * 9)(*lat.ravel(order="F")),
                     int(kinetic), lam, mu, alpha, beta, gamma, rho0, rho_s, ion_ion, int(precision))
        s = ctypes.c_int()
        self._check(self.lib.ofdft_slot_create(self.h, ctypes.byref(d), ctypes.byref(s)))
        self.shapes[s.value] = tuple(int(x) for x in n)
        return s.value

    def slot_destroy(self, slot):
        self._check(self.lib.ofdft_slot_destroy(self.h, slot))
        self.shapes.pop(slot, None)

    def set_kernel(self, slot, kernel):
        """keKernel as (nplanes, k1, n2, n3) or (k1, n2, n3)."""
        k = np.asarray(kernel, float)
        if k.ndim == 3:
            k = k[None]
        flat = np.concatenate([np.asfortranarray(p).ravel(order="F") for p in k])
        self._check(self.lib.ofdft_slot_set_kernel(self.h, slot, _ptr(flat), k.shape[0]))

    def set_ion_potential(self, slot, vion):
        v = _fortran(vion, self.shapes[slot])
        self._check(self.lib.ofdft_slot_set_ion_potential(self.h, slot, _ptr(v)))

    # -------------------------------------------------------------- drop-in
    def calculate_potential_plus(self, slot, rho, opt_sqrt=True, want_energy=True):
        """CalculatePotentialPlus(rho, optSqrt, potential[, eTable]) for one spin."""
        shp = self.shapes[slot]
        r = _fortran(rho, shp)
        pot = np.zeros(shp, order="F")
        et = np.zeros(9)
        self._check(self.lib.ofdft_calculate_potential_plus(self.h, slot, _ptr(r), int(bool(opt_sqrt)),
                                                            _ptr(pot), _ptr(et) if want_energy else None))
        return pot, (et if want_energy else None)

    def proj_norm_rho_minimization(self, slot, rho, opts: NtnOptions | None = None):
        """ProjNormRhoMinimization(energy, dir_type=1): returns (rho, energy[9], stats)."""
        shp = self.shapes[slot]
        r = _fortran(rho, shp).copy(order="F")
        e = np.zeros(9)
        st = NtnStats()
        o = opts or ntn_options()
        self._check(self.lib.ofdft_proj_norm_rho_minimization(self.h, slot, _ptr(r), _ptr(e),
                                                              ctypes.byref(o), ctypes.byref(st)))
        return r, e, st.as_dict()

    # -------------------------------------------------------------- async
    def start_solve(self, slot, rho, opts: NtnOptions | None = None):
        r = _fortran(rho, self.shapes[slot])
        o = opts or ntn_options()
        self._check(self.lib.ofdft_slot_start_solve(self.h, slot, _ptr(r), ctypes.byref(o)))

    def start_solve_from_slot(self, slot, src, opts: NtnOptions | None = None):
        o = opts or ntn_options()
        self._check(self.lib.ofdft_slot_start_solve_from_slot(self.h, slot, src, ctypes.byref(o)))

    def start_eval(self, slot, rho, opt_sqrt=True, want_energy=True):
        r = _fortran(rho, self.shapes[slot])
        self._check(self.lib.ofdft_slot_start_eval(self.h, slot, _ptr(r), int(bool(opt_sqrt)),
                                                   int(bool(want_energy))))

    def run(self, ticks=1):
        n = ctypes.c_int()
        self._check(self.lib.ofdft_engine_run(self.h, int(ticks), ctypes.byref(n)))
        return n.value

    def poll(self, slot) -> bool:
        f = ctypes.c_int()
        self._check(self.lib.ofdft_slot_poll(self.h, slot, ctypes.byref(f)))
        return bool(f.value)

    def result(self, slot, want_rho=True):
        shp = self.shapes[slot]
        r = np.zeros(shp, order="F") if want_rho else None
        e = np.zeros(9)
        st = NtnStats()
        self._check(self.lib.ofdft_slot_result(self.h, slot, _ptr(r) if want_rho else None, _ptr(e),
                                               ctypes.byref(st)))
        return r, e, st.as_dict()

    def history(self, slot, max_entries=256):
        e = np.zeros(max_entries)
        p = np.zeros(max_entries)
        t = np.zeros(max_entries)
        ncg = np.zeros(max_entries, dtype=np.int32)
        nl = np.zeros(max_entries, dtype=np.int32)
        n = ctypes.c_int()
        self._check(self.lib.ofdft_slot_history(self.h, slot, max_entries, _ptr(e), _ptr(p), _ptr(t),
                                                ncg.ctypes.data_as(_ip), nl.ctypes.data_as(_ip),
                                                ctypes.byref(n)))
        m = n.value
        return [dict(energy=e[i], pot_norm=p[i], theta=t[i], ncg=int(ncg[i]), nline=int(nl[i])) for i in range(m)]

    def download(self, slot, which=0):
        out = np.zeros(self.shapes[slot], order="F")
        self._check(self.lib.ofdft_slot_download(self.h, slot, which, _ptr(out)))
        return out
