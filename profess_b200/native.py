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
# The in-tree CUDA build; PROFESS_B200_LIB names another build of the same ABI.
DEFAULT_LIB = os.environ.get("PROFESS_B200_LIB") or os.path.join(HERE, "_lib", "libprofess_b200.so")

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
                ("max_line", ctypes.c_int), ("max_ticks", ctypes.c_int), ("stall_line", ctypes.c_int)]


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
    "ofdft_slot_set_ion_ion_energy": [_vp, ctypes.c_int, ctypes.c_double],
    "ofdft_slot_hold_density": [_vp, ctypes.c_int],
    "ofdft_slot_copy_tables": [_vp, ctypes.c_int, ctypes.c_int],
    "ofdft_engine_capture_stats": [_vp, ctypes.POINTER(ctypes.c_longlong), _dp],
    "ofdft_slot_ewald": [_vp, ctypes.c_int, _dp, _dp],
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
    "ofdft_slot_cancel": [_vp, ctypes.c_int],
    "ofdft_slot_result": [_vp, ctypes.c_int, _dp, _dp, ctypes.POINTER(NtnStats)],
    "ofdft_slot_history": [_vp, ctypes.c_int, ctypes.c_int, _dp, _dp, _dp, _ip, _ip, _ip],
    "ofdft_slot_download": [_vp, ctypes.c_int, ctypes.c_int, _dp],
    "ofdft_slot_forces": [_vp, ctypes.c_int, _dp, ctypes.c_int, _dp],
    "ofdft_slot_stress": [_vp, ctypes.c_int, _dp, ctypes.c_int, _dp, _dp],
    "ofdft_slot_set_lattice": [_vp, ctypes.c_int, _dp, ctypes.c_double, ctypes.c_double],
    "ofdft_engine_tune": [_vp, ctypes.c_int, ctypes.c_int, _dp, _dp, _ip],
    "ofdft_slot_set_shape": [_vp, ctypes.c_int, _ip],
    "ofdft_slot_shape": [_vp, ctypes.c_int, _ip],
    "ofdft_slot_rescale_input": [_vp, ctypes.c_int, ctypes.c_double],
    "ofdft_slot_set_input": [_vp, ctypes.c_int, _dp],
    "ofdft_slot_footprint": [ctypes.POINTER(CellDesc), ctypes.POINTER(ctypes.c_ulonglong)],
    "ofdft_engine_stream": [_vp, ctypes.POINTER(_vp)],
    "ofdft_engine_counters": [_vp, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_longlong)],
    "ofdft_engine_time_eval": [_vp, ctypes.c_int, _dp],
    "ofdft_ewald": [_dp, ctypes.c_int, _dp, _dp, _dp, _dp],
    "ofdft_dcsrch": [_vp, _dp, ctypes.c_double, ctypes.c_double, ctypes.c_int],
    "ofdft_grid_size": [ctypes.c_double, _dp, _ip],
    "ofdft_wgc_radial_tables": [ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int, _dp, _dp, _dp,
                                _dp, _ip],
}

_LIBS = {}


def ewald(lib, lattice, frac, charges, want_forces=False):
    """Ewald ion-ion energy (Ha) and forces of point charges (host)."""
    lat = np.ascontiguousarray(np.asarray(lattice, float).ravel(order="F"))
    fr = np.ascontiguousarray(frac, dtype=np.float64).reshape(-1, 3)
    z = np.ascontiguousarray(charges, dtype=np.float64)
    e = np.zeros(1)
    f = np.zeros_like(fr) if want_forces else None
    rc = lib.ofdft_ewald(_ptr(lat), fr.shape[0], _ptr(fr), _ptr(z), _ptr(e), _ptr(f) if want_forces else None)
    if rc:
        raise OfdftError(rc, lib.ofdft_last_error().decode())
    return float(e[0]), f


class LineSearchRecord(ctypes.Structure):
    """ofdft_line_search: Dcsrch's saved state."""
    _fields_ = [(n, ctypes.c_double) for n in ("ftol", "gtol", "xtol", "stpmin", "stpmax")] + \
               [("brackt", ctypes.c_int), ("stage", ctypes.c_int)] + \
               [(n, ctypes.c_double) for n in ("ginit", "gtest", "gx", "gy", "finit", "fx", "fy", "stx", "sty",
                                               "stmin", "stmax", "width", "width1")]


LS_START, LS_FG, LS_CONV, LS_WARN, LS_ERROR = range(5)


class Dcsrch:
    """The library's More-Thuente search (ofdft_dcsrch) for host optimisers:
    step(stp, f, g, task) -> (stp, task), task LS_START first, then LS_FG while
    it asks for a point."""

    def __init__(self, lib, ftol, gtol, xtol, stpmin, stpmax):
        self.lib = lib
        self.rec = LineSearchRecord(ftol=ftol, gtol=gtol, xtol=xtol, stpmin=stpmin, stpmax=stpmax)

    def step(self, stp, f, g, task):
        s = ctypes.c_double(stp)
        out = self.lib.ofdft_dcsrch(ctypes.byref(self.rec), ctypes.byref(s), float(f), float(g), int(task))
        if out < 0:
            raise OfdftError(-out, self.lib.ofdft_last_error().decode())
        return s.value, out


def slot_footprint(lib, n, kinetic, alpha, beta, precision) -> int:
    """Device bytes of one slot (upper bound), for admission control."""
    d = CellDesc(int(n[0]), int(n[1]), int(n[2]), (ctypes.c_double * 9)(*([1.0] * 9)), int(kinetic), 1.0, 1.0,
                 alpha, beta, 2.7, 0.0, 0.0, 0.0, int(precision))
    b = ctypes.c_ulonglong()
    rc = lib.ofdft_slot_footprint(ctypes.byref(d), ctypes.byref(b))
    if rc:
        raise OfdftError(rc, lib.ofdft_last_error().decode())
    return int(b.value)


def grid_size(lib, ecut_ha, lattice):
    """SizeSystem: 7-smooth grid for the cutoff (Ha)."""
    lat = np.ascontiguousarray(np.asarray(lattice, float).ravel(order="F"))
    n = np.zeros(3, dtype=np.int32)
    rc = lib.ofdft_grid_size(float(ecut_ha), _ptr(lat), n.ctypes.data_as(_ip))
    if rc:
        raise OfdftError(rc, lib.ofdft_last_error().decode())
    return tuple(int(x) for x in n)


def wgc_radial_tables(lib, alpha, beta, gamma):
    """(eta, w, eta w', eta^2 w'') of the WGC kernel ODE, integrated by the library."""
    n = ctypes.c_int()
    lib.ofdft_wgc_radial_tables(alpha, beta, gamma, 0, None, None, None, None, ctypes.byref(n))
    arrs = [np.zeros(n.value) for _ in range(4)]
    rc = lib.ofdft_wgc_radial_tables(alpha, beta, gamma, n.value, *[_ptr(a) for a in arrs], ctypes.byref(n))
    if rc:
        raise OfdftError(rc, lib.ofdft_last_error().decode())
    return tuple(arrs)


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


def ntn_options(max_iter=500, conv_check=CONV_ENE, pot_tol=1.0e-5, tole=1.0e-6, max_line=200, max_ticks=0,
                stall_line=0):
    """RhoOptimizers defaults (Source/RhoOptimizers.f90:44-101); stall_line > 0
    stops at the line-search precision floor (mixed-precision FP32 phase)."""
    return NtnOptions(max_iter, conv_check, pot_tol, tole, max_line, max_ticks, stall_line)


class Engine:
    """An engine holding up to 256 slots (cells) on the current GPU."""

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

    def build_wt_kernel(self, slot):
        """FillWT on the device (needs rho0 in the slot description)."""
        self._check(self.lib.ofdft_slot_build_wt_kernel(self.h, slot))

    def build_wgc_kernel(self, slot, tables=None):
        """WGC kernel planes on the device; tables = (eta, w, eta w', eta^2 w'')
        or None for the library's own ODE integration."""
        if tables is None:
            self._check(self.lib.ofdft_slot_build_wgc_kernel(self.h, slot, 0, None, None, None, None))
            return
        t = [np.ascontiguousarray(x, dtype=np.float64) for x in tables]
        self._check(self.lib.ofdft_slot_build_wgc_kernel(self.h, slot, len(t[0]), _ptr(t[0]), _ptr(t[1]),
                                                         _ptr(t[2]), _ptr(t[3])))

    def build_ion_potential(self, slot, frac, species_of_ion, species):
        """Ion-electron potential by the B-spline method on the device.

        ``species``: sequence of objects with charge, max_g (bohr^-1),
        pot_values (Ha bohr^3), vqs and pot_dd arrays (ReadPseudo's tables)."""
        fr = np.ascontiguousarray(frac, dtype=np.float64).reshape(-1, 3)
        sp = np.ascontiguousarray(species_of_ion, dtype=np.int32)
        npts = np.array([len(x.pot_values) for x in species], dtype=np.int32)
        maxg = np.array([x.max_g for x in species], dtype=np.float64)
        chg = np.array([float(x.charge) for x in species], dtype=np.float64)
        pv = np.ascontiguousarray(np.concatenate([x.pot_values for x in species]), dtype=np.float64)
        vq = np.ascontiguousarray(np.concatenate([x.vqs for x in species]), dtype=np.float64)
        pd = np.ascontiguousarray(np.concatenate([x.pot_dd for x in species]), dtype=np.float64)
        self._check(self.lib.ofdft_slot_build_ion_potential(
            self.h, slot, fr.shape[0], _ptr(fr), sp.ctypes.data_as(_ip), len(species), npts.ctypes.data_as(_ip),
            _ptr(maxg), _ptr(chg), _ptr(pv), _ptr(vq), _ptr(pd)))

    def forces(self, slot, nion, rho=None, include_ewald=True):
        """Ion forces (nion, 3) in Ha/bohr on rho (or the slot's solved density)."""
        out = np.zeros((nion, 3))
        r = _fortran(rho, self.shapes[slot]) if rho is not None else None
        self._check(self.lib.ofdft_slot_forces(self.h, slot, _ptr(r) if r is not None else None,
                                               int(bool(include_ewald)), _ptr(out)))
        return out

    def tune(self, slot, iters=5):
        """Autotune the launch shape of the slot's kind of cell (it needs a
        resident input density, set_input).  Returns a dict with the median
        evaluation time before and after (ms) and the chosen shape."""
        t0, t1 = np.zeros(1), np.zeros(1)
        shp = np.zeros(4, dtype=np.int32)
        self._check(self.lib.ofdft_engine_tune(self.h, slot, int(iters), _ptr(t0), _ptr(t1),
                                               shp.ctypes.data_as(_ip)))
        return {"ms_default": float(t0[0]), "ms_tuned": float(t1[0]), "shape": self._shape_dict(shp)}

    SHAPE_KEYS = ("x_radix_cap", "xfwd_row_pairs", "xinv_row_pairs", "yz_threads")

    def _shape_dict(self, v):
        return dict(zip(self.SHAPE_KEYS, (int(x) for x in v)))

    def shape(self, slot):
        """The slot's launch shape (as tune reports it)."""
        shp = np.zeros(4, dtype=np.int32)
        self._check(self.lib.ofdft_slot_shape(self.h, slot, shp.ctypes.data_as(_ip)))
        return self._shape_dict(shp)

    def set_shape(self, slot, x_radix_cap=0, xfwd_row_pairs=1, xinv_row_pairs=1, yz_threads=0):
        """Pin the slot's launch shape (as tune reports it)."""
        v = np.array([x_radix_cap, xfwd_row_pairs, xinv_row_pairs, yz_threads], dtype=np.int32)
        self._check(self.lib.ofdft_slot_set_shape(self.h, slot, v.ctypes.data_as(_ip)))

    def set_lattice(self, slot, lattice, rho0, rho_s=None):
        """New lattice (3x3, columns are the lattice vectors, bohr) for the slot."""
        lat = np.ascontiguousarray(np.asarray(lattice, float).ravel(order="F"))
        self._check(self.lib.ofdft_slot_set_lattice(self.h, slot, _ptr(lat), float(rho0),
                                                    float(rho0 if rho_s is None else rho_s)))

    def rescale_input(self, slot, num_electrons):
        """RescaleDensity of the held input density to num_electrons."""
        self._check(self.lib.ofdft_slot_rescale_input(self.h, slot, float(num_electrons)))

    STRESS_TERMS = ("TF", "vW", "nonlocal", "Hartree", "LDA", "ion-electron", "Ewald")

    def stress(self, slot, rho=None, include_ewald=True, terms=False):
        """Stress tensor (3, 3) in Ha/bohr^3 of rho (or the slot's solved
        density); with terms, also a dict of its seven parts."""
        out = np.zeros((3, 3))
        parts = np.zeros((7, 3, 3)) if terms else None
        r = _fortran(rho, self.shapes[slot]) if rho is not None else None
        self._check(self.lib.ofdft_slot_stress(self.h, slot, _ptr(r) if r is not None else None,
                                               int(bool(include_ewald)), _ptr(out),
                                               _ptr(parts) if terms else None))
        if terms:
            return out, dict(zip(self.STRESS_TERMS, parts))
        return out

    def ewald(self, slot, nion, want_forces=True):
        """Device Ewald energy (Ha) and forces (nion, 3) of the slot's ions; the
        energy also becomes the slot's ion-ion energy."""
        e = np.zeros(1)
        f = np.zeros((nion, 3)) if want_forces else None
        self._check(self.lib.ofdft_slot_ewald(self.h, slot, _ptr(e), _ptr(f) if want_forces else None))
        return float(e[0]), f

    def copy_tables(self, slot, src):
        """Kernel planes, ion potential and ion-ion energy of slot src, converted into slot."""
        self._check(self.lib.ofdft_slot_copy_tables(self.h, slot, src))

    def hold_density(self, slot):
        """Keep the slot's solved density as its resident input (start_solve(slot) resumes from it)."""
        self._check(self.lib.ofdft_slot_hold_density(self.h, slot))

    def set_ion_ion_energy(self, slot, energy):
        """The Ewald energy (Ha) reported in the slot's energies, after the ions moved."""
        self._check(self.lib.ofdft_slot_set_ion_ion_energy(self.h, slot, float(energy)))

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
    def start_solve(self, slot, rho=None, opts: NtnOptions | None = None):
        """Start a solve from host rho, or from the resident input when rho is None."""
        o = opts or ntn_options()
        if rho is None:
            self._check(self.lib.ofdft_slot_start_solve(self.h, slot, None, ctypes.byref(o)))
            return
        r = _fortran(rho, self.shapes[slot])
        self._check(self.lib.ofdft_slot_start_solve(self.h, slot, _ptr(r), ctypes.byref(o)))

    def set_input(self, slot, rho):
        r = _fortran(rho, self.shapes[slot])
        self._check(self.lib.ofdft_slot_set_input(self.h, slot, _ptr(r)))

    def stream(self) -> int:
        p = _vp()
        self._check(self.lib.ofdft_engine_stream(self.h, ctypes.byref(p)))
        return p.value or 0

    def counters(self):
        a, b = ctypes.c_longlong(), ctypes.c_longlong()
        self._check(self.lib.ofdft_engine_counters(self.h, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def capture_stats(self):
        """(graphs captured, host ms spent capturing them)."""
        n = ctypes.c_longlong()
        ms = np.zeros(1)
        self._check(self.lib.ofdft_engine_capture_stats(self.h, ctypes.byref(n), _ptr(ms)))
        return n.value, float(ms[0])

    def time_eval(self, iters=10) -> float:
        ms = np.zeros(1)
        self._check(self.lib.ofdft_engine_time_eval(self.h, int(iters), _ptr(ms)))
        return float(ms[0])

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

    def cancel(self, slot):
        """Stop the slot's running solve or evaluation; the slot goes idle."""
        self._check(self.lib.ofdft_slot_cancel(self.h, slot))

    def poll(self, slot) -> bool:
        f = ctypes.c_int()
        self._check(self.lib.ofdft_slot_poll(self.h, slot, ctypes.byref(f)))
        return bool(f.value)

    def result(self, slot, want_rho=True, out=None):
        """(rho, energies, stats) of a finished slot; `out` (an F-ordered float64
        array of the slot's shape) receives rho instead of a new array."""
        shp = self.shapes[slot]
        r = None
        if want_rho:
            r = out if out is not None else np.empty(shp, order="F")
            if r.shape != tuple(shp) or r.dtype != np.float64 or not r.flags.f_contiguous:
                raise ValueError("out must be an F-ordered float64 array of the slot's shape")
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
