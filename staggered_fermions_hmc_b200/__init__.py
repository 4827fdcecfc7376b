"""B200-native staggered-fermion HMC hot path (Python binding of libsfh.so).

The product is the C ABI in include/sfh.h, implemented by the CUDA library
libsfh.so built in-tree by ``staggered_fermions_hmc_b200.build``.  This module
binds it with ctypes and mirrors the reference's function names
(alexanderchasteen/Staggered_Fermions_HMC, Fermions.h / Lattice.h) so code
written against the reference reads the same:

    lat = Lattice(dims=(4, 4, 4, 4), mass=0.1, beta=4.2)
    lat.upload_gauge(U)                    # double[V*72], reference layout
    out = lat.apply_DDdagger(psi)          # Fermions.cpp:530
    X = lat.solve_CG_DDdagger(phi, tol)    # Fermions.cpp:553
    Y = lat.solve_Y_field(X)               # Fermions.cpp:623

There is no CPU fallback: importing raises if libsfh.so is missing, and every
call runs on the GPU.
"""
import ctypes
import os

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libsfh.so")

SFH_OK = 0
SFH_ERR_NOCONV = 1
SFH_ERR_BREAKDOWN = 2
SFH_ERR_DOMAIN = 3
SFH_ERR_NOT_HERMITIAN = 4
SFH_ERR_TIMEOUT = 5
SFH_ERR_CUDA = 6
SFH_ERR_INVALID = 7
SFH_ERR_NOMEM = 8
SFH_ERR_IO = 9
FORCE_GAUGE = 1
# sfh_kernel_timing's kernels (Lattice.HMC_KERNELS in the same order)
(KERNEL_GAUGE_FORCE, KERNEL_FERMION_FORCE, KERNEL_STAPLES, KERNEL_LINK_UPDATE, KERNEL_STOUT_LEVEL,
 KERNEL_STOUT_FORCE, KERNEL_ACTION, KERNEL_PLAQUETTE) = range(8)
FORCE_FERMION = 2

PREC_F64, PREC_F32, PREC_F16, PREC_F32_18, PREC_BF16 = 0, 1, 2, 3, 4
PRECISIONS = {"f64": PREC_F64, "f32": PREC_F32, "f16": PREC_F16, "f32_18": PREC_F32_18, "bf16": PREC_BF16}
BATCH_FULL_LATTICE = 1


class SfhError(RuntimeError):
    """Raised for a non-zero status; the reference throws std::runtime_error
    (CG breakdown / non-convergence, Fermions.cpp:574-614) or
    std::invalid_argument (exp domain, Fermions.cpp:848-857)."""

    def __init__(self, status, message):
        super().__init__(message)
        self.status = status


class CgParams(ctypes.Structure):
    _fields_ = [("dims", ctypes.c_int * 4), ("mass", ctypes.c_double), ("beta", ctypes.c_double),
                ("c11", ctypes.c_double), ("c12", ctypes.c_double), ("device", ctypes.c_int)]


class CgInfo(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int), ("iters", ctypes.c_int), ("iters_parity", ctypes.c_int * 2),
                ("reliable_updates", ctypes.c_int), ("rsq_rel", ctypes.c_double),
                ("true_resid", ctypes.c_double)]

    def as_dict(self):
        return {"status": self.status, "iters": self.iters,
                "iters_parity": [self.iters_parity[0], self.iters_parity[1]],
                "reliable_updates": self.reliable_updates, "rsq_rel": self.rsq_rel,
                "true_resid": self.true_resid}


class TrajInfo(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int), ("accepted", ctypes.c_int), ("solves", ctypes.c_int),
                ("pad", ctypes.c_int), ("cg_iters", ctypes.c_long), ("dH", ctypes.c_double),
                ("H_initial", ctypes.c_double * 3), ("H_final", ctypes.c_double * 3),
                ("uniform", ctypes.c_double), ("plaquette", ctypes.c_double), ("seconds", ctypes.c_double)]

    def as_dict(self):
        return {"status": self.status, "accepted": bool(self.accepted), "solves": self.solves,
                "cg_iters": self.cg_iters, "dH": self.dH, "H_initial": list(self.H_initial),
                "H_final": list(self.H_final), "uniform": self.uniform, "plaquette": self.plaquette,
                "seconds": self.seconds}


class SystemDesc(ctypes.Structure):
    _fields_ = [("dims", ctypes.c_int * 4), ("mass", ctypes.c_double), ("nrhs", ctypes.c_int)]


_D = ctypes.POINTER(ctypes.c_double)
_VP = ctypes.c_void_p

# name -> (restype, argtypes); the list is also the ABI symbol inventory
SIGNATURES = {
    "sfh_version": (ctypes.c_int, []),
    "sfh_status_string": (ctypes.c_char_p, [ctypes.c_int]),
    "sfh_create": (ctypes.c_int, [ctypes.POINTER(CgParams), ctypes.POINTER(_VP)]),
    "sfh_destroy": (ctypes.c_int, [_VP]),
    "sfh_last_error": (ctypes.c_char_p, [_VP]),
    "sfh_set_stream": (ctypes.c_int, [_VP, _VP]),
    "sfh_get_stream": (_VP, [_VP]),
    "sfh_set_mass": (ctypes.c_int, [_VP, ctypes.c_double]),
    "sfh_synchronize": (ctypes.c_int, [_VP]),
    "sfh_upload_gauge": (ctypes.c_int, [_VP, _D]),
    "sfh_download_gauge": (ctypes.c_int, [_VP, _D]),
    "sfh_random_gauge": (ctypes.c_int, [_VP, ctypes.c_double, ctypes.c_ulonglong]),
    "sfh_gaussian_spinor": (ctypes.c_int, [_VP, ctypes.c_ulonglong, ctypes.c_double, _D]),
    "sfh_random_momenta": (ctypes.c_int, [_VP, ctypes.c_ulonglong]),
    "sfh_upload_momenta": (ctypes.c_int, [_VP, _D]),
    "sfh_download_momenta": (ctypes.c_int, [_VP, _D]),
    "sfh_dirac": (ctypes.c_int, [_VP, ctypes.c_int, _D, _D]),
    "sfh_ddag": (ctypes.c_int, [_VP, _D, _D]),
    "sfh_dslash_timing": (ctypes.c_int, [_VP, ctypes.c_int, ctypes.c_int, _D]),
    "sfh_dslash_storage": (ctypes.c_int, [_VP, ctypes.c_int, _D, _D]),
    "sfh_set_staging_fault": (ctypes.c_int, [_VP, ctypes.c_int]),
    "sfh_cg_solve": (ctypes.c_int, [_VP, _D, _D, ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                    ctypes.POINTER(CgInfo)]),
    "sfh_staples": (ctypes.c_int, [_VP, _D, _D]),
    "sfh_gauge_force": (ctypes.c_int, [_VP, _D]),
    "sfh_fermion_force": (ctypes.c_int, [_VP, _D, _D, _D]),
    "sfh_full_force": (ctypes.c_int, [_VP, _D, _D, _D]),
    "sfh_link_update": (ctypes.c_int, [_VP, ctypes.c_double, ctypes.c_int]),
    "sfh_set_fermion_smearing": (ctypes.c_int, [_VP, ctypes.c_double, ctypes.c_int]),
    "sfh_heatbath": (ctypes.c_int, [_VP, ctypes.c_int, ctypes.c_ulonglong, ctypes.c_int, _D, _D]),
    "sfh_set_hasenbusch": (ctypes.c_int, [_VP, ctypes.c_double, _D]),
    "sfh_smeared_fermion_force": (ctypes.c_int, [_VP, _D, ctypes.c_double, ctypes.c_int, ctypes.c_int, _D, _D]),
    "sfh_momentum_kick": (ctypes.c_int, [_VP, ctypes.c_int, _D, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                         ctypes.c_int, _D, ctypes.POINTER(ctypes.c_long)]),
    "sfh_trp2": (ctypes.c_int, [_VP, _D]),
    "sfh_gauge_action": (ctypes.c_int, [_VP, _D]),
    "sfh_plaquette": (ctypes.c_int, [_VP, _D]),
    "sfh_set_beta": (ctypes.c_int, [_VP, ctypes.c_double]),
    "sfh_leapfrog": (ctypes.c_int, [_VP, _D, ctypes.c_double, ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                    ctypes.c_int, _D, ctypes.POINTER(ctypes.c_long)]),
    "sfh_hmc_trajectory": (ctypes.c_int, [_VP, ctypes.c_double, ctypes.c_int, ctypes.c_ulonglong,
                                          ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                          ctypes.POINTER(TrajInfo)]),
    "sfh_polyakov_grid": (ctypes.c_int, [_VP, _D]),
    "sfh_polyakov_correlator": (ctypes.c_int, [_VP, ctypes.c_int, _D]),
    "sfh_polyakov_correlator_grid": (ctypes.c_int, [_VP, _D, ctypes.c_int, _D]),
    "sfh_save_gauge": (ctypes.c_int, [_VP, ctypes.c_char_p]),
    "sfh_load_gauge": (ctypes.c_int, [_VP, ctypes.c_char_p]),
    "sfh_smear_stout": (ctypes.c_int, [_VP, ctypes.c_double, ctypes.c_int]),
    "sfh_smear_hex": (ctypes.c_int, [_VP, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int]),
    "sfh_hex_staples": (ctypes.c_int, [_VP, ctypes.c_int, _D, _D]),
    "sfh_kernel_timing": (ctypes.c_int, [_VP, ctypes.c_int, ctypes.c_int, _D]),
    "sfh_set_schedule": (ctypes.c_int, [_VP, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "sfh_batch_set_barrier_polls": (ctypes.c_int, [_VP, ctypes.c_longlong]),
    "sfh_batch_set_rhs_mass": (ctypes.c_int, [_VP, ctypes.c_int, ctypes.c_int, ctypes.c_double]),
    "sfh_batch_create": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.POINTER(SystemDesc),
                                        ctypes.c_int, ctypes.c_int, ctypes.POINTER(_VP)]),
    "sfh_batch_destroy": (ctypes.c_int, [_VP]),
    "sfh_batch_last_error": (ctypes.c_char_p, [_VP]),
    "sfh_batch_set_stream": (ctypes.c_int, [_VP, _VP]),
    "sfh_batch_get_stream": (_VP, [_VP]),
    "sfh_batch_set_rhs_block": (ctypes.c_int, [_VP, ctypes.c_int]),
    "sfh_batch_set_hop_widths": (ctypes.c_int, [_VP, ctypes.c_int, ctypes.c_int]),
    "sfh_batch_get_hop_widths": (ctypes.c_int, [_VP, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]),
    "sfh_batch_autotune": (ctypes.c_int, [_VP, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]),
    "sfh_batch_set_schedule": (ctypes.c_int, [_VP, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "sfh_batch_set_reliable_delta": (ctypes.c_int, [_VP, ctypes.c_double]),
    "sfh_batch_solve_timed": (ctypes.c_int, [_VP, ctypes.c_double, ctypes.c_int, _D,
                                             ctypes.POINTER(ctypes.c_long)]),
    "sfh_batch_get_schedule": (ctypes.c_int, [_VP, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                              ctypes.POINTER(ctypes.c_int)]),
    "sfh_batch_set_gauge": (ctypes.c_int, [_VP, ctypes.c_int, _D]),
    "sfh_batch_set_rhs": (ctypes.c_int, [_VP, ctypes.c_int, ctypes.c_int, _D]),
    "sfh_batch_solve": (ctypes.c_int, [_VP, ctypes.c_double, ctypes.c_int]),
    "sfh_batch_get_solution": (ctypes.c_int, [_VP, ctypes.c_int, ctypes.c_int, _D]),
    "sfh_batch_get_info": (ctypes.c_int, [_VP, ctypes.c_int, ctypes.c_int, ctypes.POINTER(CgInfo)]),
    "sfh_batch_random_gauge": (ctypes.c_int, [_VP, ctypes.c_int, ctypes.c_double, ctypes.c_ulonglong]),
    "sfh_batch_random_rhs": (ctypes.c_int, [_VP, ctypes.c_int, ctypes.c_int, ctypes.c_ulonglong,
                                            ctypes.c_double]),
    "sfh_batch_get_gauge": (ctypes.c_int, [_VP, ctypes.c_int, _D]),
    "sfh_batch_get_rhs": (ctypes.c_int, [_VP, ctypes.c_int, ctypes.c_int, _D]),
    "sfh_batch_true_residual": (ctypes.c_int, [_VP, ctypes.c_int, ctypes.c_int, _D]),
    "sfh_batch_kernel_launches": (ctypes.c_int, [_VP, ctypes.POINTER(ctypes.c_long)]),
    "sfh_cg_solve_noalloc": (ctypes.c_int, [ctypes.POINTER(ctypes.c_int), ctypes.c_double, _VP, _VP, _VP,
                                            ctypes.c_double, ctypes.c_int, _VP, ctypes.POINTER(CgInfo)]),
}

NOALLOC_MAX_SITES = 65536
TIMED_KERNELS = 6

_lib = None


def load_library(path=LIB_PATH):
    """Load libsfh.so; raises (no fallback) if it is missing."""
    global _lib
    if _lib is None:
        if not os.path.exists(path):
            raise ImportError(f"{path} is missing: build it with "
                              "`python -m staggered_fermions_hmc_b200.build`")
        lib = ctypes.CDLL(path)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
        _lib = lib
    return _lib


def _dptr(a):
    if a.dtype != np.float64 or not a.flags["C_CONTIGUOUS"]:
        raise TypeError("expected a C-contiguous float64 array")
    return a.ctypes.data_as(_D)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def volume(dims):
    return int(np.prod(dims))


class Lattice:
    """One lattice on one GPU: the runtime replacement of the reference's
    compile-time lattice (Parameters.h) and its static tables
    (Fermions.cpp:20-96).  Methods keep the reference's names."""

    def __init__(self, dims, mass, beta=4.2, c11=5.0 / 3.0, c12=-1.0 / 12.0, device=0):
        self.lib = load_library()
        self.dims = tuple(int(d) for d in dims)
        self.V = volume(self.dims)
        p = CgParams((ctypes.c_int * 4)(*self.dims), mass, beta, c11, c12, device)
        h = _VP()
        st = self.lib.sfh_create(ctypes.byref(p), ctypes.byref(h))
        if st != SFH_OK:
            raise SfhError(st, f"sfh_create: {self.lib.sfh_status_string(st).decode()}")
        self.h = h
        self.mass = mass
        self.beta = beta

    def close(self):
        if getattr(self, "h", None):
            self.lib.sfh_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st, what):
        if st != SFH_OK:
            msg = self.lib.sfh_last_error(self.h)
            raise SfhError(st, f"{what}: {self.lib.sfh_status_string(st).decode()}: "
                               f"{msg.decode() if msg else ''}")

    @property
    def stream(self):
        return self.lib.sfh_get_stream(self.h)

    def set_mass(self, m):
        self._check(self.lib.sfh_set_mass(self.h, m), "set_mass")
        self.mass = m

    def upload_gauge(self, U):
        U = _f64(U).reshape(-1)
        assert U.size == 72 * self.V
        self._check(self.lib.sfh_upload_gauge(self.h, _dptr(U)), "upload_gauge")

    def download_gauge(self):
        out = np.empty(72 * self.V)
        self._check(self.lib.sfh_download_gauge(self.h, _dptr(out)), "download_gauge")
        return out

    # --- seeded generators ---------------------------------------------------
    def random_gauge(self, eps, seed):
        """U = exp(i eps H) on every link (seeded hot start)."""
        self._check(self.lib.sfh_random_gauge(self.h, eps, seed), "random_gauge")

    def gaussian_spinor(self, seed, sigma=1.0):
        out = np.empty(6 * self.V)
        self._check(self.lib.sfh_gaussian_spinor(self.h, seed, sigma, _dptr(out)), "gaussian_spinor")
        return out

    def generate_conjugate_field_configuration(self, seed):
        """Fermions.cpp:342-360, seeded; stays on the device."""
        self._check(self.lib.sfh_random_momenta(self.h, seed), "random_momenta")

    def upload_momenta(self, P):
        P = _f64(P).reshape(-1)
        self._check(self.lib.sfh_upload_momenta(self.h, _dptr(P)), "upload_momenta")

    def download_momenta(self):
        out = np.empty(72 * self.V)
        self._check(self.lib.sfh_download_momenta(self.h, _dptr(out)), "download_momenta")
        return out

    # --- Fermions.cpp:218-283 --------------------------------------------
    def apply_dirac_operator(self, psi):
        psi = _f64(psi).reshape(-1)
        out = np.empty_like(psi)
        self._check(self.lib.sfh_dirac(self.h, 0, _dptr(psi), _dptr(out)), "dirac")
        return out

    def apply_dirac_dagger(self, psi):
        psi = _f64(psi).reshape(-1)
        out = np.empty_like(psi)
        self._check(self.lib.sfh_dirac(self.h, 1, _dptr(psi), _dptr(out)), "dirac_dagger")
        return out

    def dslash_storage(self, storage, psi):
        """K psi (the hopping term, both parities) by the standalone Dslash in
        a storage format (0 FP64-18, 1 FP32-12, 2 FP16-12, 3 FP32-18,
        4 BF16-12, 5 FP64-12; 6 and 7 the storages of 2 and 4 with each
        block's time and z neighbours staged in shared memory by one bulk
        asynchronous copy), returned in FP64."""
        psi = _f64(psi).reshape(-1)
        out = np.empty_like(psi)
        self._check(self.lib.sfh_dslash_storage(self.h, storage, _dptr(psi), _dptr(out)), "dslash storage")
        return out

    def set_staging_fault(self, extra_bytes):
        """Test hook of the time-staged Dslash (storages 6, 7): announce
        extra_bytes more per block than its bulk copy delivers, so every
        staging wait runs out (SFH_ERR_TIMEOUT, same result); 0 turns it off."""
        self._check(self.lib.sfh_set_staging_fault(self.h, int(extra_bytes)), "set_staging_fault")

    def dslash_timing(self, storage, nrep=20):
        """ms per even-odd hop (V/2 output sites); storage 0 FP64-18, 1 FP32-12,
        2 FP16-12, 3 FP32-18, 4 BF16-12, 5 FP64-12, 6 FP16-12 and 7 BF16-12
        with the neighbours staged along the time direction."""
        ms = ctypes.c_double(0.0)
        self._check(self.lib.sfh_dslash_timing(self.h, storage, nrep, ctypes.byref(ms)), "dslash timing")
        return ms.value

    # --- Fermions.cpp:530-547 ----------------------------------------------
    def apply_DDdagger(self, psi):
        psi = _f64(psi).reshape(-1)
        out = np.empty_like(psi)
        self._check(self.lib.sfh_ddag(self.h, _dptr(psi), _dptr(out)), "apply_DDdagger")
        return out

    # --- Fermions.cpp:553-633 ----------------------------------------------
    def solve_CG_DDdagger(self, phi, tol=1e-12, max_iter=50000, precision="f64", info=False):
        phi = _f64(phi).reshape(-1)
        X = np.empty_like(phi)
        inf = CgInfo()
        st = self.lib.sfh_cg_solve(self.h, _dptr(phi), _dptr(X), tol, max_iter,
                                   PRECISIONS[precision], ctypes.byref(inf))
        self._check(st, "solve_CG_DDdagger")
        return (X, inf.as_dict()) if info else X

    def solve_X_field(self, phi, tol=1e-12, max_iter=50000, precision="f64"):
        return self.solve_CG_DDdagger(phi, tol, max_iter, precision)

    def solve_Y_field(self, X):
        return self.apply_dirac_dagger(X)

    # --- forces, link update, observables (Fermions.cpp:372-828, Lattice.cpp:249-804)
    def _link_field(self):
        return np.empty(72 * self.V)

    def staples(self):
        A1, A2 = self._link_field(), self._link_field()
        self._check(self.lib.sfh_staples(self.h, _dptr(A1), _dptr(A2)), "staples")
        return A1, A2

    def compute_gauge_only_force_field(self):
        F = self._link_field()
        self._check(self.lib.sfh_gauge_force(self.h, _dptr(F)), "gauge force")
        return F

    def compute_fermion_only_force_field(self, X, Y):
        X, Y, F = _f64(X).reshape(-1), _f64(Y).reshape(-1), self._link_field()
        self._check(self.lib.sfh_fermion_force(self.h, _dptr(X), _dptr(Y), _dptr(F)), "fermion force")
        return F

    def compute_full_force_field(self, X, Y):
        X, Y, F = _f64(X).reshape(-1), _f64(Y).reshape(-1), self._link_field()
        self._check(self.lib.sfh_full_force(self.h, _dptr(X), _dptr(Y), _dptr(F)), "full force")
        return F

    def link_update(self, eps, check=False):
        self._check(self.lib.sfh_link_update(self.h, eps, 1 if check else 0), "link update")

    def _scalar(self, fn, what):
        out = ctypes.c_double(0.0)
        self._check(fn(self.h, ctypes.byref(out)), what)
        return out.value

    def compute_Tr_P2(self):
        return self._scalar(self.lib.sfh_trp2, "Tr P^2")

    def compute_action(self):
        return self._scalar(self.lib.sfh_gauge_action, "gauge action")

    def compute_avg_plaq(self):
        return self._scalar(self.lib.sfh_plaquette, "plaquette")

    def set_beta(self, beta):
        self._check(self.lib.sfh_set_beta(self.h, beta), "set_beta")
        self.beta = beta

    def leapfrog(self, phi, eps, n_steps, tol=1e-12, max_iter=50000, precision="f64"):
        """local_initial_half_step + local_leapfrog_steps + local_final_step
        (Fermions.cpp:967-1028) on the device gauge field and momenta."""
        phi = _f64(phi).reshape(-1)
        X = np.empty_like(phi)
        its = ctypes.c_long(0)
        st = self.lib.sfh_leapfrog(self.h, _dptr(phi), eps, n_steps, tol, max_iter, PRECISIONS[precision],
                                   _dptr(X), ctypes.byref(its))
        self._check(st, "leapfrog")
        return X, its.value

    def heatbath_update(self, n_sweeps=1, seed=1, sweep0=0):
        """heatbath_update (Lattice.cpp:722-757) n_sweeps times at the context's
        beta; returns (average plaquette, action per site) after the sweeps."""
        p, a = ctypes.c_double(0.0), ctypes.c_double(0.0)
        self._check(self.lib.sfh_heatbath(self.h, n_sweeps, seed, sweep0, ctypes.byref(p), ctypes.byref(a)),
                    "heatbath")
        return p.value, a.value

    def set_hasenbusch(self, heavy_mass, phi_heavy=None):
        """Hasenbusch pair: heavy pseudofermion at heavy_mass (0 = off)."""
        ph = None if phi_heavy is None else _f64(phi_heavy).reshape(-1)
        self._check(self.lib.sfh_set_hasenbusch(self.h, heavy_mass, None if ph is None else _dptr(ph)),
                    "set_hasenbusch")

    def set_fermion_smearing(self, rho, n_levels):
        """Fermion operator on stout^n(U) in the HMC (n_levels = 0: thin links)."""
        self._check(self.lib.sfh_set_fermion_smearing(self.h, rho, n_levels), "set_fermion_smearing")

    def smeared_fermion_force(self, phi, tol=1e-12, max_iter=50000, precision="f64"):
        """Thin-link fermion force with stout-smeared fermion links; returns (F, X)."""
        phi = _f64(phi).reshape(-1)
        F = np.empty(72 * self.V)
        X = np.empty_like(phi)
        self._check(self.lib.sfh_smeared_fermion_force(self.h, _dptr(phi), tol, max_iter, PRECISIONS[precision],
                                                       _dptr(F), _dptr(X)), "smeared_fermion_force")
        return F, X

    def momentum_kick(self, dt, phi=None, forces="full", tol=1e-12, max_iter=50000, precision="f64"):
        """P -= dt F on the device momenta, F the gauge, fermion or full force
        (Fermions.cpp:690-695, 730-735, 767-773).  Returns (X, cg_iters); X is
        None for the gauge force alone."""
        bits = {"gauge": FORCE_GAUGE, "fermion": FORCE_FERMION, "full": FORCE_GAUGE | FORCE_FERMION}[forces]
        its = ctypes.c_long(0)
        if bits & FORCE_FERMION:
            phi = _f64(phi).reshape(-1)
            X = np.empty_like(phi)
            st = self.lib.sfh_momentum_kick(self.h, bits, _dptr(phi), dt, tol, max_iter, PRECISIONS[precision],
                                            _dptr(X), ctypes.byref(its))
        else:
            X = None
            st = self.lib.sfh_momentum_kick(self.h, bits, None, dt, tol, max_iter, PRECISIONS[precision],
                                            None, ctypes.byref(its))
        self._check(st, "momentum kick")
        return X, its.value

    def hmc_trajectory(self, eps, n_steps, seed, tol=1e-10, max_iter=50000, precision="f64"):
        """single_sweep_monte_carlo_update_WITH_FERMIONS (Fermions.cpp:812-828)."""
        inf = TrajInfo()
        st = self.lib.sfh_hmc_trajectory(self.h, eps, n_steps, seed, tol, max_iter, PRECISIONS[precision],
                                         ctypes.byref(inf))
        self._check(st, "hmc trajectory")
        return inf.as_dict()

    # --- observables, checkpoints (Lattice.cpp:810-948) ------------------------
    def precompute_polyakov_grid(self):
        out = np.empty(2 * self.dims[0] * self.dims[1] * self.dims[2])
        self._check(self.lib.sfh_polyakov_grid(self.h, _dptr(out)), "polyakov grid")
        return out.view(np.complex128)

    def correlator_over_fixed_distance(self, r_squared):
        out = np.empty(2)
        self._check(self.lib.sfh_polyakov_correlator(self.h, int(r_squared), _dptr(out)), "polyakov correlator")
        return complex(out[0], out[1])

    def correlator_over_fixed_distance_fast(self, P_grid, r_squared):
        """correlator_over_fixed_distance_fast(P_grid, r2) (Lattice.cpp:886-948)
        from a grid as precompute_polyakov_grid returns it."""
        g = np.ascontiguousarray(np.asarray(P_grid, dtype=np.complex128)).view(np.float64)
        if g.size != 2 * self.dims[0] * self.dims[1] * self.dims[2]:
            raise ValueError("P_grid must hold one complex value per spatial site")
        out = np.empty(2)
        self._check(self.lib.sfh_polyakov_correlator_grid(self.h, _dptr(g), int(r_squared), _dptr(out)),
                    "polyakov correlator")
        return complex(out[0], out[1])

    def save_lattice_config(self, path):
        self._check(self.lib.sfh_save_gauge(self.h, os.fsencode(path)), "save_lattice_config")

    def load_lattice_config(self, path):
        self._check(self.lib.sfh_load_gauge(self.h, os.fsencode(path)), "load_lattice_config")

    # --- smearing (Smearing.cpp) ---------------------------------------------
    def smear_stout(self, rho, n_levels=1):
        self._check(self.lib.sfh_smear_stout(self.h, rho, n_levels), "stout smearing")

    def set_schedule(self, width=0, tiles_per_block=0, stage_links=0):
        """Schedule of this lattice's mixed-precision solves (as
        Batch.set_schedule; stage_links 3: one persistent launch per solve)."""
        self._check(self.lib.sfh_set_schedule(self.h, width, tiles_per_block, int(stage_links)), "set_schedule")

    HMC_KERNELS = ("gauge_force", "fermion_force", "staples", "link_update", "stout_level", "stout_force",
                   "action", "plaquette")

    def kernel_timing(self, kernel, nrep=10):
        """ms per launch of one HMC kernel (a name of HMC_KERNELS) on the
        context's fields, CUDA events on its stream."""
        ms = ctypes.c_double(0.0)
        self._check(self.lib.sfh_kernel_timing(self.h, self.HMC_KERNELS.index(kernel), nrep, ctypes.byref(ms)),
                    "kernel_timing")
        return ms.value

    def hex_staples(self, level, field):
        """apply_step_1 / apply_step_3 / apply_step_5 (Smearing.cpp:76-275) for
        level 1 / 2 / 3 on a host field in the reference's flat tensor layout."""
        field = _f64(field).reshape(-1)
        out = np.empty({1: 64, 2: 16, 3: 4}[level] * self.V * 18)
        self._check(self.lib.sfh_hex_staples(self.h, level, _dptr(field), _dptr(out)), "hex_staples")
        return out

    def Apply_HEX_smearing(self, alphas=(0.95, 0.76, 0.38), passes=1):
        self._check(self.lib.sfh_smear_hex(self.h, alphas[0], alphas[1], alphas[2], passes), "HEX smearing")

    def Apply_4HEX_smearing(self, alphas=(0.95, 0.76, 0.38)):
        self.Apply_HEX_smearing(alphas, passes=4)


class Batch:
    """Many independent D D^dag solves (lattices, masses, right-hand sides)
    solved by one persistent launch.  No reference counterpart."""

    def __init__(self, systems, precision="f32", full_lattice=False, device=0):
        self.lib = load_library()
        n = len(systems)
        arr = (SystemDesc * n)()
        self.systems = []
        for k, (dims, mass, nrhs) in enumerate(systems):
            arr[k] = SystemDesc((ctypes.c_int * 4)(*dims), mass, nrhs)
            self.systems.append((tuple(dims), float(mass), int(nrhs)))
        h = _VP()
        st = self.lib.sfh_batch_create(device, n, arr, PRECISIONS[precision],
                                       BATCH_FULL_LATTICE if full_lattice else 0, ctypes.byref(h))
        if st != SFH_OK:
            raise SfhError(st, f"sfh_batch_create: {self.lib.sfh_status_string(st).decode()}")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.lib.sfh_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st, what):
        if st != SFH_OK:
            msg = self.lib.sfh_batch_last_error(self.h)
            raise SfhError(st, f"{what}: {self.lib.sfh_status_string(st).decode()}: "
                               f"{msg.decode() if msg else ''}")

    @property
    def stream(self):
        return self.lib.sfh_batch_get_stream(self.h)

    def set_rhs_block(self, width):
        self._check(self.lib.sfh_batch_set_rhs_block(self.h, width), "set_rhs_block")

    def set_hop_widths(self, hop1_width, hop2_width):
        """RHS-block widths of the first and second hop kernels separately
        (after set_schedule, which sets both)."""
        self._check(self.lib.sfh_batch_set_hop_widths(self.h, hop1_width, hop2_width), "set_hop_widths")

    def hop_widths(self):
        """(first hop's, second hop's) RHS-block widths the next solve uses."""
        a, b = ctypes.c_int(0), ctypes.c_int(0)
        self._check(self.lib.sfh_batch_get_hop_widths(self.h, ctypes.byref(a), ctypes.byref(b)), "hop_widths")
        return a.value, b.value

    def autotune(self, probe_iters=48):
        """Pick the fastest RHS-block width and tiles per block for this batch
        (schedule only); returns the width."""
        w = ctypes.c_int(0)
        self._check(self.lib.sfh_batch_autotune(self.h, probe_iters, ctypes.byref(w)), "autotune")
        return w.value

    def solve_timed(self, tol=1e-10, max_iter=20000):
        """Solve with per-kernel CUDA-event timing; returns {kernel: (ms, launches)}
        for the kernels the schedule launched (the reliable-update kernels
        cg_ru1 / cg_ru2 with the system-blocked schedule only; cg_persistent
        alone with the persistent schedule)."""
        ms = np.zeros(TIMED_KERNELS)
        n = (ctypes.c_long * TIMED_KERNELS)()
        self._check(self.lib.sfh_batch_solve_timed(self.h, tol, max_iter, _dptr(ms), n), "solve_timed")
        names = ("cg_hop1", "cg_hop2", "cg_update", "cg_ru1", "cg_ru2", "cg_persistent")
        return {k: (float(ms[i]), int(n[i])) for i, k in enumerate(names) if n[i] > 0}

    def set_schedule(self, width, tiles_per_block, stage_links=0):
        """stage_links: 0 (or False) links read directly, 1 (or True) staged per
        work item, 2 system-blocked (one tile per block serving every RHS of
        the system, links read once per tile), 3 the system-blocked work in
        one persistent cooperative launch, 4 and 5: 0 and 1 with the reliable
        updates in lane-list kernels, 6 (FP16): 4 with each tile's time and z
        neighbours staged in shared memory by bulk asynchronous copies, 7: 4
        with the hop kernels on resident grids taking their work items from
        a device counter."""
        self._check(self.lib.sfh_batch_set_schedule(self.h, width, tiles_per_block, int(stage_links)),
                    "set_schedule")

    def set_rhs_mass(self, k, j, mass):
        """Mass of right-hand side j of system k (default: the system's)."""
        self._check(self.lib.sfh_batch_set_rhs_mass(self.h, k, j, mass), "set_rhs_mass")

    def set_barrier_polls(self, polls):
        """Bound on each grid-barrier wait of the persistent schedule (0: the
        default, about 4 s)."""
        self._check(self.lib.sfh_batch_set_barrier_polls(self.h, int(polls)), "set_barrier_polls")

    def set_reliable_delta(self, delta):
        """Reliable-update threshold of the mixed precisions (default 0.1 for
        "f16" and "bf16", 0.01 for the FP32 storages)."""
        self._check(self.lib.sfh_batch_set_reliable_delta(self.h, delta), "set_reliable_delta")

    def schedule(self):
        """(RHS-block width, tiles per block, link staging 0 / 1 / 2) the next
        solve uses."""
        w, t, g = ctypes.c_int(0), ctypes.c_int(0), ctypes.c_int(0)
        self._check(self.lib.sfh_batch_get_schedule(self.h, ctypes.byref(w), ctypes.byref(t), ctypes.byref(g)),
                    "schedule")
        return w.value, t.value, g.value

    def set_gauge(self, k, U):
        U = _f64(U).reshape(-1)
        self._check(self.lib.sfh_batch_set_gauge(self.h, k, _dptr(U)), "set_gauge")

    def set_rhs(self, k, j, phi):
        phi = _f64(phi).reshape(-1)
        self._check(self.lib.sfh_batch_set_rhs(self.h, k, j, _dptr(phi)), "set_rhs")

    def random_gauge(self, k, eps, seed):
        self._check(self.lib.sfh_batch_random_gauge(self.h, k, eps, seed), "random_gauge")

    def random_rhs(self, k, j, seed, sigma=1.0):
        self._check(self.lib.sfh_batch_random_rhs(self.h, k, j, seed, sigma), "random_rhs")

    def gauge(self, k):
        out = np.empty(72 * volume(self.systems[k][0]))
        self._check(self.lib.sfh_batch_get_gauge(self.h, k, _dptr(out)), "get_gauge")
        return out

    def rhs(self, k, j):
        out = np.empty(6 * volume(self.systems[k][0]))
        self._check(self.lib.sfh_batch_get_rhs(self.h, k, j, _dptr(out)), "get_rhs")
        return out

    def solve(self, tol=1e-10, max_iter=50000, check=True):
        st = self.lib.sfh_batch_solve(self.h, tol, max_iter)
        if check:
            self._check(st, "batch solve")
        return st

    def solution(self, k, j, out=None):
        """X of system k, right-hand side j (reference layout).  With ``out``
        (a C-contiguous float64 array of 6 V, e.g. in pinned memory) the
        solution is copied straight into it."""
        n = 6 * volume(self.systems[k][0])
        X = np.empty(n) if out is None else out
        if X.size != n:
            raise ValueError(f"out has {X.size} elements, expected {n}")
        self._check(self.lib.sfh_batch_get_solution(self.h, k, j, _dptr(X)), "get_solution")
        return X

    def info(self, k, j):
        inf = CgInfo()
        self._check(self.lib.sfh_batch_get_info(self.h, k, j, ctypes.byref(inf)), "get_info")
        return inf.as_dict()

    def kernel_launches(self):
        n = ctypes.c_long(0)
        self._check(self.lib.sfh_batch_kernel_launches(self.h, ctypes.byref(n)), "kernel_launches")
        return n.value

    def true_residual(self, k, j):
        r = ctypes.c_double(0)
        self._check(self.lib.sfh_batch_true_residual(self.h, k, j, ctypes.byref(r)), "true_residual")
        return r.value
