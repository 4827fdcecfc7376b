"""CPU oracle for the staggered-fermion HMC hot path (test infrastructure).

This package is the checker: a plain-C restatement of the reference
algorithms (sfh_oracle.c) loaded through ctypes, plus helpers to build the
reference's own sources (build_ref.py) for golden fixtures.  Only tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline leg import it; the
product library never does.

Arrays use the reference's AoS layouts: gauge / momentum / force fields are
float64 [V, 4, 3, 3, 2] (72 doubles per site), spinors float64 [V, 3, 2].
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liborc.so")

ORC_OK, ORC_ERR_NOCONV, ORC_ERR_BREAKDOWN, ORC_ERR_DOMAIN = 0, 1, 2, 3


def build(force=False):
    """Compile sfh_oracle.c into oracle/liborc.so (gcc, OpenMP)."""
    src = os.path.join(HERE, "sfh_oracle.c")
    if (not force and os.path.exists(LIB_PATH)
            and os.path.getmtime(LIB_PATH) >= os.path.getmtime(src)):
        return LIB_PATH
    tmp = LIB_PATH + ".tmp"
    subprocess.run(["gcc", "-O3", "-fopenmp", "-fPIC", "-shared", "-std=c11",
                    "-o", tmp, src, "-lm"], check=True)
    os.replace(tmp, LIB_PATH)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(LIB_PATH)
        D = ctypes.POINTER(ctypes.c_double)
        I = ctypes.POINTER(ctypes.c_int)
        dims = ctypes.c_int * 4
        sig = {
            "orc_tables": (None, [dims, I, I, I, I, I]),
            "orc_dirac": (None, [dims, ctypes.c_double, ctypes.c_int, D, D, D]),
            "orc_ddag": (None, [dims, ctypes.c_double, D, D, D]),
            "orc_dot": (ctypes.c_double, [ctypes.c_long, D, D]),
            "orc_cg": (ctypes.c_int, [dims, ctypes.c_double, D, D, ctypes.c_double,
                                      ctypes.c_int, D, I, D]),
            "orc_staples": (None, [dims, D, D, D]),
            "orc_gauge_force": (None, [dims, ctypes.c_double, ctypes.c_double,
                                       ctypes.c_double, D, D]),
            "orc_fermion_force": (None, [dims, D, D, D, D]),
            "orc_full_force": (None, [dims, ctypes.c_double, ctypes.c_double,
                                      ctypes.c_double, D, D, D, D]),
            "orc_expiq": (ctypes.c_int, [D, D]),
            "orc_link_update": (ctypes.c_int, [dims, ctypes.c_double, D, D]),
            "orc_trp2": (ctypes.c_double, [dims, D]),
            "orc_action": (ctypes.c_double, [dims, ctypes.c_double, ctypes.c_double,
                                             ctypes.c_double, D]),
            "orc_avg_plaq": (ctypes.c_double, [dims, D]),
            "orc_leapfrog": (ctypes.c_int, [dims, ctypes.c_double, ctypes.c_double,
                                            ctypes.c_double, ctypes.c_double,
                                            ctypes.c_double, ctypes.c_int,
                                            ctypes.c_double, ctypes.c_int, D, D, D, D,
                                            ctypes.POINTER(ctypes.c_long)]),
            "orc_polyakov_grid": (None, [dims, D, D]),
            "orc_polyakov_corr": (None, [dims, D, ctypes.c_int, D]),
            "orc_stout": (ctypes.c_int, [dims, ctypes.c_double, ctypes.c_int, D]),
            "orc_hex": (ctypes.c_int, [dims, D, D]),
            "orc_stout_force": (ctypes.c_int, [dims, ctypes.c_double, ctypes.c_int, D, D, D]),
            "orc_heatbath": (ctypes.c_int, [dims, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                            ctypes.c_ulonglong, ctypes.c_int, ctypes.c_int, D]),
            "orc_exp_field": (ctypes.c_int, [ctypes.c_long, ctypes.c_double, D, D]),
            "orc_hex_gamma1": (None, [dims, D, D]),
            "orc_hex_gamma2": (None, [dims, D, D]),
            "orc_hex_gamma3": (None, [dims, D, D]),
            "orc_philox4x32_10": (None, [ctypes.POINTER(ctypes.c_uint), ctypes.POINTER(ctypes.c_uint),
                                         ctypes.POINTER(ctypes.c_uint)]),
            "orc_gen_normals": (None, [ctypes.c_ulonglong, ctypes.c_uint, ctypes.c_ulonglong, ctypes.c_int, D]),
            "orc_gen_gauge": (ctypes.c_int, [dims, ctypes.c_double, ctypes.c_ulonglong, D]),
            "orc_gen_spinor": (None, [dims, ctypes.c_double, ctypes.c_ulonglong, D]),
            "orc_gen_momenta": (None, [dims, ctypes.c_ulonglong, D]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _d(a):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _i(a):
    assert a.dtype == np.int32 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


def _dims(dims):
    return (ctypes.c_int * 4)(*[int(x) for x in dims])


def volume(dims):
    return int(np.prod(dims))


class OracleError(RuntimeError):
    def __init__(self, status, what):
        super().__init__(f"{what}: oracle status {status}")
        self.status = status


def tables(dims):
    V = volume(dims)
    arrs = [np.zeros(4 * V, np.int32) for _ in range(5)]
    lib().orc_tables(_dims(dims), *[_i(a) for a in arrs])
    return dict(zip(["up", "dn", "bc_up", "bc_dn", "eta"], arrs))


def dirac(dims, mass, U, psi, dagger=False):
    out = np.empty_like(psi)
    lib().orc_dirac(_dims(dims), mass, -1 if dagger else 1, _d(U), _d(psi), _d(out))
    return out


def ddag(dims, mass, U, psi):
    out = np.empty_like(psi)
    lib().orc_ddag(_dims(dims), mass, _d(U), _d(psi), _d(out))
    return out


def dot(a, b):
    return lib().orc_dot(a.size, _d(a), _d(b))


def cg(dims, mass, U, phi, tol, maxit=50000, check=True):
    X = np.empty_like(phi)
    it = ctypes.c_int(0)
    rsq = ctypes.c_double(0.0)
    st = lib().orc_cg(_dims(dims), mass, _d(U), _d(phi), tol, maxit, _d(X),
                      ctypes.byref(it), ctypes.byref(rsq))
    if check and st != ORC_OK:
        raise OracleError(st, "cg")
    return X, it.value, rsq.value, st


def staples(dims, U):
    A1 = np.empty_like(U)
    A2 = np.empty_like(U)
    lib().orc_staples(_dims(dims), _d(U), _d(A1), _d(A2))
    return A1, A2


def gauge_force(dims, beta, U, c11=5.0 / 3.0, c12=-1.0 / 12.0):
    F = np.empty_like(U)
    lib().orc_gauge_force(_dims(dims), beta, c11, c12, _d(U), _d(F))
    return F


def fermion_force(dims, U, X, Y):
    F = np.empty_like(U)
    lib().orc_fermion_force(_dims(dims), _d(U), _d(X), _d(Y), _d(F))
    return F


def full_force(dims, beta, U, X, Y, c11=5.0 / 3.0, c12=-1.0 / 12.0):
    F = np.empty_like(U)
    lib().orc_full_force(_dims(dims), beta, c11, c12, _d(U), _d(X), _d(Y), _d(F))
    return F


def expiq(Q):
    Q = np.ascontiguousarray(Q, dtype=np.float64).reshape(18)
    out = np.empty(18)
    st = lib().orc_expiq(_d(Q), _d(out))
    if st != ORC_OK:
        raise OracleError(st, "expiq")
    return out


def exp_field(eps, H):
    H = np.ascontiguousarray(H, dtype=np.float64)
    U = np.empty_like(H)
    st = lib().orc_exp_field(H.size // 18, eps, _d(H), _d(U))
    if st != ORC_OK:
        raise OracleError(st, "exp_field")
    return U


def link_update(dims, eps, P, U):
    U = U.copy()
    st = lib().orc_link_update(_dims(dims), eps, _d(P), _d(U))
    if st != ORC_OK:
        raise OracleError(st, "link_update")
    return U


def trp2(dims, P):
    return lib().orc_trp2(_dims(dims), _d(P))


def action(dims, beta, U, c11=5.0 / 3.0, c12=-1.0 / 12.0):
    return lib().orc_action(_dims(dims), beta, c11, c12, _d(U))


def avg_plaq(dims, U):
    return lib().orc_avg_plaq(_dims(dims), _d(U))


def leapfrog(dims, mass, beta, eps, n_steps, phi, P, U, tol=1e-12, maxit=50000,
             c11=5.0 / 3.0, c12=-1.0 / 12.0):
    P = P.copy()
    U = U.copy()
    X = np.empty_like(phi)
    its = ctypes.c_long(0)
    st = lib().orc_leapfrog(_dims(dims), mass, beta, c11, c12, eps, n_steps, tol,
                            maxit, _d(phi), _d(P), _d(U), _d(X), ctypes.byref(its))
    if st != ORC_OK:
        raise OracleError(st, "leapfrog")
    return P, U, X, its.value


def polyakov_grid(dims, U):
    out = np.empty(2 * dims[0] * dims[1] * dims[2])
    lib().orc_polyakov_grid(_dims(dims), _d(U), _d(out))
    return out


def polyakov_corr(dims, grid, r2):
    out = np.empty(2)
    lib().orc_polyakov_corr(_dims(dims), _d(grid), int(r2), _d(out))
    return complex(out[0], out[1])


def stout(dims, rho, n_levels, U):
    U = U.copy()
    st = lib().orc_stout(_dims(dims), rho, n_levels, _d(U))
    if st != ORC_OK:
        raise OracleError(st, "stout")
    return U


def heatbath(dims, beta, U, seed, nsweeps=1, sweep0=0, c11=5.0 / 3.0, c12=-1.0 / 12.0):
    """nsweeps heatbath sweeps in colour order with seeded uniforms."""
    U = U.copy()
    st = lib().orc_heatbath(_dims(dims), beta, c11, c12, seed, sweep0, nsweeps, _d(U))
    if st != ORC_OK:
        raise OracleError(st, "heatbath")
    return U


def stout_force(dims, rho, n_levels, U, F_top):
    """Thin-link force of an action on n_levels stout levels of U, given the
    force on the smeared links (chain rule; no reference counterpart)."""
    F = np.empty_like(U)
    st = lib().orc_stout_force(_dims(dims), rho, n_levels, _d(U), _d(F_top), _d(F))
    if st != ORC_OK:
        raise OracleError(st, "stout_force")
    return F


def hex_smear(dims, U, alphas=(0.95, 0.76, 0.38)):
    U = U.copy()
    a = np.array(alphas, dtype=np.float64)
    st = lib().orc_hex(_dims(dims), _d(a), _d(U))
    if st != ORC_OK:
        raise OracleError(st, "hex")
    return U


# ---------------------------------------------------------------------------
# seeded synthetic inputs (same distributions as the reference generators)
# ---------------------------------------------------------------------------

def random_hermitian(rng, n):
    """n traceless Hermitian 3x3 with N(0,1) diagonal and N(0,1) off-diagonal
    real/imag parts, trace removed (Lattice.cpp:1001-1033), as [n,18]."""
    H = np.zeros((n, 3, 3), np.complex128)
    d = rng.standard_normal((n, 3))
    for i in range(3):
        H[:, i, i] = d[:, i]
    for i, j in ((0, 1), (0, 2), (1, 2)):
        re = rng.standard_normal(n)
        im = rng.standard_normal(n)
        H[:, i, j] = re + 1j * im
        H[:, j, i] = re - 1j * im
    tr = np.trace(H, axis1=1, axis2=2) / 3.0
    for i in range(3):
        H[:, i, i] -= tr
    return np.ascontiguousarray(H.view(np.float64).reshape(n, 18))


def random_gauge(dims, eps, seed):
    """U = exp(i eps H) on every link, H from random_hermitian."""
    rng = np.random.default_rng(seed)
    V = volume(dims)
    H = random_hermitian(rng, 4 * V)
    return exp_field(eps, H).reshape(72 * V)


def random_spinor(dims, seed, sigma=1.0):
    rng = np.random.default_rng(seed)
    return sigma * rng.standard_normal(6 * volume(dims))


GELL_MANN = None


def gell_mann():
    """Gell-Mann matrices lambda_1..8 (Fermions.cpp:321-340)."""
    global GELL_MANN
    if GELL_MANN is None:
        g = np.zeros((8, 3, 3), np.complex128)
        g[0][0, 1] = g[0][1, 0] = 1
        g[1][0, 1] = -1j; g[1][1, 0] = 1j
        g[2][0, 0] = 1; g[2][1, 1] = -1
        g[3][0, 2] = g[3][2, 0] = 1
        g[4][0, 2] = -1j; g[4][2, 0] = 1j
        g[5][1, 2] = g[5][2, 1] = 1
        g[6][1, 2] = -1j; g[6][2, 1] = 1j
        a = 1.0 / np.sqrt(3.0)
        g[7][0, 0] = a; g[7][1, 1] = a; g[7][2, 2] = -2 * a
        GELL_MANN = g
    return GELL_MANN


def random_momenta(dims, seed):
    """P = sum_a 1/2 p_a lambda_a, p_a ~ N(0,1) (Fermions.cpp:342-360)."""
    rng = np.random.default_rng(seed)
    n = 4 * volume(dims)
    p = rng.standard_normal((n, 8))
    P = 0.5 * np.einsum("na,aij->nij", p, gell_mann())
    return np.ascontiguousarray(P.view(np.float64).reshape(18 * n))


def cold_gauge(dims):
    V = volume(dims)
    U = np.zeros((4 * V, 3, 3), np.complex128)
    U[:, 0, 0] = U[:, 1, 1] = U[:, 2, 2] = 1
    return np.ascontiguousarray(U.view(np.float64).reshape(72 * V))


# ---------------------------------------------------------------------------
# the library's seeded generators restated on the CPU (Philox-4x32-10 keyed by
# the seed, Box-Muller normals): the same fields sfh_random_gauge,
# sfh_gaussian_spinor / sfh_batch_random_rhs and sfh_random_momenta produce
# ---------------------------------------------------------------------------
def philox4x32_10(ctr, key):
    c = (ctypes.c_uint * 4)(*[int(x) & 0xFFFFFFFF for x in ctr])
    k = (ctypes.c_uint * 2)(*[int(x) & 0xFFFFFFFF for x in key])
    o = (ctypes.c_uint * 4)()
    lib().orc_philox4x32_10(c, k, o)
    return [int(x) for x in o]


def philox_normals(seed, stream, obj_id, n):
    z = np.zeros(n)
    lib().orc_gen_normals(int(seed), int(stream), int(obj_id), int(n), _d(z))
    return z


def philox_gauge(dims, eps, seed):
    U = np.zeros(72 * volume(dims))
    st = lib().orc_gen_gauge(_dims(dims), float(eps), int(seed), _d(U))
    if st != ORC_OK:
        raise OracleError(st, "philox_gauge")
    return U


def philox_spinor(dims, seed, sigma=1.0):
    out = np.zeros(6 * volume(dims))
    lib().orc_gen_spinor(_dims(dims), float(sigma), int(seed), _d(out))
    return out


def philox_momenta(dims, seed):
    P = np.zeros(72 * volume(dims))
    lib().orc_gen_momenta(_dims(dims), int(seed), _d(P))
    return P


# HEX staple steps in the reference's flat tensor layouts (combo * V + site)
def hex_gamma(level, dims, field):
    V = volume(dims)
    n = {1: 64, 2: 16, 3: 4}[level]
    out = np.zeros(n * V * 18)
    fn = {1: lib().orc_hex_gamma1, 2: lib().orc_hex_gamma2, 3: lib().orc_hex_gamma3}[level]
    fn(_dims(dims), _d(np.ascontiguousarray(field, dtype=np.float64)), _d(out))
    return out
