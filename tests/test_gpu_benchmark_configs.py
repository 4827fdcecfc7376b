"""GPU parity at the benchmark configurations, against the CPU oracle.

The solver tests elsewhere pin the operators and the CG at 8^4 and smaller;
these run the benchmark's own lattices and conditioning:

* the uneven batch's four lattices (8^4, 12^4, 16^4, 16^3x32) at eps = 1.0,
  m = 0.05, inputs from the library's seeded generators;
* the 16^4 precision grid (eps 0.3 / 1.0, m 0.1 / 0.02);
* the ill-conditioned 32^3x64 solve (eps = 1.0, m = 0.01).

Checks, all computed on the host from the downloaded device fields:

* the FP64 full-lattice CG (the reference's solve_CG_DDdagger,
  Fermions.cpp:553-617) against the oracle's CG on the same inputs: the
  iteration count to +-1 and the solution to 1e-10 relative (2-norm);
* every solution's true residual |phi - D D^dag X| / |phi| with the oracle's
  D D^dag (apply_DDdagger, Fermions.cpp:530-547): FP64 < 2 tol (the
  reference stops on its recursive residual), the mixed precisions < 1.05
  tol (they stop on the library's FP64 true residual; the 5 % covers the
  host's summation order);
* the distance of each mixed-precision solution to the oracle's solution,
  below cond(M) * 2 tol with cond(M) <= (m^2 + 16) / m^2.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-10
C4_LATTICES = [(8, 8, 8, 8), (12, 12, 12, 12), (16, 16, 16, 16), (16, 16, 16, 32)]


@pytest.fixture(scope="module")
def sfh():
    import staggered_fermions_hmc_b200 as m
    m.load_library()
    return m


def l2rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def true_resid(orc, dims, mass, U, b, x):
    return l2rel(orc.ddag(dims, mass, U, x), b)


def cond_bound(mass):
    return (mass * mass + 16.0) / (mass * mass)


@pytest.mark.parametrize("dims", C4_LATTICES, ids=["x".join(map(str, d)) for d in C4_LATTICES])
def test_c4_lattice_solves_vs_oracle(sfh, orc, dims):
    mass = 0.05
    lat = sfh.Lattice(dims, mass)
    try:
        lat.random_gauge(1.0, 1000 + dims[3])
        U = lat.download_gauge()
        phi = lat.gaussian_spinor(100000 + dims[0])
        Xo, it_o, _, st = orc.cg(dims, mass, U, phi, TOL, 40000)
        assert st == 0
        X64, i64 = lat.solve_CG_DDdagger(phi, tol=TOL, max_iter=40000, precision="f64", info=True)
        assert abs(i64["iters"] - it_o) <= 1
        assert l2rel(X64, Xo) < 1e-10
        assert true_resid(orc, dims, mass, U, phi, X64) < 2 * TOL
        for prec in ("f16", "f32", "bf16"):
            X, inf = lat.solve_CG_DDdagger(phi, tol=TOL, max_iter=40000, precision=prec, info=True)
            assert inf["status"] == 0
            assert true_resid(orc, dims, mass, U, phi, X) < 1.05 * TOL, prec
            assert l2rel(X, Xo) < cond_bound(mass) * 2 * TOL, prec
    finally:
        lat.close()


@pytest.mark.parametrize("precision", ["f16", "f64"])
def test_c4_batch_lanes_vs_oracle(sfh, orc, precision):
    """One batch holding every C4 lattice and mass, 1-3 RHS each: each lane's
    solution by the oracle's true residual (the batch solves the two parity
    blocks as separate lanes, so FP64 lanes stop on their own recursive
    residual per parity)."""
    systems = [((8, 8, 8, 8), 0.05, 3), ((12, 12, 12, 12), 0.1, 2), ((16, 16, 16, 16), 0.2, 1),
               ((16, 16, 16, 32), 0.05, 2)]
    B = sfh.Batch(systems, precision=precision)
    try:
        for k, (dims, mass, nrhs) in enumerate(systems):
            B.random_gauge(k, 1.0 if k % 2 == 0 else 0.3, 1000 + k)
            for j in range(nrhs):
                B.random_rhs(k, j, 100000 + 100 * k + j)
        B.solve(tol=TOL, max_iter=20000)
        for k, (dims, mass, nrhs) in enumerate(systems):
            U = B.gauge(k)
            for j in range(nrhs):
                X, b = B.solution(k, j), B.rhs(k, j)
                r = true_resid(orc, dims, mass, U, b, X)
                assert r < (2.0 if precision == "f64" else 1.05) * TOL, (k, j, r)
    finally:
        B.close()


C2_GRID = [(0.3, 0.1), (0.3, 0.02), (1.0, 0.1), (1.0, 0.02)]


@pytest.mark.parametrize("geps,mass", C2_GRID, ids=[f"eps{e}_m{m}" for e, m in C2_GRID])
def test_c2_grid_vs_oracle(sfh, orc, geps, mass):
    """16^4 at eps {0.3, 1.0} x m {0.1, 0.02}: FP64 against the oracle's CG;
    FP32 with 12-real and 18-real links by the oracle's true residual."""
    dims = (16, 16, 16, 16)
    lat = sfh.Lattice(dims, mass)
    try:
        lat.random_gauge(geps, 21)
        U = lat.download_gauge()
        phi = lat.gaussian_spinor(22)
        Xo, it_o, _, st = orc.cg(dims, mass, U, phi, TOL, 40000)
        assert st == 0
        X64, i64 = lat.solve_CG_DDdagger(phi, tol=TOL, max_iter=40000, precision="f64", info=True)
        assert abs(i64["iters"] - it_o) <= 1
        assert l2rel(X64, Xo) < 1e-10
        for prec in ("f32", "f32_18"):
            X, inf = lat.solve_CG_DDdagger(phi, tol=TOL, max_iter=40000, precision=prec, info=True)
            assert true_resid(orc, dims, mass, U, phi, X) < 1.05 * TOL, prec
            assert l2rel(X, Xo) < cond_bound(mass) * 2 * TOL, prec
    finally:
        lat.close()


def test_c3_ill_conditioned_solve_true_residual(sfh, orc):
    """32^3x64, eps = 1.0, m = 0.01: the 16-bit storages (FP16 and BF16 with a
    per-site scale) reach the FP64 true residual by the oracle's D D^dag, and
    stay within cond(M) * 2 tol of the FP64 solve (the oracle's own CG takes
    minutes at this size; the FP64 CG is the one pinned to it above)."""
    dims, mass = (32, 32, 32, 64), 0.01
    lat = sfh.Lattice(dims, mass)
    try:
        lat.random_gauge(1.0, 3)
        U = lat.download_gauge()
        phi = lat.gaussian_spinor(11)
        X64 = lat.solve_CG_DDdagger(phi, tol=TOL, max_iter=40000, precision="f64")
        assert true_resid(orc, dims, mass, U, phi, X64) < 2 * TOL
        for prec in ("f16", "bf16"):
            X, inf = lat.solve_CG_DDdagger(phi, tol=TOL, max_iter=40000, precision=prec, info=True)
            assert inf["status"] == 0
            assert true_resid(orc, dims, mass, U, phi, X) < 1.05 * TOL, prec
            assert l2rel(X, X64) < cond_bound(mass) * 4 * TOL, prec
    finally:
        lat.close()
