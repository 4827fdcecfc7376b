"""Pin the CPU oracle against the reference's own outputs and analytic KATs.

The fixtures in tests/golden/ were produced by the reference's unmodified
functions (tests/golden/make_golden.py).  Tolerances: bit-exact for the
integer tables; 1e-12 relative for the FP64 operators, forces, staples and
exp(iQ); 1e-11 relative for CG solutions and the trajectory (the reference
solves to a relative residual of 1e-12, so summation-order differences are
amplified by the condition number).
"""
import glob
import os

import numpy as np
import pytest

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "ref_*.npz")))


def rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def load(path):
    g = np.load(path)
    L, T, mass, tol, geps, seed, beta, eps, nsteps = g["meta"]
    return g, (int(L), int(L), int(L), int(T)), float(mass), float(tol), float(beta), float(eps), int(nsteps)


@pytest.fixture(params=GOLDEN, ids=[os.path.basename(p) for p in GOLDEN])
def golden(request):
    return load(request.param)


def test_fixtures_present():
    assert len(GOLDEN) >= 2


def test_tables_bit_exact(orc, golden):
    g, dims, *_ = golden
    V = int(np.prod(dims))
    t = orc.tables(dims)
    tab = g["tables"].reshape(5, 4 * V)
    for i, k in enumerate(["up", "dn", "bc_up", "bc_dn", "eta"]):
        assert np.array_equal(t[k], tab[i]), k


def test_dirac_operators(orc, golden):
    g, dims, mass, *_ = golden
    U, phi = g["U"], g["phi"]
    assert rel(orc.dirac(dims, mass, U, phi), g["Dphi"]) < 1e-12
    assert rel(orc.dirac(dims, mass, U, phi, dagger=True), g["Ddagphi"]) < 1e-12
    assert rel(orc.ddag(dims, mass, U, phi), g["DDdagphi"]) < 1e-12


def test_cg_and_y(orc, golden):
    g, dims, mass, tol, *_ = golden
    X, it, rsq, st = orc.cg(dims, mass, g["U"], g["phi"], tol)
    assert rel(X, g["X"]) < 1e-11
    Y = orc.dirac(dims, mass, g["U"], X, dagger=True)
    assert rel(Y, g["Y"]) < 1e-11


def test_staples_and_forces(orc, golden):
    g, dims, mass, tol, beta, *_ = golden
    U = g["U"]
    A1, A2 = orc.staples(dims, U)
    assert rel(A1, g["A1"]) < 1e-12
    assert rel(A2, g["A2"]) < 1e-12
    assert rel(orc.gauge_force(dims, beta, U), g["Fgauge"]) < 1e-12
    assert rel(orc.fermion_force(dims, U, g["X"], g["Y"]), g["Ffermion"]) < 1e-12
    assert rel(orc.full_force(dims, beta, U, g["X"], g["Y"]), g["Ffull"]) < 1e-12


def test_scalars(orc, golden):
    g, dims, mass, tol, beta, *_ = golden
    act, plaq, trp2, phix = g["scalars"]
    assert abs(orc.action(dims, beta, g["U"]) - act) <= 1e-12 * abs(act)
    assert abs(orc.avg_plaq(dims, g["U"]) - plaq) <= 1e-12 * max(abs(plaq), 1.0)
    assert abs(orc.trp2(dims, g["P"]) - trp2) <= 1e-12 * abs(trp2)
    assert abs(orc.dot(g["phi"], g["X"]) - phix) <= 1e-12 * abs(phix)


def test_expiq(orc, golden):
    g, *_ = golden
    H = g["H"]
    E = np.concatenate([orc.expiq(H[k]) for k in range(H.shape[0])])
    assert rel(E, g["expH"]) < 1e-12


def test_polyakov(orc, golden):
    g, dims, *_ = golden
    grid = orc.polyakov_grid(dims, g["U"])
    assert rel(grid, g["poly_grid"]) < 1e-12
    corr = g["poly_corr"].reshape(-1, 2)
    for r2 in (1, 2, 3):
        c = orc.polyakov_corr(dims, grid, r2)
        assert abs(c - complex(*corr[r2 - 1])) <= 1e-12 * max(abs(c), 1.0)


def test_trajectory(orc, golden):
    g, dims, mass, tol, beta, eps, nsteps = golden
    P, U, X, its = orc.leapfrog(dims, mass, beta, eps, nsteps, g["phi"], g["P"], g["U"], tol=tol)
    assert rel(U, g["traj_U"]) < 1e-11
    assert rel(P, g["traj_P"]) < 1e-11
    assert rel(X, g["traj_X"]) < 1e-10
    h = g["traj_H"]
    h1 = np.array([orc.trp2(dims, P), orc.action(dims, beta, U), orc.dot(g["phi"], X)])
    assert np.allclose(h1, h[3:], rtol=1e-10, atol=1e-9)


# ---------------------------------------------------------------------------
# analytic known-answer tests from the reference's own self-checks
# ---------------------------------------------------------------------------

@pytest.mark.parametrize("dims", [(4, 4, 4, 4), (4, 4, 4, 6), (6, 6, 6, 4)])
def test_cold_start_kats(orc, dims):
    """ai_check.cpp:172-223 (A1 = 6I, A2 = 18I), ai_check.cpp:227-333 (cold
    action = -beta (c11 6V + c12 12V)), Lattice.cpp:784-804 (plaquette 6.0)."""
    U = orc.cold_gauge(dims)
    V = int(np.prod(dims))
    A1, A2 = orc.staples(dims, U)
    eye = np.zeros((3, 3, 2))
    for i in range(3):
        eye[i, i, 0] = 1
    A1 = A1.reshape(4 * V, 3, 3, 2)
    A2 = A2.reshape(4 * V, 3, 3, 2)
    assert np.abs(A1 - 6 * eye).max() < 1e-12
    assert np.abs(A2 - 18 * eye).max() < 1e-12
    beta, c11, c12 = 4.2, 5.0 / 3.0, -1.0 / 12.0
    expected = -beta * (c11 * 6 * V + c12 * 12 * V)
    # reference criterion 1e-10 absolute at 4^4; scaled with the action's size
    assert abs(orc.action(dims, beta, U) - expected) < max(1e-10, 1e-13 * abs(expected))
    assert abs(orc.avg_plaq(dims, U) - 6.0) < 1e-12
    # cold field: the gauge force vanishes
    assert np.abs(orc.gauge_force(dims, beta, U)).max() < 1e-12


def test_unitarity_of_generated_links(orc):
    """Lattice.cpp:950-986: det U = 1 and U^dag U = I to 1e-12."""
    dims = (4, 4, 4, 4)
    U = orc.random_gauge(dims, 1.0, 5).view(np.complex128).reshape(-1, 3, 3)
    eye = np.eye(3)
    assert np.abs(np.einsum("nji,njk->nik", U.conj(), U) - eye).max() < 1e-12
    assert np.abs(np.linalg.det(U) - 1).max() < 1e-12


def test_ddag_equals_dagd_and_eo_structure(orc):
    """D D^dag = D^dag D = m^2 - K^2 and K^2 does not mix parities."""
    dims = (4, 4, 4, 6)
    mass = 0.3
    U = orc.random_gauge(dims, 0.7, 11)
    psi = orc.random_spinor(dims, 12)
    a = orc.ddag(dims, mass, U, psi)
    b = orc.dirac(dims, mass, U, orc.dirac(dims, mass, U, psi), dagger=True)
    assert rel(a, b) < 1e-13
    # keep only even sites in psi: the result must vanish on odd sites
    V = int(np.prod(dims))
    c = np.indices(dims).reshape(4, V).sum(0) % 2
    pe = psi.reshape(V, 6).copy()
    pe[c == 1] = 0
    out = orc.ddag(dims, mass, U, pe.reshape(-1)).reshape(V, 6)
    assert np.abs(out[c == 1]).max() < 1e-13


def test_gauge_force_finite_difference(orc):
    """dS/deps under U -> exp(i eps H) U equals 2 Tr(F H) (ai_check.cpp:149-166)."""
    dims = (4, 4, 4, 4)
    beta = 4.2
    U = orc.random_gauge(dims, 0.4, 21)
    F = orc.gauge_force(dims, beta, U).reshape(-1, 18)
    rng = np.random.default_rng(3)
    H = orc.random_hermitian(rng, 1)[0]
    link = 4 * 37 + 2
    h = 1e-5

    def S(e):
        Ue = U.reshape(-1, 18).copy()
        E = orc.expiq(e * H)
        m = (E.view(np.complex128).reshape(3, 3) @ Ue[link].view(np.complex128).reshape(3, 3))
        Ue[link] = m.reshape(9).view(np.float64)
        return orc.action(dims, beta, Ue.reshape(-1))

    num = (S(h) - S(-h)) / (2 * h)
    Fm = F[link].view(np.complex128).reshape(3, 3)
    Hm = H.view(np.complex128).reshape(3, 3)
    ana = 2 * np.trace(Fm @ Hm).real
    assert abs(num - ana) < 1e-6 * max(1.0, abs(ana))


def test_expiq_domain_errors(orc):
    """Fermions.cpp:848-857: anti-Hermitian input is rejected."""
    rng = np.random.default_rng(9)
    H = orc.random_hermitian(rng, 1)[0].view(np.complex128)
    with pytest.raises(orc.OracleError):
        orc.expiq((1j * H).view(np.float64))


@pytest.mark.parametrize("n_levels", [1, 3])
def test_stout_force_finite_difference(orc, n_levels):
    """Smeared-link fermion force (no reference counterpart; self-consistency):
    S(U) = phi^dag (D D^dag)^-1 phi on V = stout^n(U); under every link
    U -> exp(i eps H) U, dS/deps = sum 2 Tr(F H) with F the chain-rule force."""
    dims, mass, rho = (4, 4, 4, 4), 0.3, 0.125
    U = orc.random_gauge(dims, 0.4, 31)
    phi = orc.random_spinor(dims, 32)
    H = orc.random_momenta(dims, 33)

    def action(Uin):
        Vs = orc.stout(dims, rho, n_levels, Uin)
        X, _, _, _ = orc.cg(dims, mass, Vs, phi, 1e-14)
        return orc.dot(phi, X)

    Vs = orc.stout(dims, rho, n_levels, U)
    X, _, _, _ = orc.cg(dims, mass, Vs, phi, 1e-14)
    Y = orc.dirac(dims, mass, Vs, X, dagger=True)
    F = orc.stout_force(dims, rho, n_levels, U, orc.fermion_force(dims, Vs, X, Y))
    h = 1e-4
    num = (action(orc.link_update(dims, h, H, U)) - action(orc.link_update(dims, -h, H, U))) / (2 * h)
    Fm = F.view(np.complex128).reshape(-1, 3, 3)
    Hm = H.view(np.complex128).reshape(-1, 3, 3)
    ana = 2.0 * np.einsum("lij,lji->", Fm, Hm).real
    assert abs(num - ana) < 1e-6 * abs(ana), (num, ana)  # O(h^2) = 1e-7 observed
    # the same check without smearing (n = 0 reduces to the plain force)
    F0 = orc.stout_force(dims, rho, 0, U, orc.fermion_force(dims, U, *_xy(orc, dims, mass, U, phi)))
    assert np.allclose(F0, orc.fermion_force(dims, U, *_xy(orc, dims, mass, U, phi)), atol=1e-14)


def _xy(orc, dims, mass, U, phi):
    X, _, _, _ = orc.cg(dims, mass, U, phi, 1e-14)
    return X, orc.dirac(dims, mass, U, X, dagger=True)


def _hb_equilibrium(hist, start=30):
    """Mean plaquette over the sweeps after start and its standard error from
    the spread of independent runs."""
    m = hist[:, start:].mean(axis=1)
    return float(m.mean()), float(m.std(ddof=1) / np.sqrt(len(m)))


def test_heatbath_oracle_vs_reference_statistics(orc):
    """heatbath_update (Lattice.cpp:722-757): the reference's generator is
    unseeded, so tests/golden holds independent plaquette histories of its own
    chain (4^4 from a cold start).  The oracle's chain (colour order, seeded
    uniforms) must reach the same equilibrium plaquette at each beta."""
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "heatbath_ref_L4T4.npz"))
    dims = (4, 4, 4, 4)
    for b, beta in enumerate(g["betas"]):
        ref_mean, ref_se = _hb_equilibrium(g["plaq"][b])
        hist = []
        for seed in range(4):
            U = orc.cold_gauge(dims)
            h = []
            for sw in range(g["plaq"].shape[2]):
                U = orc.heatbath(dims, beta, U, seed=100 + seed, nsweeps=1, sweep0=sw)
                h.append(orc.avg_plaq(dims, U))
            hist.append(h)
        mean, se = _hb_equilibrium(np.array(hist))
        tol = 4.0 * np.hypot(ref_se, se) + 2e-3
        assert abs(mean - ref_mean) < tol, (beta, mean, ref_mean, tol)
    V = U.view(np.complex128).reshape(-1, 3, 3)
    assert np.abs(np.einsum("lij,lkj->lik", V, V.conj()) - np.eye(3)).max() < 1e-12


# ---------------------------------------------------------------------------
# HEX staple steps against the reference's own apply_step_1 / 3 / 5
# (Smearing.cpp:76-275, run unmodified by oracle/hex_harness.cpp; fixture
# tests/golden/hex_ref_L4T4.npz).  Their exp steps cannot run as shipped, so
# the staple steps carry the index conventions of the smearing restatement:
# which links form the decorated staples, and in which tensor slots.
# ---------------------------------------------------------------------------
HEX_GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "hex_ref_L4T4.npz")


def hex_fixture():
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
    import make_golden
    g = np.load(HEX_GOLDEN)
    m = g["meta"]
    dims = tuple(int(x) for x in m[:4])
    eps, seeds, wseed = float(m[4]), tuple(int(x) for x in m[5:8]), int(m[8])
    return g, dims, make_golden.hex_inputs(dims, eps, seeds), wseed, make_golden.hex_checksum


def check_hex_level(g, level, G, V, wseed, checksum):
    n = G.size // (18 * V)
    sites = g[f"G{level}_sites"]
    ref = g[f"G{level}_at_sites"]
    assert rel(G.reshape(n, V, 18)[:, sites, :], ref) < 1e-12
    cs = checksum(G, wseed, level)
    assert np.abs(cs - g[f"G{level}_checksum"]).max() < 1e-12 * np.abs(g[f"G{level}_checksum"]).max()


@pytest.mark.parametrize("level", [1, 2, 3])
def test_hex_staple_steps_vs_reference(orc, level):
    g, dims, (U, V1, V2), wseed, checksum = hex_fixture()
    G = orc.hex_gamma(level, dims, {1: U, 2: V1, 3: V2}[level])
    check_hex_level(g, level, G, orc.volume(dims), wseed, checksum)
