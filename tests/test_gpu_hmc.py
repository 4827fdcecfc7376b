"""GPU parity for the HMC path: staples, gauge and fermion forces, the link
update, Tr P^2 / action / plaquette, the leapfrog trajectory, the full HMC
update and link smearing.

Tolerances: per-link quantities (staples, forces, exp) 1e-12 relative
(max-norm over the field); reductions 1e-12 relative; a trajectory 1e-10
relative against the reference's own trajectory (it contains 11 CG solves at
the reference's 1e-12 tolerance); reversibility 1e-10 absolute on the links
(Fermions.cpp:947); dH(eps)/dH(eps/2) in [3.5, 4.5] (Fermions.cpp:1098).
Smearing compares with the oracle restatement: the reference's HEX cannot run
as shipped (its exp steps reject their input), but its exp-free staple steps
apply_step_1/3/5 do, and the device's staple steps are checked against their
outputs (tests/golden/hex_ref_L4T4.npz) to 1e-12.
"""
import glob
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "ref_*.npz")))


def rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def load(path):
    g = np.load(path)
    L, T, mass, tol, geps, seed, beta, eps, nsteps = g["meta"]
    return g, (int(L), int(L), int(L), int(T)), float(mass), float(tol), float(beta), float(eps), int(nsteps)


@pytest.fixture(scope="module")
def sfh():
    import staggered_fermions_hmc_b200 as m
    m.load_library()
    return m


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p) for p in GOLDEN])
def test_staples_forces_scalars_vs_reference(sfh, path):
    g, dims, mass, tol, beta, eps, nsteps = load(path)
    lat = sfh.Lattice(dims, mass, beta)
    lat.upload_gauge(g["U"])
    A1, A2 = lat.staples()
    assert rel(A1, g["A1"]) < 1e-12
    assert rel(A2, g["A2"]) < 1e-12
    assert rel(lat.compute_gauge_only_force_field(), g["Fgauge"]) < 1e-12
    assert rel(lat.compute_fermion_only_force_field(g["X"], g["Y"]), g["Ffermion"]) < 1e-12
    assert rel(lat.compute_full_force_field(g["X"], g["Y"]), g["Ffull"]) < 1e-12
    act, plaq, trp2, phix = g["scalars"]
    assert abs(lat.compute_action() - act) <= 1e-12 * abs(act)
    assert abs(lat.compute_avg_plaq() - plaq) <= 1e-12 * max(abs(plaq), 1.0)
    lat.upload_momenta(g["P"])
    assert rel(lat.download_momenta(), g["P"]) == 0.0
    assert abs(lat.compute_Tr_P2() - trp2) <= 1e-12 * abs(trp2)


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p) for p in GOLDEN])
def test_leapfrog_vs_reference(sfh, path):
    """local_initial_half_step / local_leapfrog_steps / local_final_step
    (Fermions.cpp:967-1028) from the same (U, P, phi)."""
    g, dims, mass, tol, beta, eps, nsteps = load(path)
    lat = sfh.Lattice(dims, mass, beta)
    lat.upload_gauge(g["U"])
    lat.upload_momenta(g["P"])
    X, its = lat.leapfrog(g["phi"], eps, nsteps, tol=tol, precision="f64")
    assert rel(lat.download_gauge(), g["traj_U"]) < 1e-10
    assert rel(lat.download_momenta(), g["traj_P"]) < 1e-10
    assert rel(X, g["traj_X"]) < 1e-9
    h = g["traj_H"]
    h1 = np.array([lat.compute_Tr_P2(), lat.compute_action(), float(np.dot(g["phi"], X))])
    assert np.allclose(h1, h[3:], rtol=1e-10, atol=1e-9)


@pytest.mark.parametrize("dims,geps", [((6, 6, 6, 6), 0.5), ((4, 6, 8, 10), 0.3)])
def test_forces_vs_oracle(sfh, orc, dims, geps):
    mass, beta = 0.2, 4.2
    U = orc.random_gauge(dims, geps, 61)
    X = orc.random_spinor(dims, 62)
    Y = orc.random_spinor(dims, 63)
    lat = sfh.Lattice(dims, mass, beta)
    lat.upload_gauge(U)
    assert rel(lat.compute_gauge_only_force_field(), orc.gauge_force(dims, beta, U)) < 1e-12
    assert rel(lat.compute_fermion_only_force_field(X, Y), orc.fermion_force(dims, U, X, Y)) < 1e-12
    assert abs(lat.compute_action() - orc.action(dims, beta, U)) < 1e-12 * abs(orc.action(dims, beta, U))


@pytest.mark.parametrize("forces", ["gauge", "fermion", "full"])
def test_momentum_kick_vs_oracle(sfh, orc, forces):
    """P -= dt F (Fermions.cpp:690-695) with F from the oracle's forces on
    X = (D D^dag)^-1 phi, Y = D^dag X."""
    dims, mass, beta, dt = (4, 4, 6, 8), 0.2, 4.2, 0.05
    U = orc.random_gauge(dims, 0.4, 65)
    P = orc.random_momenta(dims, 66)
    phi = orc.random_spinor(dims, 67)
    lat = sfh.Lattice(dims, mass, beta)
    lat.upload_gauge(U)
    lat.upload_momenta(P)
    X, its = lat.momentum_kick(dt, phi, forces=forces, tol=1e-13)
    F = np.zeros_like(P)
    if forces != "fermion":
        F += orc.gauge_force(dims, beta, U)
    if forces != "gauge":
        Xo, _, _, _ = orc.cg(dims, mass, U, phi, 1e-13)
        Yo = orc.dirac(dims, mass, U, Xo, dagger=True)
        assert rel(X, Xo) < 1e-10 and its > 0
        F += orc.fermion_force(dims, U, Xo, Yo)
    else:
        assert X is None and its == 0
    assert rel(lat.download_momenta(), P - dt * F) < 1e-11


def test_staged_leapfrog_equals_fused(sfh, orc):
    """kick(eps/2), [update(eps), kick(eps)] x (N-1), update(eps), kick(eps/2)
    through the single-step entries reproduces sfh_leapfrog exactly."""
    dims, mass, beta, eps, n = (4, 4, 4, 8), 0.2, 4.2, 0.05, 3
    U = orc.random_gauge(dims, 0.3, 68)
    P = orc.random_momenta(dims, 69)
    phi = orc.random_spinor(dims, 70)
    a = sfh.Lattice(dims, mass, beta)
    a.upload_gauge(U)
    a.upload_momenta(P)
    Xa, _ = a.leapfrog(phi, eps, n, tol=1e-12)
    b = sfh.Lattice(dims, mass, beta)
    b.upload_gauge(U)
    b.upload_momenta(P)
    b.momentum_kick(0.5 * eps, phi, tol=1e-12)
    for _ in range(n - 1):
        b.link_update(eps, check=False)
        b.momentum_kick(eps, phi, tol=1e-12)
    b.link_update(eps, check=False)
    Xb, _ = b.momentum_kick(0.5 * eps, phi, tol=1e-12)
    assert np.array_equal(a.download_gauge(), b.download_gauge())
    assert np.array_equal(a.download_momenta(), b.download_momenta())
    assert np.array_equal(Xa, Xb)


def test_link_update_vs_oracle(sfh, orc):
    dims = (4, 4, 4, 8)
    U = orc.random_gauge(dims, 0.7, 71)
    P = orc.random_momenta(dims, 72)
    lat = sfh.Lattice(dims, 0.1)
    lat.upload_gauge(U)
    lat.upload_momenta(P)
    lat.link_update(0.05, check=True)
    assert rel(lat.download_gauge(), orc.link_update(dims, 0.05, P, U)) < 1e-13


def test_link_update_rejects_non_hermitian_momentum(sfh, orc):
    """Fermions.cpp:712-716: a non-Hermitian P_pre is an error."""
    dims = (4, 4, 4, 4)
    U = orc.random_gauge(dims, 0.3, 73)
    P = orc.random_momenta(dims, 74)
    P[1] += 0.5  # imaginary part of P_00 on one link: no longer Hermitian
    lat = sfh.Lattice(dims, 0.1)
    lat.upload_gauge(U)
    lat.upload_momenta(P)
    with pytest.raises(sfh.SfhError) as e:
        lat.link_update(0.1, check=True)
    assert e.value.status == sfh.SFH_ERR_NOT_HERMITIAN


def test_cold_start_kats_on_gpu(sfh, orc):
    """ai_check.cpp:172-333, Lattice.cpp:784-804 on the GPU path."""
    dims = (4, 4, 4, 6)
    V = int(np.prod(dims))
    lat = sfh.Lattice(dims, 0.1, 4.2)
    lat.upload_gauge(orc.cold_gauge(dims))
    A1, A2 = lat.staples()
    eye = np.zeros((3, 3, 2))
    for i in range(3):
        eye[i, i, 0] = 1
    assert np.abs(A1.reshape(-1, 3, 3, 2) - 6 * eye).max() < 1e-12
    assert np.abs(A2.reshape(-1, 3, 3, 2) - 18 * eye).max() < 1e-12
    c11, c12 = 5.0 / 3.0, -1.0 / 12.0
    assert abs(lat.compute_action() + 4.2 * (c11 * 6 * V + c12 * 12 * V)) < 1e-10
    assert abs(lat.compute_avg_plaq() - 6.0) < 1e-12
    assert np.abs(lat.compute_gauge_only_force_field()).max() < 1e-12


def test_reversibility(sfh, orc):
    """Fermions.cpp:908-955: forward, flip P, backward returns to U within 1e-10."""
    dims = (4, 4, 4, 4)
    U = orc.random_gauge(dims, 0.2, 81)
    P = orc.random_momenta(dims, 82)
    phi = orc.random_spinor(dims, 83)
    lat = sfh.Lattice(dims, 0.5, 4.2)
    lat.upload_gauge(U)
    lat.upload_momenta(P)
    lat.leapfrog(phi, 0.02, 10, tol=1e-14)
    lat.upload_momenta(-lat.download_momenta())
    lat.leapfrog(phi, 0.02, 10, tol=1e-14)
    assert np.abs(lat.download_gauge() - U).max() < 1e-10
    assert np.abs(lat.download_momenta() + P).max() < 1e-9


def test_delta_h_step_scaling(sfh, orc):
    """Fermions.cpp:1061-1108 (with a consistent H): dH(eps)/dH(eps/2) ~ 4."""
    dims = (4, 4, 4, 4)
    U = orc.random_gauge(dims, 0.15, 91)
    P = orc.random_momenta(dims, 92)
    phi = orc.random_spinor(dims, 93)
    lat = sfh.Lattice(dims, 0.5, 4.2)

    def dH(eps, n):
        lat.upload_gauge(U)
        lat.upload_momenta(P)
        X0 = lat.solve_CG_DDdagger(phi, tol=1e-14)
        h0 = lat.compute_Tr_P2() + lat.compute_action() + float(np.dot(phi, X0))
        X, _ = lat.leapfrog(phi, eps, n, tol=1e-14)
        h1 = lat.compute_Tr_P2() + lat.compute_action() + float(np.dot(phi, X))
        return h1 - h0

    d1 = dH(0.02, 10)
    d2 = dH(0.01, 20)
    ratio = abs(d1) / abs(d2)
    assert 3.5 < ratio < 4.5, (d1, d2, ratio)


@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_hmc_trajectory(sfh, orc, precision):
    """single_sweep_monte_carlo_update_WITH_FERMIONS: H bookkeeping and the
    Metropolis decision are self-consistent, and a rejected trajectory leaves
    the field unchanged."""
    dims = (4, 4, 4, 4)
    U = orc.random_gauge(dims, 0.3, 101)
    lat = sfh.Lattice(dims, 0.1, 4.2)
    lat.upload_gauge(U)
    info = lat.hmc_trajectory(0.1, 10, seed=5, tol=1e-10, precision=precision)
    assert info["status"] == 0
    dH = sum(info["H_final"]) - sum(info["H_initial"])
    assert abs(dH - info["dH"]) < 1e-8 * max(1.0, abs(dH))
    assert info["accepted"] == (info["uniform"] < np.exp(-info["dH"]))
    assert info["solves"] == 12  # initial solve + N + 1 force solves
    U1 = lat.download_gauge()
    if not info["accepted"]:
        assert np.array_equal(U1, U)
    assert abs(lat.compute_avg_plaq() - info["plaquette"]) < 1e-14


def test_hmc_trajectory_accepts_small_steps(sfh, orc):
    dims = (4, 4, 4, 4)
    lat = sfh.Lattice(dims, 0.5, 4.2)
    lat.upload_gauge(orc.random_gauge(dims, 0.05, 111))
    info = lat.hmc_trajectory(0.005, 10, seed=9, tol=1e-12)
    assert info["status"] == 0
    assert abs(info["dH"]) < 0.1


@pytest.mark.parametrize("dims", [(4, 4, 4, 4), (4, 4, 6, 8)])
def test_stout_vs_oracle(sfh, orc, dims):
    U = orc.random_gauge(dims, 0.3, 121)
    lat = sfh.Lattice(dims, 0.1)
    lat.upload_gauge(U)
    lat.smear_stout(0.125, 4)
    assert rel(lat.download_gauge(), orc.stout(dims, 0.125, 4, U)) < 1e-12


@pytest.mark.parametrize("dims", [(4, 4, 4, 4), (4, 4, 6, 8)])
def test_hex_vs_oracle(sfh, orc, dims):
    U = orc.random_gauge(dims, 0.3, 131)
    lat = sfh.Lattice(dims, 0.1)
    lat.upload_gauge(U)
    lat.Apply_HEX_smearing()
    assert rel(lat.download_gauge(), orc.hex_smear(dims, U)) < 1e-12
    lat.upload_gauge(U)
    lat.Apply_4HEX_smearing()
    ref = U
    for _ in range(4):
        ref = orc.hex_smear(dims, ref)
    assert rel(lat.download_gauge(), ref) < 1e-11


@pytest.mark.parametrize("level", [1, 2, 3])
def test_hex_staple_steps_vs_reference(sfh, orc, level):
    """apply_step_1 / 3 / 5 (Smearing.cpp:76-275) on the device against the
    reference's own outputs on the same seeded inputs."""
    from test_oracle_golden import check_hex_level, hex_fixture
    g, dims, (U, V1, V2), wseed, checksum = hex_fixture()
    lat = sfh.Lattice(dims, 0.1)
    try:
        G = lat.hex_staples(level, {1: U, 2: V1, 3: V2}[level])
    finally:
        lat.close()
    check_hex_level(g, level, G, orc.volume(dims), wseed, checksum)


def test_smeared_links_stay_special_unitary(sfh, orc):
    dims = (4, 4, 4, 4)
    lat = sfh.Lattice(dims, 0.1)
    lat.upload_gauge(orc.random_gauge(dims, 1.0, 141))
    lat.Apply_4HEX_smearing()
    lat.smear_stout(0.125, 4)
    M = lat.download_gauge().view(np.complex128).reshape(-1, 3, 3)
    assert np.abs(np.einsum("nji,njk->nik", M.conj(), M) - np.eye(3)).max() < 1e-12
    assert np.abs(np.linalg.det(M) - 1).max() < 1e-12


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p) for p in GOLDEN])
def test_polyakov_vs_reference(sfh, path):
    """precompute_polyakov_grid and correlator_over_fixed_distance_fast
    (Lattice.cpp:869-948) against the reference's outputs."""
    g, dims, mass, tol, beta, eps, nsteps = load(path)
    lat = sfh.Lattice(dims, mass, beta)
    lat.upload_gauge(g["U"])
    grid = lat.precompute_polyakov_grid()
    assert rel(grid.view(np.float64), g["poly_grid"]) < 1e-12
    corr = g["poly_corr"].reshape(-1, 2)
    for r2 in (1, 2, 3):
        c = lat.correlator_over_fixed_distance(r2)
        assert abs(c - complex(*corr[r2 - 1])) <= 1e-12 * max(abs(c), 1.0)
        cg = lat.correlator_over_fixed_distance_fast(grid, r2)
        assert cg == c


def test_checkpoint_round_trip_is_byte_exact(sfh, orc, tmp_path):
    """save_all_lattice_configs / load_all_lattice_configs (Lattice.cpp:810-847):
    the file is the reference's raw double array."""
    dims = (4, 4, 4, 6)
    U = orc.random_gauge(dims, 0.4, 151)
    lat = sfh.Lattice(dims, 0.1)
    lat.upload_gauge(U)
    path = tmp_path / "final_lattice_configs.bin"
    lat.save_lattice_config(str(path))
    assert path.read_bytes() == U.astype("<f8").tobytes()
    lat2 = sfh.Lattice(dims, 0.1)
    lat2.load_lattice_config(str(path))
    assert np.array_equal(lat2.download_gauge(), U)
    with pytest.raises(sfh.SfhError) as e:
        lat2.load_lattice_config(str(tmp_path / "missing.bin"))
    assert e.value.status == sfh.SFH_ERR_IO


# --- stout-smeared fermion links (no counterpart in the reference) --------
@pytest.mark.parametrize("n_levels", [1, 3])
def test_smeared_fermion_force_vs_oracle(sfh, orc, n_levels):
    """GPU chain-rule force vs the oracle's (itself checked by finite
    differences in test_oracle_golden::test_stout_force_finite_difference)."""
    dims, mass, rho = (4, 4, 6, 8), 0.3, 0.125
    U = orc.random_gauge(dims, 0.4, 161)
    phi = orc.random_spinor(dims, 162)
    lat = sfh.Lattice(dims, mass, 4.2)
    lat.upload_gauge(U)
    lat.set_fermion_smearing(rho, n_levels)
    F, X = lat.smeared_fermion_force(phi, tol=1e-13)
    Vs = orc.stout(dims, rho, n_levels, U)
    Xo, _, _, _ = orc.cg(dims, mass, Vs, phi, 1e-13)
    Yo = orc.dirac(dims, mass, Vs, Xo, dagger=True)
    Fo = orc.stout_force(dims, rho, n_levels, U, orc.fermion_force(dims, Vs, Xo, Yo))
    assert rel(X, Xo) < 1e-10
    assert rel(F, Fo) < 1e-10
    assert np.array_equal(lat.download_gauge(), U)  # the thin field is left as it was


def test_smeared_leapfrog_reversible_and_second_order(sfh, orc):
    """With smeared fermion links the integrator stays reversible and
    dH(eps)/dH(eps/2) ~ 4 (force consistent with the action)."""
    dims, mass, rho, nl = (4, 4, 4, 4), 0.5, 0.125, 2
    U = orc.random_gauge(dims, 0.15, 171)
    P = orc.random_momenta(dims, 172)
    phi = orc.random_spinor(dims, 173)
    lat = sfh.Lattice(dims, mass, 4.2)
    lat.set_fermion_smearing(rho, nl)
    lat.upload_gauge(U)
    lat.upload_momenta(P)
    lat.leapfrog(phi, 0.02, 10, tol=1e-14)
    lat.upload_momenta(-lat.download_momenta())
    lat.leapfrog(phi, 0.02, 10, tol=1e-14)
    assert np.abs(lat.download_gauge() - U).max() < 1e-10
    assert np.abs(lat.download_momenta() + P).max() < 1e-9

    def dH(eps, n):
        lat.upload_gauge(U)
        lat.upload_momenta(P)
        _, X0 = lat.smeared_fermion_force(phi, tol=1e-14)
        h0 = lat.compute_Tr_P2() + lat.compute_action() + float(np.dot(phi, X0))
        X, _ = lat.leapfrog(phi, eps, n, tol=1e-14)
        h1 = lat.compute_Tr_P2() + lat.compute_action() + float(np.dot(phi, X))
        return h1 - h0

    d1, d2 = dH(0.02, 10), dH(0.01, 20)
    assert 3.5 < abs(d1) / abs(d2) < 4.5, (d1, d2)


def test_smeared_hmc_trajectory_accepts_small_steps(sfh, orc):
    dims = (4, 4, 4, 4)
    lat = sfh.Lattice(dims, 0.3, 4.2)
    lat.upload_gauge(orc.random_gauge(dims, 0.05, 181))
    lat.set_fermion_smearing(0.125, 4)
    info = lat.hmc_trajectory(0.005, 10, seed=77, tol=1e-12)
    assert info["status"] == 0
    assert abs(info["dH"]) < 0.1  # the same bound as the thin-link trajectory
    assert np.isfinite(info["plaquette"])


# --- heatbath (Lattice.cpp:722-757, SU3_Sampling.cpp) --------------------
@pytest.mark.parametrize("dims", [(4, 4, 4, 4), (4, 4, 8, 8)])
def test_heatbath_vs_oracle(sfh, orc, dims):
    """Same colour order and the same seeded uniforms: the GPU sweeps equal the
    oracle's to rounding."""
    U = orc.random_gauge(dims, 0.6, 191)
    lat = sfh.Lattice(dims, 0.1, 4.2)
    lat.upload_gauge(U)
    plaq, act = lat.heatbath_update(n_sweeps=2, seed=17, sweep0=3)
    ref = orc.heatbath(dims, 4.2, U, seed=17, nsweeps=2, sweep0=3)
    assert rel(lat.download_gauge(), ref) < 1e-12
    V = int(np.prod(dims))
    assert abs(plaq - orc.avg_plaq(dims, ref) / 6.0) < 1e-12
    assert abs(act - orc.action(dims, 4.2, ref) / V) < 1e-10 * max(1.0, abs(act))


def test_heatbath_equilibrium_vs_reference(sfh, orc):
    """The GPU chain reaches the reference's equilibrium plaquette (its
    recorded, unseeded chains in tests/golden) at beta 2.0 and 4.2."""
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "heatbath_ref_L4T4.npz"))
    dims = (4, 4, 4, 4)
    nsw = g["plaq"].shape[2]
    for b, beta in enumerate(g["betas"]):
        m = g["plaq"][b][:, 30:].mean(axis=1)
        ref_mean, ref_se = m.mean(), m.std(ddof=1) / np.sqrt(len(m))
        means = []
        for seed in range(8):
            lat = sfh.Lattice(dims, 0.1, beta)
            lat.upload_gauge(orc.cold_gauge(dims))
            h = [lat.heatbath_update(1, seed=900 + seed, sweep0=sw)[0] * 6.0 for sw in range(nsw)]
            means.append(np.mean(h[30:]))
            lat.close()
        mean, se = np.mean(means), np.std(means, ddof=1) / np.sqrt(len(means))
        assert abs(mean - ref_mean) < 4.0 * np.hypot(ref_se, se) + 2e-3, (beta, mean, ref_mean)


def test_heatbath_rejects_extents_not_multiple_of_four(sfh, orc):
    lat = sfh.Lattice((4, 4, 4, 6), 0.1, 4.2)
    with pytest.raises(sfh.SfhError) as e:
        lat.heatbath_update(1)
    assert e.value.status == sfh.SFH_ERR_INVALID


# --- Hasenbusch pair (no counterpart in the reference) --------------------
@pytest.mark.parametrize("precision,tol,bound", [("f64", 1e-13, 1e-10), ("f16", 1e-11, 1e-7)])
def test_hasenbusch_force_vs_oracle(sfh, orc, precision, tol, bound):
    """P -= dt F with F = F_f(X_h, Y_h) + (m_h^2 - m^2) F_f(X, Y), X_h solved at
    the heavy mass, X at the light one: the two solves run as one system with
    two right-hand sides, each lane at its own mass (FP64, and FP16 with FP64
    reliable updates, whose solutions sit within cond(M) tol of the oracle's)."""
    dims, m, mh, beta, dt = (4, 4, 4, 8), 0.1, 0.4, 4.2, 0.05
    U = orc.random_gauge(dims, 0.4, 201)
    phi = orc.random_spinor(dims, 202)
    phih = orc.random_spinor(dims, 203)
    lat = sfh.Lattice(dims, m, beta)
    lat.upload_gauge(U)
    lat.upload_momenta(np.zeros(72 * int(np.prod(dims))))
    lat.set_hasenbusch(mh, phih)
    lat.momentum_kick(dt, phi, forces="fermion", tol=tol, precision=precision)
    Xh, _, _, _ = orc.cg(dims, mh, U, phih, 1e-13)
    Xr, _, _, _ = orc.cg(dims, m, U, phi, 1e-13)
    F = orc.fermion_force(dims, U, Xh, orc.dirac(dims, mh, U, Xh, dagger=True)) + \
        (mh * mh - m * m) * orc.fermion_force(dims, U, Xr, orc.dirac(dims, m, U, Xr, dagger=True))
    assert rel(lat.download_momenta(), -dt * F) < bound


@pytest.mark.parametrize("smear", [0, 2])
def test_hasenbusch_trajectory_second_order(sfh, orc, smear):
    """dH(eps)/dH(eps/2) ~ 4 for the two-pseudofermion action (and on smeared
    links), from the same field and seed."""
    dims = (4, 4, 4, 4)
    U = orc.random_gauge(dims, 0.15, 211)
    lat = sfh.Lattice(dims, 0.1, 4.2)
    lat.set_hasenbusch(0.4)
    if smear:
        lat.set_fermion_smearing(0.125, smear)

    def dH(eps, n):
        lat.upload_gauge(U)
        return lat.hmc_trajectory(eps, n, seed=31, tol=1e-14)["dH"]

    d1, d2 = dH(0.04, 5), dH(0.02, 10)
    assert 3.5 < abs(d1) / abs(d2) < 4.5, (d1, d2)


def test_kernel_timing_leaves_fields_unchanged(sfh, orc):
    """sfh_kernel_timing times every HMC kernel on the context's fields and
    leaves its links and momenta as they were (zero kicks, scratch copies)."""
    dims = (8, 8, 8, 8)
    lat = sfh.Lattice(dims, 0.1)
    try:
        U = orc.random_gauge(dims, 0.5, 151)
        P = orc.random_momenta(dims, 152)
        lat.upload_gauge(U)
        lat.upload_momenta(P)
        for name in lat.HMC_KERNELS:
            ms = lat.kernel_timing(name, nrep=3)
            assert 0.0 < ms < 1e3, name
        assert np.array_equal(lat.download_gauge(), U)
        assert np.array_equal(lat.download_momenta(), P)
    finally:
        lat.close()
