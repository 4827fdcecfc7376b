"""GPU parity: Dslash / D / D^dag / D D^dag and the CG solvers against the
reference's own outputs (tests/golden) and the CPU oracle.

Tolerances (FP64 path): operators 1e-12 relative (max-norm); the FP64
full-lattice CG, which runs the reference's algorithm, matches the reference
solution to 1e-11 and its iteration count to +-1.  Mixed-precision solvers
stop on an FP64 true residual: |b - D D^dag x| / |b| < tol is checked in
FP64 on the host, and the solution agrees with a tight FP64 oracle solve to
100 * tol * cond-bound (see each test).
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
    return g, (int(L), int(L), int(L), int(T)), float(mass), float(tol), float(beta)


@pytest.fixture(scope="module")
def sfh():
    import staggered_fermions_hmc_b200 as m
    m.load_library()
    return m


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p) for p in GOLDEN])
def test_operators_vs_reference(sfh, path):
    g, dims, mass, tol, beta = load(path)
    lat = sfh.Lattice(dims, mass, beta)
    lat.upload_gauge(g["U"])
    assert rel(lat.download_gauge(), g["U"]) == 0.0
    assert rel(lat.apply_dirac_operator(g["phi"]), g["Dphi"]) < 1e-12
    assert rel(lat.apply_dirac_dagger(g["phi"]), g["Ddagphi"]) < 1e-12
    assert rel(lat.apply_DDdagger(g["phi"]), g["DDdagphi"]) < 1e-12


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p) for p in GOLDEN])
def test_fp64_cg_vs_reference(sfh, orc, path):
    g, dims, mass, tol, beta = load(path)
    lat = sfh.Lattice(dims, mass, beta)
    lat.upload_gauge(g["U"])
    X, info = lat.solve_CG_DDdagger(g["phi"], tol=tol, precision="f64", info=True)
    assert rel(X, g["X"]) < 1e-11
    _, it_ref, _, _ = orc.cg(dims, mass, g["U"], g["phi"], tol)
    assert abs(info["iters"] - it_ref) <= 1
    Y = lat.solve_Y_field(X)
    assert rel(Y, g["Y"]) < 1e-11


@pytest.mark.parametrize("dims,mass,geps", [((8, 8, 8, 8), 0.1, 0.3), ((4, 6, 8, 10), 0.25, 1.0)])
def test_operators_vs_oracle(sfh, orc, dims, mass, geps):
    U = orc.random_gauge(dims, geps, 31)
    psi = orc.random_spinor(dims, 32)
    lat = sfh.Lattice(dims, mass)
    lat.upload_gauge(U)
    assert rel(lat.apply_dirac_operator(psi), orc.dirac(dims, mass, U, psi)) < 1e-12
    assert rel(lat.apply_dirac_dagger(psi), orc.dirac(dims, mass, U, psi, dagger=True)) < 1e-12
    assert rel(lat.apply_DDdagger(psi), orc.ddag(dims, mass, U, psi)) < 1e-12


@pytest.mark.parametrize("storage,tol", [(0, 1e-14), (5, 1e-14), (1, 1e-6), (3, 1e-6), (2, 2e-3), (4, 1.5e-2),
                                         (6, 2e-3), (7, 1.5e-2)])
def test_dslash_storage_formats_vs_oracle(sfh, orc, storage, tol):
    """The standalone Dslash in each storage format (the kernels the bench's
    Dslash GB/s times) against the oracle's hopping term K = D - m, within
    the format's rounding (relative 2-norm; per element FP32 ~6e-8, FP16
    ~2.4e-4, BF16 ~2e-3 of the site's largest component)."""
    dims, mass = (8, 8, 8, 12), 0.1
    U = orc.random_gauge(dims, 1.0, 51)
    psi = orc.random_spinor(dims, 52)
    lat = sfh.Lattice(dims, mass)
    try:
        lat.upload_gauge(U)
        K = orc.dirac(dims, mass, U, psi) - mass * psi
        out = lat.dslash_storage(storage, psi)
        assert np.linalg.norm(out - K) / np.linalg.norm(K) < tol
    finally:
        lat.close()


@pytest.mark.parametrize("dims", [(8, 8, 8, 12), (4, 6, 8, 10), (6, 4, 4, 2), (16, 16, 16, 32), (12, 6, 10, 64)])
def test_dslash_time_staged_bit_identical(sfh, orc, dims):
    """The 16-bit Dslash with each block's time and z neighbours staged in
    shared memory by one bulk copy (storages 6, 7) gives exactly the result
    of the unstaged kernel (2, 4): same operands in the same order.  The
    shapes cover tiles whose staged range is clipped at both ends of the
    parity (Vh not a multiple of 256), Lt = 2 (a time hop that wraps onto
    the same line), Lt = 64, and z wraps that fall back to global loads."""
    mass = 0.1
    U = orc.random_gauge(dims, 1.0, 61)
    psi = orc.random_spinor(dims, 62)
    lat = sfh.Lattice(dims, mass)
    try:
        lat.upload_gauge(U)
        for plain, staged in ((2, 6), (4, 7)):
            a = lat.dslash_storage(plain, psi)
            b = lat.dslash_storage(staged, psi)
            assert np.array_equal(a, b), (plain, staged)
    finally:
        lat.close()


def test_dslash_staging_wait_runs_out_and_the_context_stays_usable(sfh, orc):
    """The staged Dslash's waits are bounded.  With the test hook on, every
    block announces 16 bytes more on its barrier than its bulk copy
    delivers: the copy lands, the barrier never completes, each wait gives
    up after its bound, and the call reports SFH_ERR_TIMEOUT (no GPU fault:
    no copy is left in flight).  With the hook off the next call succeeds
    and equals the unstaged kernel's result."""
    dims, mass = (4, 4, 4, 8), 0.1  # two blocks: one 256-site tile per parity
    U = orc.random_gauge(dims, 1.0, 71)
    psi = orc.random_spinor(dims, 72)
    lat = sfh.Lattice(dims, mass)
    try:
        lat.upload_gauge(U)
        with pytest.raises(sfh.SfhError) as e:
            lat.set_staging_fault(16)
            lat.dslash_storage(6, psi)
        assert e.value.status == sfh.SFH_ERR_TIMEOUT
        lat.set_staging_fault(0)
        assert np.array_equal(lat.dslash_storage(6, psi), lat.dslash_storage(2, psi))
    finally:
        lat.close()


def true_resid(orc, dims, mass, U, b, x):
    r = b - orc.ddag(dims, mass, U, x)
    return float(np.linalg.norm(r) / np.linalg.norm(b))


@pytest.mark.parametrize("precision", ["f64", "f32", "f16", "f32_18", "bf16"])
def test_cg_precisions_true_residual(sfh, orc, precision):
    dims, mass = (8, 8, 8, 8), 0.1
    U = orc.random_gauge(dims, 0.3, 41)
    b = orc.random_spinor(dims, 42)
    lat = sfh.Lattice(dims, mass)
    lat.upload_gauge(U)
    tol = 1e-10
    X, info = lat.solve_CG_DDdagger(b, tol=tol, precision=precision, info=True)
    assert info["status"] == 0
    assert true_resid(orc, dims, mass, U, b, X) < (1.01 if precision == "f64" else 1.0) * tol * 1.5
    Xref, _, _, _ = orc.cg(dims, mass, U, b, 1e-13)
    # |x - x*| / |x*| <= cond(M) * resid; cond <= (m^2 + 4) / m^2 = 401 here
    assert np.linalg.norm(X - Xref) / np.linalg.norm(Xref) < 401 * tol * 2
    if precision != "f64":
        assert info["reliable_updates"] >= 1


def test_cg_zero_rhs_returns_zero(sfh, orc):
    """Fermions.cpp:562-564: |phi|^2 < 1e-28 returns X = 0."""
    dims = (4, 4, 4, 4)
    lat = sfh.Lattice(dims, 0.1)
    lat.upload_gauge(orc.random_gauge(dims, 0.3, 1))
    X = lat.solve_CG_DDdagger(np.zeros(6 * 256), precision="f64")
    assert np.all(X == 0)


def test_cg_noconv_raises(sfh, orc):
    """Fermions.cpp:609-614: non-convergence is an error, not a silent result."""
    dims = (4, 4, 4, 4)
    lat = sfh.Lattice(dims, 0.05)
    lat.upload_gauge(orc.random_gauge(dims, 1.0, 2))
    b = orc.random_spinor(dims, 3)
    for prec in ("f64", "f32"):
        with pytest.raises(sfh.SfhError) as e:
            lat.solve_CG_DDdagger(b, tol=1e-12, max_iter=5, precision=prec)
        assert e.value.status == sfh.SFH_ERR_NOCONV


def test_invalid_dims_rejected(sfh):
    with pytest.raises(sfh.SfhError) as e:
        sfh.Lattice((4, 4, 4, 5), 0.1)
    assert e.value.status == sfh.SFH_ERR_INVALID


@pytest.mark.parametrize("precision", ["f64", "f32", "f16", "f32_18", "bf16"])
def test_batch_uneven_systems(sfh, orc, precision):
    systems = [((4, 4, 4, 4), 0.2, 2), ((6, 6, 6, 8), 0.05, 3), ((8, 8, 8, 4), 0.1, 1),
               ((4, 4, 8, 8), 0.1, 5)]
    tol = 1e-10
    B = sfh.Batch(systems, precision=precision)
    data = []
    for k, (dims, mass, nrhs) in enumerate(systems):
        U = orc.random_gauge(dims, 0.3 if k % 2 == 0 else 1.0, 100 + k)
        B.set_gauge(k, U)
        bs = [orc.random_spinor(dims, 200 + 10 * k + j) for j in range(nrhs)]
        for j, b in enumerate(bs):
            B.set_rhs(k, j, b)
        data.append((U, bs))
    B.solve(tol=tol, max_iter=20000)
    for k, (dims, mass, nrhs) in enumerate(systems):
        U, bs = data[k]
        for j in range(nrhs):
            X = B.solution(k, j)
            info = B.info(k, j)
            assert info["status"] == 0
            r = true_resid(orc, dims, mass, U, bs[j], X)
            assert r < 1.5 * tol, (k, j, r, info)
            assert abs(B.true_residual(k, j) - r) < 1e-3 * tol + 1e-3 * r
            out = np.full(X.size, np.nan)
            assert B.solution(k, j, out=out) is out
            assert np.array_equal(out, X)


def test_batch_full_lattice_matches_single(sfh, orc):
    """Full-lattice batch lanes run the same algorithm as sfh_cg_solve(F64)."""
    g, dims, mass, tol, beta = load(GOLDEN[0])
    B = sfh.Batch([(dims, mass, 2)], precision="f64", full_lattice=True)
    B.set_gauge(0, g["U"])
    B.set_rhs(0, 0, g["phi"])
    B.set_rhs(0, 1, 2.0 * g["phi"])
    B.solve(tol=tol)
    assert rel(B.solution(0, 0), g["X"]) < 1e-11
    assert rel(B.solution(0, 1), 2.0 * g["X"]) < 1e-11


def test_batch_rhs_block_widths_agree(sfh, orc):
    """The RHS-block width, the tiles per block, link staging and where the
    reliable updates run (inside the hop kernels or in the lane-list kernels,
    stages 4 and 5) change scheduling only, not results (bit-identical
    solutions)."""
    systems = [((4, 4, 4, 8), 0.1, 6)]
    U = orc.random_gauge(systems[0][0], 0.5, 7)
    out = []
    for w, tiles, stage in ((1, 1, False), (2, 2, True), (4, 3, False), (8, 4, True), (2, 1, True), (2, 4, 4),
                            (4, 2, 5)):
        B = sfh.Batch(systems, precision="f32")
        B.set_schedule(w, tiles, stage)
        assert B.schedule() == (w, tiles, stage)
        B.set_gauge(0, U)
        for j in range(6):
            B.set_rhs(0, j, orc.random_spinor(systems[0][0], 300 + j))
        B.solve(tol=1e-10)
        out.append(np.concatenate([B.solution(0, j) for j in range(6)]))
    for o in out[1:]:
        assert np.array_equal(o, out[0])


def test_batch_split_hop_widths_agree(sfh, orc):
    """FP16 storage: the two hop kernels in groups of different widths (the
    first hop in fours, the second in twos) give the solutions of equal
    widths bit for bit; the solution passes the oracle's true residual."""
    systems = [((4, 4, 4, 8), 0.1, 5), ((6, 6, 6, 6), 0.05, 3)]
    fields = [orc.random_gauge(d, 0.5, 40 + k) for k, (d, m, n) in enumerate(systems)]
    out = []
    for w1, w2, stage in ((2, 2, 4), (4, 2, 4), (4, 4, 4), (4, 2, 5), (1, 1, 0)):
        B = sfh.Batch(systems, precision="f16")
        B.set_schedule(w2, 2, stage)
        B.set_hop_widths(w1, w2)
        assert B.hop_widths() == (w1, w2)
        for k, (d, m, n) in enumerate(systems):
            B.set_gauge(k, fields[k])
            for j in range(n):
                B.set_rhs(k, j, orc.random_spinor(d, 600 + 10 * k + j))
        B.solve(tol=1e-10)
        out.append([B.solution(k, j) for k, (d, m, n) in enumerate(systems) for j in range(n)])
    for o in out[1:]:
        assert all(np.array_equal(a, b) for a, b in zip(o, out[0]))
    d, m, n = systems[1]
    b = orc.random_spinor(d, 600 + 10 + 2)  # system 1, RHS 2: after system 0's five
    r = b - orc.ddag(d, m, fields[1], out[1][5 + 2])
    assert np.linalg.norm(r) / np.linalg.norm(b) < 1.5e-10


def test_batch_neighbour_staging_bit_identical(sfh, orc):
    """Schedule 6 (FP16: schedule 4 with each tile's time and z neighbours
    staged in shared memory by bulk copies, double-buffered over the work
    item's tiles) gives schedule 4's solutions bit for bit, for hop widths
    1 to 4 and 1, 2 or 4 tiles per item, in the graph solve and the timed
    solve.  The systems cover a partial last tile (Vh not a multiple of
    256), Lt = 2, and Lt = 64 (the widest staged range of the batch); FP32
    storage with schedule 6 runs schedule 4."""
    systems = [((4, 4, 4, 8), 0.1, 5), ((6, 6, 6, 6), 0.05, 3), ((4, 6, 8, 2), 0.2, 2), ((6, 4, 4, 64), 0.1, 2)]
    fields = [orc.random_gauge(d, 0.5 + 0.25 * (k % 2), 80 + k) for k, (d, m, n) in enumerate(systems)]

    def run(prec, w1, w2, tiles, stage, timed=False):
        B = sfh.Batch(systems, precision=prec)
        B.set_schedule(w2, tiles, stage)
        B.set_hop_widths(w1, w2)
        for k, (d, m, n) in enumerate(systems):
            B.set_gauge(k, fields[k])
            for j in range(n):
                B.set_rhs(k, j, orc.random_spinor(d, 900 + 10 * k + j))
        times = B.solve_timed(tol=1e-10) if timed else B.solve(tol=1e-10)
        return [B.solution(k, j) for k, (d, m, n) in enumerate(systems) for j in range(n)], times

    for w1, w2, tiles in ((4, 2, 4), (2, 2, 2), (1, 1, 1), (4, 4, 4), (8, 2, 2)):
        ref, _ = run("f16", w1, w2, tiles, 4)
        got, _ = run("f16", w1, w2, tiles, 6)
        assert all(np.array_equal(a, b) for a, b in zip(ref, got)), (w1, w2, tiles)
    ref, _ = run("f16", 4, 2, 4, 4)
    got, times = run("f16", 4, 2, 4, 6, timed=True)
    assert all(np.array_equal(a, b) for a, b in zip(ref, got))
    assert times["cg_hop1"][1] == times["cg_hop2"][1] > 0
    ref32, _ = run("f32", 2, 2, 2, 4)
    got32, _ = run("f32", 2, 2, 2, 6)
    assert all(np.array_equal(a, b) for a, b in zip(ref32, got32))
    d, m, n = systems[3]
    b = orc.random_spinor(d, 900 + 30 + 1)
    r = b - orc.ddag(d, m, fields[3], got[5 + 3 + 2 + 1])
    assert np.linalg.norm(r) / np.linalg.norm(b) < 1.5e-10


@pytest.mark.parametrize("precision", ["f16", "f32", "bf16", "f32_18", "f64"])
def test_batch_resident_grid_schedule_bit_identical(sfh, orc, precision):
    """Schedule 7 (the hop kernels on grids of resident blocks, each taking
    work items in turn from a device counter that the update kernel zeroes)
    gives schedule 4's solutions bit for bit, over several solves of the
    same batch (the counters start from zero each time) and in the timed
    solve; FP64 runs schedule 0 for both."""
    systems = [((4, 4, 4, 8), 0.1, 5), ((6, 6, 6, 6), 0.05, 3), ((8, 8, 8, 8), 0.2, 2)]
    fields = [orc.random_gauge(d, 0.5 + 0.25 * (k % 2), 120 + k) for k, (d, m, n) in enumerate(systems)]

    def run(stage, w1, w2, tiles, timed=False):
        B = sfh.Batch(systems, precision=precision)
        B.set_schedule(w2, tiles, stage)
        B.set_hop_widths(w1, w2)
        for k, (d, m, n) in enumerate(systems):
            B.set_gauge(k, fields[k])
            for j in range(n):
                B.set_rhs(k, j, orc.random_spinor(d, 1300 + 10 * k + j))
        out = []
        for _ in range(2):
            if timed:
                B.solve_timed(tol=1e-10)
            else:
                B.solve(tol=1e-10)
            out.append([B.solution(k, j) for k, (d, m, n) in enumerate(systems) for j in range(n)])
        return out

    for w1, w2, tiles in ((4, 2, 4), (2, 2, 1), (1, 1, 2)):
        ref = run(4, w1, w2, tiles)
        got = run(7, w1, w2, tiles)
        for a, b in zip(ref, got):
            assert all(np.array_equal(x, y) for x, y in zip(a, b)), (w1, w2, tiles)
    got = run(7, 4, 2, 4, timed=True)
    assert all(np.array_equal(x, y) for x, y in zip(run(4, 4, 2, 4)[0], got[1]))
    d, m, n = systems[2]
    b = orc.random_spinor(d, 1300 + 20 + 1)
    r = b - orc.ddag(d, m, fields[2], got[1][5 + 3 + 1])
    assert np.linalg.norm(r) / np.linalg.norm(b) < 1.5e-10


def test_batch_autotune_keeps_results(sfh, orc):
    """The autotuner only changes the schedule: solutions are bit-identical."""
    systems = [((4, 4, 4, 8), 0.1, 3), ((6, 6, 6, 6), 0.2, 2)]
    outs = []
    for tune in (False, True):
        B = sfh.Batch(systems, precision="f32")
        for k, (dims, m, n) in enumerate(systems):
            B.set_gauge(k, orc.random_gauge(dims, 0.5, 400 + k))
            for j in range(n):
                B.set_rhs(k, j, orc.random_spinor(dims, 500 + 10 * k + j))
        if tune:
            assert B.autotune(probe_iters=16) in (1, 2, 4, 8)
            assert B.schedule()[1] in (1, 2, 4)
        B.solve(tol=1e-10)
        outs.append(np.concatenate([B.solution(k, j) for k, (d, m, n) in enumerate(systems) for j in range(n)]))
    assert np.array_equal(outs[0], outs[1])


def test_batch_timed_solve_matches_graph_solve(sfh, orc):
    """The per-kernel timed solve runs the same kernels: identical solutions,
    every iteration's three kernels timed."""
    systems = [((4, 4, 4, 8), 0.1, 3), ((6, 6, 6, 6), 0.2, 2)]
    outs, times = [], None
    for timed in (False, True):
        B = sfh.Batch(systems, precision="f32")
        for k, (dims, m, n) in enumerate(systems):
            B.set_gauge(k, orc.random_gauge(dims, 0.5, 600 + k))
            for j in range(n):
                B.set_rhs(k, j, orc.random_spinor(dims, 700 + 10 * k + j))
        if timed:
            times = B.solve_timed(tol=1e-10)
        else:
            B.solve(tol=1e-10)
        outs.append(np.concatenate([B.solution(k, j) for k, (d, m, n) in enumerate(systems) for j in range(n)]))
    assert np.array_equal(outs[0], outs[1])
    n = [times[k][1] for k in ("cg_hop1", "cg_hop2", "cg_update")]
    assert n[0] == n[1] == n[2] > 0
    assert all(times[k][0] > 0 for k in times)


@pytest.mark.parametrize("precision,bound", [("f16", 1.25), ("f32", 1.25), ("bf16", 1.35)])
def test_mixed_cg_rough_light_mass_keeps_krylov_progress(sfh, orc, precision, bound):
    """eps = 1 links at m = 0.02 on 16^4: the mixed-precision CG needs at most
    `bound` times FP64's iterations (the reliable update rebuilds the search
    direction on the true residual; without it FP16 took 4.9 times FP64's
    count here), and reaches the FP64 true residual, recomputed by the
    oracle's D D^dag (apply_DDdagger, Fermions.cpp:530-547) on the host; the
    FP64 solve is the oracle's CG (Fermions.cpp:553-617) to 1e-10."""
    tol = 1e-10
    dims, mass = (16, 16, 16, 16), 0.02
    lat = sfh.Lattice(dims, mass, 4.2)
    try:
        lat.random_gauge(1.0, 21)
        U = lat.download_gauge()
        phi = lat.gaussian_spinor(22)
        X64, i64 = lat.solve_CG_DDdagger(phi, tol=tol, max_iter=40000, precision="f64", info=True)
        X, inf = lat.solve_CG_DDdagger(phi, tol=tol, max_iter=40000, precision=precision, info=True)
        assert inf["status"] == 0
        assert inf["iters"] <= bound * i64["iters"], (inf, i64)
        assert true_resid(orc, dims, mass, U, phi, X) < 1.05 * tol
        Xo, it_o, _, st = orc.cg(dims, mass, U, phi, tol, 40000)
        assert st == 0 and abs(i64["iters"] - it_o) <= 1
        assert np.linalg.norm(X64 - Xo) / np.linalg.norm(Xo) < 1e-10
        # |x - x*| / |x*| <= cond(M) resid, cond(M) <= (m^2 + 16) / m^2 = 40001
        assert np.linalg.norm(X - Xo) / np.linalg.norm(Xo) < 40001 * 2 * tol
    finally:
        lat.close()


SYS_SYSTEMS = [((8, 8, 8, 8), 0.1, 5), ((6, 6, 6, 8), 0.05, 3), ((4, 4, 4, 4), 0.2, 9)]


def _sys_batch(sfh, orc, precision, schedule):
    B = sfh.Batch(SYS_SYSTEMS, precision=precision)
    B.set_schedule(*schedule)
    data = []
    for k, (dims, mass, nrhs) in enumerate(SYS_SYSTEMS):
        U = orc.random_gauge(dims, 1.0 if k % 2 == 0 else 0.3, 800 + k)
        B.set_gauge(k, U)
        bs = [orc.random_spinor(dims, 900 + 10 * k + j) for j in range(nrhs)]
        for j, b in enumerate(bs):
            B.set_rhs(k, j, b)
        data.append((U, bs))
    return B, data


@pytest.mark.parametrize("precision", ["f16", "bf16", "f32"])
def test_batch_system_blocked_schedule(sfh, orc, precision):
    """The system-blocked schedule (one block per tile serving every RHS of
    its system, links staged once per tile, reliable updates in kernels of
    their own) on systems with several tiles, a partial last tile and more
    RHS than one group: every RHS-group width gives bit-identical solutions
    (the per-group sums have a fixed order), each reaches the FP64 true
    residual by the oracle's D D^dag, the timed solve runs the same kernels
    to the same solutions, and so does the persistent schedule (one
    cooperative launch)."""
    tol = 1e-10
    outs = []
    for w in (1, 2, 4, 8):
        B, data = _sys_batch(sfh, orc, precision, (w, 1, 2))
        assert B.schedule() == (w, 1, 2)
        B.solve(tol=tol, max_iter=20000)
        sol = []
        for k, (dims, mass, nrhs) in enumerate(SYS_SYSTEMS):
            U, bs = data[k]
            for j in range(nrhs):
                X = B.solution(k, j)
                info = B.info(k, j)
                assert info["status"] == 0 and info["reliable_updates"] >= 1
                assert true_resid(orc, dims, mass, U, bs[j], X) < 1.05 * tol, (w, k, j)
                sol.append(X)
        outs.append(np.concatenate(sol))
        B.close()
    for o in outs[1:]:
        assert np.array_equal(o, outs[0])
    B, _ = _sys_batch(sfh, orc, precision, (4, 1, 2))
    times = B.solve_timed(tol=tol)
    timed = np.concatenate([B.solution(k, j) for k, (d, m, n) in enumerate(SYS_SYSTEMS) for j in range(n)])
    B.close()
    assert np.array_equal(timed, outs[0])
    assert set(times) == {"cg_hop1", "cg_hop2", "cg_update", "cg_ru1", "cg_ru2"}
    assert len({times[k][1] for k in times}) == 1  # every iteration launches all five
    # the persistent schedule: the same per-tile work in one cooperative
    # launch gives the same solutions bit for bit, in one launch per solve
    for w, timed_solve in ((2, False), (8, True)):
        B, _ = _sys_batch(sfh, orc, precision, (w, 1, 3))
        if timed_solve:
            times = B.solve_timed(tol=tol)
            assert set(times) == {"cg_persistent"} and times["cg_persistent"][1] == 1
        else:
            B.solve(tol=tol, max_iter=20000)
            assert B.kernel_launches() == 2  # cg_init and the persistent kernel
        pers = np.concatenate([B.solution(k, j) for k, (d, m, n) in enumerate(SYS_SYSTEMS) for j in range(n)])
        B.close()
        assert np.array_equal(pers, outs[0])


@pytest.mark.parametrize("precision", ["f16", "f32"])
def test_lattice_solve_persistent_schedule(sfh, orc, precision):
    """A single solve with the context's schedule set to the persistent launch
    (3) equals the system-blocked graph schedule (2) bit for bit and reaches
    the FP64 true residual by the oracle's D D^dag."""
    dims, mass, tol = (8, 8, 8, 12), 0.05, 1e-10
    U = orc.random_gauge(dims, 1.0, 171)
    b = orc.random_spinor(dims, 172)
    lat = sfh.Lattice(dims, mass)
    try:
        lat.upload_gauge(U)
        out = []
        for stage in (2, 3):
            lat.set_schedule(1, 1, stage)
            X, info = lat.solve_CG_DDdagger(b, tol=tol, precision=precision, info=True)
            assert info["status"] == 0
            assert true_resid(orc, dims, mass, U, b, X) < 1.05 * tol
            out.append(X)
        assert np.array_equal(out[0], out[1])
    finally:
        lat.close()


def test_persistent_barrier_wait_runs_out_and_the_batch_stays_usable(sfh, orc):
    """The persistent schedule's grid barrier waits a bounded number of polls.
    With the bound cut to one poll the first wait of a multi-block launch runs
    out: every block leaves at its next wait, the solve returns
    SFH_ERR_TIMEOUT, and the next solve with the default bound on the same
    batch (same context) is correct."""
    tol = 1e-10
    B, data = _sys_batch(sfh, orc, "f16", (2, 1, 3))
    try:
        B.set_barrier_polls(1)
        with pytest.raises(sfh.SfhError) as e:
            B.solve(tol=tol, max_iter=20000)
        assert e.value.status == sfh.SFH_ERR_TIMEOUT
        B.set_barrier_polls(0)
        B.solve(tol=tol, max_iter=20000)
        for k, (dims, mass, nrhs) in enumerate(SYS_SYSTEMS):
            U, bs = data[k]
            for j in range(nrhs):
                assert true_resid(orc, dims, mass, U, bs[j], B.solution(k, j)) < 1.05 * tol
    finally:
        B.close()


@pytest.mark.parametrize("precision", ["f64", "f16"])
def test_batch_rhs_at_their_own_masses(sfh, orc, precision):
    """The RHS of one system solved at three masses on the same links: each
    solution reaches the true residual of D(m) D(m)^dag at its own mass (by
    the oracle), and the batch's own residual check uses that mass."""
    dims, tol = (8, 8, 8, 8), 1e-10
    masses = [0.05, 0.2, 0.8]
    U = orc.random_gauge(dims, 1.0, 301)
    B = sfh.Batch([(dims, 0.5, 3)], precision=precision)
    try:
        B.set_gauge(0, U)
        bs = [orc.random_spinor(dims, 302 + j) for j in range(3)]
        for j, (b, m) in enumerate(zip(bs, masses)):
            B.set_rhs(0, j, b)
            B.set_rhs_mass(0, j, m)
        B.solve(tol=tol, max_iter=20000)
        iters = []
        for j, (b, m) in enumerate(zip(bs, masses)):
            X = B.solution(0, j)
            r = true_resid(orc, dims, m, U, b, X)
            assert r < (2.0 if precision == "f64" else 1.05) * tol, (j, r)
            assert abs(B.true_residual(0, j) - r) < 1e-3 * tol + 1e-3 * r
            iters.append(B.info(0, j)["iters"])
        assert iters[0] > iters[1] > iters[2]  # lighter masses need more iterations
    finally:
        B.close()
