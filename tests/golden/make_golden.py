#!/usr/bin/env python3
"""Generate the golden fixtures in tests/golden/ from the reference itself.

Runs the reference's own, unmodified functions (built by oracle/build_ref.py
from the reference sources) on seeded inputs and stores inputs and outputs as
compressed .npz files.  Needs the reference sources, so it runs only where
they are present; the committed fixtures are what the tests read.

usage: python tests/golden/make_golden.py --reference DIR [--hex-only]
       (DIR: a checkout of the reference; or set SFH_REFERENCE_DIR)
"""
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from oracle import build_ref  # noqa: E402

# (L, T, mass, tol, gauge eps, seed, beta, md eps, md steps)
FIXTURES = [
    (4, 4, 0.1, 1e-12, 0.3, 1, 4.2, 0.1, 10),
    (4, 6, 0.5, 1e-12, 1.0, 2, 4.2, 0.05, 4),
]


def exp_test_matrices(rng):
    """Hermitian traceless inputs for exp(iQ): generic, tiny (small-c1 branch),
    negative-determinant-sign and diagonal cases."""
    H = oracle.random_hermitian(rng, 16)
    scales = np.array([1.0, 0.3, 2.0, 1e-7, 0.05, 1.5, 3.0, 1e-4,
                       0.7, 0.01, 5.0, 0.2, 1.0, 1.0, 0.9, 0.4])
    H = H * scales[:, None]
    H[12] = -H[0]                    # flips the sign of c0
    d = np.zeros(18)
    d[0], d[8], d[16] = 0.5, -0.2, -0.3  # diagonal
    H[13] = d
    return np.ascontiguousarray(H)


def make(L, T, mass, tol, geps, seed, beta, eps, nsteps):
    dims = (L, L, L, T)
    exe = build_ref.build(L, T, mass, tol)
    rng = np.random.default_rng(1000 + seed)
    U = oracle.random_gauge(dims, geps, seed)
    phi = rng.standard_normal(6 * oracle.volume(dims))
    P = oracle.random_momenta(dims, 2000 + seed)
    H = exp_test_matrices(rng)
    with tempfile.TemporaryDirectory() as td:
        ind, outd = os.path.join(td, "in"), os.path.join(td, "out")
        os.makedirs(ind)
        os.makedirs(outd)
        for name, arr in (("U", U), ("phi", phi), ("P", P), ("H", H)):
            arr.astype("<f8").tofile(os.path.join(ind, name + ".bin"))
        subprocess.run([exe, "run", ind, outd, repr(beta), repr(eps), str(nsteps)],
                       check=True)
        res = {}
        for f in sorted(os.listdir(outd)):
            key = f.rsplit(".", 1)[0]
            dt = "<i4" if f.endswith(".i32") else "<f8"
            res[key] = np.fromfile(os.path.join(outd, f), dtype=dt)
    meta = np.array([L, T, mass, tol, geps, seed, beta, eps, nsteps], dtype=np.float64)
    path = os.path.join(HERE, f"ref_L{L}T{T}.npz")
    np.savez_compressed(path, meta=meta, U=U, phi=phi, P=P, H=H, **res)
    print("wrote", path, os.path.getsize(path), "bytes")


# heatbath: (beta values, runs per beta, sweeps) on 4^4 from a cold start
HEATBATH = ((2.0, 4.2), 4, 100)


def make_heatbath():
    """Plaquette histories of the reference's heatbath_update (Lattice.cpp:
    722-757).  Its generator is unseeded, so these are independent
    realisations of its Markov chain; the tests compare equilibrium means."""
    betas, runs, sweeps = HEATBATH
    exe = build_ref.build(4, 4, 0.1, 1e-12)
    hist = np.zeros((len(betas), runs, sweeps))
    with tempfile.TemporaryDirectory() as td:
        ind = os.path.join(td, "in")
        os.makedirs(ind)
        oracle.cold_gauge((4, 4, 4, 4)).astype("<f8").tofile(os.path.join(ind, "U.bin"))
        for b, beta in enumerate(betas):
            for r in range(runs):
                outd = os.path.join(td, f"out{b}_{r}")
                os.makedirs(outd)
                subprocess.run([exe, "heatbath", ind, outd, repr(beta), str(sweeps)], check=True)
                hist[b, r] = np.fromfile(os.path.join(outd, "plaq.bin"))
    path = os.path.join(HERE, "heatbath_ref_L4T4.npz")  # outside the ref_*.npz operator fixtures
    np.savez_compressed(path, betas=np.array(betas), plaq=hist)
    print("wrote", path, os.path.getsize(path), "bytes")


# HEX staple steps: the reference's apply_step_1 / 3 / 5 (Smearing.cpp:76-275)
# on 4^4 with seeded SU(3) inputs (gauge links; decorated V1 [64][V] and
# V2 [16][V] fields drawn as plain SU(3) matrices by the oracle's Philox
# generator: the steps are defined for any inputs).  Stored: the seeds, the
# outputs at a fixed subset of sites and, over every matrix, a checksum with
# seeded N(0,1) weights, sum_k w_k G_k.
HEX = {"dims": (4, 4, 4, 4), "eps": 0.5, "seeds": (31, 32, 33), "weight_seed": 34,
       "sites": {1: 8, 2: 16, 3: 64}}


def hex_inputs(dims, eps, seeds):
    L, T = dims[0], dims[3]
    U = oracle.philox_gauge(dims, eps, seeds[0])
    V1 = oracle.philox_gauge((L, L, L, 16 * T), eps, seeds[1])  # 64 V matrices
    V2 = oracle.philox_gauge((L, L, L, 4 * T), eps, seeds[2])   # 16 V matrices
    return U, V1, V2


def hex_checksum(G, weight_seed, level):
    w = np.random.default_rng(weight_seed + level).standard_normal(G.size // 18)
    return np.einsum("k,kx->x", w, G.reshape(-1, 18))


def hex_site_subset(V, n):
    return np.linspace(0, V - 1, n).astype(np.int64)


def make_hex():
    dims, eps, seeds = HEX["dims"], HEX["eps"], HEX["seeds"]
    exe = build_ref.build_hex()
    U, V1, V2 = hex_inputs(dims, eps, seeds)
    V = oracle.volume(dims)
    res = {}
    with tempfile.TemporaryDirectory() as td:
        ind, outd = os.path.join(td, "in"), os.path.join(td, "out")
        os.makedirs(ind)
        os.makedirs(outd)
        for name, arr in (("U", U), ("V1", V1), ("V2", V2)):
            arr.astype("<f8").tofile(os.path.join(ind, name + ".bin"))
        subprocess.run([exe, ind, outd], check=True)
        for level in (1, 2, 3):
            G = np.fromfile(os.path.join(outd, f"G{level}.bin"), dtype="<f8")
            n = G.size // (18 * V)
            sites = hex_site_subset(V, HEX["sites"][level])
            res[f"G{level}_sites"] = sites
            res[f"G{level}_at_sites"] = G.reshape(n, V, 18)[:, sites, :]
            res[f"G{level}_checksum"] = hex_checksum(G, HEX["weight_seed"], level)
    meta = np.array(list(dims) + [eps] + list(seeds) + [HEX["weight_seed"]], dtype=np.float64)
    path = os.path.join(HERE, "hex_ref_L4T4.npz")
    np.savez_compressed(path, meta=meta, **res)
    print("wrote", path, os.path.getsize(path), "bytes")


def main(argv):
    if "--reference" in argv:
        build_ref.set_reference(argv[argv.index("--reference") + 1])
    if not build_ref.REF or not os.path.isdir(build_ref.REF):
        sys.exit("give --reference DIR (a checkout of the reference) or set SFH_REFERENCE_DIR")
    if "--hex-only" in argv:
        make_hex()
        return
    for fx in FIXTURES:
        make(*fx)
    make_heatbath()
    make_hex()


if __name__ == "__main__":
    main(sys.argv[1:])
