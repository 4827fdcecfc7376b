"""GPU: the device generators against the oracle's CPU restatement.

Every benchmark input comes from these kernels (sfh_random_gauge,
sfh_gaussian_spinor, sfh_random_momenta and the batch's sfh_batch_random_gauge
/ sfh_batch_random_rhs), so they are pinned here: the same Philox-4x32-10
counters and keys as the oracle (whose Philox is checked against the
algorithm's published known-answer vectors in test_oracle_generators.py),
the same Box-Muller normals and the same exp(i eps H).

Tolerances: the Philox words are integers and must agree exactly, which the
normals show (a wrong key, counter or word order moves a normal by O(1));
what remains is the last bit of CUDA's and the C library's log, sin and cos
(Box-Muller) and the rounding order of exp(iQ): normals and momenta agree to
1e-14 relative, links to 1e-13.  Device links are SU(3) to 1e-13.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def sfh():
    import staggered_fermions_hmc_b200 as m
    m.load_library()
    return m


def rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def mats(field):
    f = field.reshape(-1, 3, 3, 2)
    return f[..., 0] + 1j * f[..., 1]


@pytest.mark.parametrize("dims,eps,seed", [((4, 4, 4, 8), 0.3, 1), ((8, 8, 8, 8), 1.0, 1003),
                                           ((6, 4, 8, 6), 1.0, 2 ** 40 + 17)])
def test_random_gauge_matches_oracle(sfh, orc, dims, eps, seed):
    lat = sfh.Lattice(dims, 0.1)
    lat.random_gauge(eps, seed)
    U = lat.download_gauge()
    lat.close()
    assert np.abs(U - orc.philox_gauge(dims, eps, seed)).max() < 1e-13
    M = mats(U)
    assert np.abs(M @ M.conj().transpose(0, 2, 1) - np.eye(3)).max() < 1e-13
    assert np.abs(np.linalg.det(M) - 1.0).max() < 1e-13


@pytest.mark.parametrize("sigma", [1.0, 1.0 / np.sqrt(2.0)])
def test_gaussian_spinor_matches_oracle(sfh, orc, sigma):
    dims = (8, 8, 8, 12)
    lat = sfh.Lattice(dims, 0.1)
    z = lat.gaussian_spinor(22, sigma)
    lat.close()
    assert rel(z, orc.philox_spinor(dims, 22, sigma)) < 1e-14


def test_random_momenta_matches_oracle(sfh, orc):
    dims = (4, 6, 4, 8)
    lat = sfh.Lattice(dims, 0.1)
    lat.generate_conjugate_field_configuration(5)
    P = lat.download_momenta()
    lat.close()
    assert rel(P, orc.philox_momenta(dims, 5)) < 1e-14


def test_batch_generators_match_oracle(sfh, orc):
    """The benchmark batch's own generators, on two systems of different size."""
    systems = [((8, 8, 8, 8), 0.05, 2), ((12, 12, 12, 12), 0.2, 1)]
    B = sfh.Batch(systems, precision="f16")
    try:
        for k, (dims, _, nrhs) in enumerate(systems):
            B.random_gauge(k, 1.0, 1000 + k)
            assert np.abs(B.gauge(k) - orc.philox_gauge(dims, 1.0, 1000 + k)).max() < 1e-13
            for j in range(nrhs):
                B.random_rhs(k, j, 100000 + 100 * k + j)
                assert rel(B.rhs(k, j), orc.philox_spinor(dims, 100000 + 100 * k + j)) < 1e-14
    finally:
        B.close()
