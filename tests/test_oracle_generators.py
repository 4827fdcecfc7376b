"""The oracle's restatement of the library's seeded generators (CPU only).

The library draws gauge fields, sources and momenta from Philox-4x32-10
(Salmon, Moraes, Dror & Shaw, SC'11) with Box-Muller normals; the reference's
own generator (rng.cpp:7-15) is unseeded, so the fields it would draw cannot
be reproduced, but their distributions can: random_traceless_hermitian_SU3
(Lattice.cpp:1001-1033), generateGaussianComplex (Fermions.cpp:207-212) and
generate_conjugate_field_configuration (Fermions.cpp:342-360).

Pins: Philox against the published known-answer vectors of the algorithm's
authors (the Random123 distribution); the fields against the group and
distribution properties the reference's generators have.  The device
generators are compared with these functions in test_gpu_generators.py.
"""
import numpy as np
import pytest


# Philox-4x32-10 known-answer vectors (counter, key) -> output, as published
# with the algorithm (Random123 kat_vectors)
PHILOX_KAT = [
    ((0x00000000, 0x00000000, 0x00000000, 0x00000000), (0x00000000, 0x00000000),
     (0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8)),
    ((0xffffffff, 0xffffffff, 0xffffffff, 0xffffffff), (0xffffffff, 0xffffffff),
     (0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd)),
    ((0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344), (0xa4093822, 0x299f31d0),
     (0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1)),
]


@pytest.mark.parametrize("ctr,key,out", PHILOX_KAT)
def test_philox_known_answers(orc, ctr, key, out):
    assert orc.philox4x32_10(ctr, key) == list(out)


def mats(field):
    return field.reshape(-1, 3, 3, 2)[..., 0] + 1j * field.reshape(-1, 3, 3, 2)[..., 1]


def test_gauge_generator_is_special_unitary_and_seeded(orc):
    dims = (4, 4, 4, 8)
    U = orc.philox_gauge(dims, 1.0, 5)
    M = mats(U)
    eye = np.eye(3)
    assert np.abs(M @ M.conj().transpose(0, 2, 1) - eye).max() < 1e-13
    assert np.abs(np.linalg.det(M) - 1.0).max() < 1e-13
    assert np.array_equal(U, orc.philox_gauge(dims, 1.0, 5))
    assert not np.array_equal(U, orc.philox_gauge(dims, 1.0, 6))


def test_gauge_generator_is_exp_of_the_hermitian_draw(orc):
    """U = exp(i eps H) with H built from the link's nine normals exactly as
    random_traceless_hermitian_SU3 builds it (N(0,1) diagonal, trace removed;
    N(0,1) real and imaginary off-diagonal parts)."""
    dims, eps, seed = (2, 2, 2, 2), 0.3, 9
    U = orc.philox_gauge(dims, eps, seed)
    n = 4 * orc.volume(dims)
    H = np.zeros((n, 3, 3), np.complex128)
    for l in range(n):
        z = orc.philox_normals(seed, 1, l, 9)
        d = z[:3] - z[:3].mean()
        H[l] = np.diag(d)
        for (i, j), (a, b) in zip(((0, 1), (0, 2), (1, 2)), ((3, 4), (5, 6), (7, 8))):
            H[l, i, j] = z[a] + 1j * z[b]
            H[l, j, i] = z[a] - 1j * z[b]
    Hf = np.ascontiguousarray(H.view(np.float64).reshape(18 * n))
    assert np.abs(orc.exp_field(eps, Hf) - U).max() < 1e-15


def test_spinor_generator_moments(orc):
    dims = (8, 8, 8, 8)
    z = orc.philox_spinor(dims, 3, sigma=0.5)
    n = z.size
    assert abs(z.mean()) < 5 * 0.5 / np.sqrt(n)
    assert abs(z.var() / 0.25 - 1.0) < 5 * np.sqrt(2.0 / n)
    # the fourth moment of a normal: 3 sigma^4
    assert abs(np.mean(z ** 4) / (3 * 0.25 ** 2) - 1.0) < 0.05
    assert np.array_equal(z, 0.5 * orc.philox_spinor(dims, 3))


def test_momenta_generator_is_the_gell_mann_sum(orc):
    """P = 1/2 sum_a p_a lambda_a (Fermions.cpp:342-360): Hermitian, traceless,
    Tr P^2 = 1/2 sum_a p_a^2, so <Tr P^2> = 4 per link."""
    dims = (4, 4, 4, 4)
    P = orc.philox_momenta(dims, 7)
    M = mats(P)
    assert np.abs(M - M.conj().transpose(0, 2, 1)).max() == 0.0
    assert np.abs(np.trace(M, axis1=1, axis2=2)).max() < 1e-15
    n = M.shape[0]
    gm = orc.gell_mann()
    for l in (0, 1, n - 1):
        p = orc.philox_normals(7, 3, l, 8)
        assert np.abs(0.5 * np.einsum("a,aij->ij", p, gm) - M[l]).max() < 1e-15
    trp2 = np.einsum("nij,nji->n", M, M).real
    assert abs(trp2.mean() / 4.0 - 1.0) < 5 * np.sqrt(2.0 / 8 / n) * 2
