// hex_harness.cpp — runs the reference's own HEX staple steps on given fields.
//
// TEST INFRASTRUCTURE ONLY.  Built by oracle/build_ref.py into oracle/_ref/
// together with the reference's unmodified Smearing.cpp (compiled with its
// include order fixed on the command line: Smearing.h uses Spatial_Size and
// SU3 before including anything, Smearing.h:11).  Only the exp-free steps
// run, because the exp steps (apply_step_2/4/6) pass an anti-Hermitian matrix
// to numerically_stable_matrix_exponential, which rejects it
// (Fermions.cpp:848-857):
//
//   G1 = apply_step_1(U)     Smearing.cpp:76-123   [64][V] decorated staples
//   G2 = apply_step_3(V1)    Smearing.cpp:157-211  [16][V]
//   G3 = apply_step_5(V2)    Smearing.cpp:236-275  [4][V]
//
// Matrices are written as 18 doubles (row-major, re/im), in the reference's
// flat tensor order (Smearing.cpp:14-73): combo * V + site.
//
// usage: hex_harness <indir: U.bin V1.bin V2.bin> <outdir>
#include <complex>
#include <cstdio>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#include "Lattice.h"

std::vector<SU3> apply_step_1(const Link_array& U);
std::vector<SU3> apply_step_3(std::vector<SU3> V1_mu_nu_rho);
std::vector<SU3> apply_step_5(std::vector<SU3> V2_mu_nu);

static std::vector<double> read_bin(const std::string& path)
{
    std::ifstream f(path, std::ios::binary | std::ios::ate);
    if (!f) throw std::runtime_error("cannot read " + path);
    std::streamsize n = f.tellg();
    f.seekg(0);
    std::vector<double> v(n / sizeof(double));
    f.read(reinterpret_cast<char*>(v.data()), n);
    return v;
}

static std::vector<SU3> to_mats(const std::vector<double>& a)
{
    std::vector<SU3> m(a.size() / 18);
    for (size_t k = 0; k < m.size(); ++k)
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                m[k](i, j) = std::complex<double>(a[k * 18 + (i * 3 + j) * 2], a[k * 18 + (i * 3 + j) * 2 + 1]);
    return m;
}

static void write_mats(const std::string& path, const std::vector<SU3>& m)
{
    std::vector<double> a(m.size() * 18);
    for (size_t k = 0; k < m.size(); ++k)
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                a[k * 18 + (i * 3 + j) * 2] = m[k](i, j).real();
                a[k * 18 + (i * 3 + j) * 2 + 1] = m[k](i, j).imag();
            }
    std::ofstream f(path, std::ios::binary);
    f.write(reinterpret_cast<const char*>(a.data()), a.size() * sizeof(double));
}

int main(int argc, char** argv)
{
    if (argc < 3) {
        std::cerr << "usage: hex_harness <indir> <outdir>\n";
        return 1;
    }
    const std::string in = argv[1], out = argv[2];
    Link_array U = read_bin(in + "/U.bin");
    write_mats(out + "/G1.bin", apply_step_1(U));
    write_mats(out + "/G2.bin", apply_step_3(to_mats(read_bin(in + "/V1.bin"))));
    write_mats(out + "/G3.bin", apply_step_5(to_mats(read_bin(in + "/V2.bin"))));
    return 0;
}
