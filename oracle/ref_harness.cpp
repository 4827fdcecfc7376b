// ref_harness.cpp — drives the reference's own, unmodified functions
// (alexanderchasteen/Staggered_Fermions_HMC: Fermions.cpp, Lattice.cpp) on
// injected inputs and writes their outputs as raw little-endian doubles.
//
// TEST INFRASTRUCTURE ONLY.  Built by oracle/build_ref.py into oracle/_ref/
// against a generated Parameters.h (lattice size, mass, CG tolerance are
// compile-time constants in the reference) and the project's Eigen-API subset
// header.  Used to produce tests/golden fixtures and as the reference CPU
// timing arm of bench.py.
//
// usage:
//   ref_harness run  <indir> <outdir> <beta> <eps> <nsteps>
//   ref_harness time <indir> <nsolves>        (prints one JSON line)
//   ref_harness heatbath <indir> <outdir> <beta> <nsweeps>
//
// inputs in <indir>: U.bin (72V), phi.bin (6V), P.bin (72V), H.bin (18n)
#include <omp.h>

#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#include "Fermions.h"
#include "Lattice.h"
#include "Parameters.h"

static const int V = Spatial_Size * Spatial_Size * Spatial_Size * temporal_size;

static std::vector<double> read_bin(const std::string& path)
{
    std::ifstream in(path, std::ios::binary | std::ios::ate);
    if (!in) { std::cerr << "cannot read " << path << "\n"; std::exit(2); }
    std::streamsize n = in.tellg();
    in.seekg(0);
    std::vector<double> v(n / sizeof(double));
    in.read(reinterpret_cast<char*>(v.data()), n);
    return v;
}

static void write_bin(const std::string& path, const void* data, size_t bytes)
{
    std::ofstream out(path, std::ios::binary);
    out.write(reinterpret_cast<const char*>(data), bytes);
}

static void write_vec(const std::string& path, const std::vector<double>& v)
{
    write_bin(path, v.data(), v.size() * sizeof(double));
}

static lattice_index coords(int s)
{
    lattice_index c;
    c[3] = s % temporal_size; s /= temporal_size;
    c[2] = s % Spatial_Size; s /= Spatial_Size;
    c[1] = s % Spatial_Size; s /= Spatial_Size;
    c[0] = s;
    return c;
}

static void put_su3(std::vector<double>& out, size_t off, const SU3& m)
{
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            out[off + (i * 3 + j) * 2] = m(i, j).real();
            out[off + (i * 3 + j) * 2 + 1] = m(i, j).imag();
        }
}

static SU3 get_su3(const std::vector<double>& in, size_t off)
{
    SU3 m;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            m(i, j) = complex(in[off + (i * 3 + j) * 2], in[off + (i * 3 + j) * 2 + 1]);
    return m;
}

static int run(const std::string& indir, const std::string& out, double beta,
               double eps, int nsteps)
{
    std::vector<double> U = read_bin(indir + "/U.bin");
    std::vector<double> phi = read_bin(indir + "/phi.bin");
    std::vector<double> P = read_bin(indir + "/P.bin");
    std::vector<double> H = read_bin(indir + "/H.bin");
    if ((int)U.size() != 72 * V || (int)phi.size() != 6 * V || (int)P.size() != 72 * V) {
        std::cerr << "input sizes do not match the compiled lattice\n";
        return 2;
    }

    // neighbour tables and phases through the reference's own walkers
    std::vector<int> tab(5 * 4 * V);
    for (int s = 0; s < V; ++s)
        for (int d = 0; d < 4; ++d) {
            lattice_index a = coords(s), b = coords(s);
            int bu = moveup_fermion(a, d);
            int bd = movedown_fermion(b, d);
            int k = s * 4 + d;
            tab[0 * 4 * V + k] = ((a[0] * Spatial_Size + a[1]) * Spatial_Size + a[2]) * temporal_size + a[3];
            tab[1 * 4 * V + k] = ((b[0] * Spatial_Size + b[1]) * Spatial_Size + b[2]) * temporal_size + b[3];
            tab[2 * 4 * V + k] = bu;
            tab[3 * 4 * V + k] = bd;
            tab[4 * 4 * V + k] = staggered_phase_factor(coords(s), d);
        }
    write_bin(out + "/tables.i32", tab.data(), tab.size() * sizeof(int));

    // D phi and D^dag phi (Fermions.cpp:249, 285)
    std::vector<double> Dphi(6 * V), Ddphi(6 * V), DDd(6 * V);
    for (int s = 0; s < V; ++s) {
        Eigen::Vector3cd a = apply_dirac_operator_at_lattice_site(phi, U, coords(s));
        Eigen::Vector3cd b = apply_dirac_dagger_at_site(phi, U, coords(s));
        for (int c = 0; c < 3; ++c) {
            Dphi[s * 6 + 2 * c] = a[c].real(); Dphi[s * 6 + 2 * c + 1] = a[c].imag();
            Ddphi[s * 6 + 2 * c] = b[c].real(); Ddphi[s * 6 + 2 * c + 1] = b[c].imag();
        }
    }
    write_vec(out + "/Dphi.bin", Dphi);
    write_vec(out + "/Ddagphi.bin", Ddphi);
    apply_DDdagger(phi, U, DDd);
    write_vec(out + "/DDdagphi.bin", DDd);

    // CG and Y (Fermions.cpp:553, 623)
    std::vector<double> X = solve_X_field(phi, U);
    std::vector<double> Y = solve_Y_field(X, U);
    write_vec(out + "/X.bin", X);
    write_vec(out + "/Y.bin", Y);

    // per-link staples and forces
    std::vector<double> A1(72 * V), A2(72 * V), Fg(72 * V), Ff(72 * V);
    for (int s = 0; s < V; ++s) {
        lattice_index c = coords(s);
        for (int d = 0; d < 4; ++d) {
            link_index li = {c[0], c[1], c[2], c[3], d};
            size_t off = (size_t)(s * 4 + d) * 18;
            put_su3(A1, off, compute_staple_sum_at_link(U, li));
            put_su3(A2, off, compute_rectangle_staple_sum_at_link(U, li));
            put_su3(Fg, off, compute_gauge_force_at_link(U, li, beta));
            put_su3(Ff, off, compute_fermion_force_at_link(X, Y, U, li));
        }
    }
    write_vec(out + "/A1.bin", A1);
    write_vec(out + "/A2.bin", A2);
    write_vec(out + "/Fgauge.bin", Fg);
    write_vec(out + "/Ffermion.bin", Ff);
    write_vec(out + "/Ffull.bin", compute_full_force_field(X, Y, U, beta));

    // scalars: action, plaquette, Tr P^2, phi.X
    double scal[4] = {compute_action(U, beta), compute_avg_plaq(U),
                      compute_Tr_P2(P), field_inner_product_real(phi, X)};
    write_bin(out + "/scalars.bin", scal, sizeof(scal));

    // exp(iQ) on supplied Hermitian matrices (Fermions.cpp:843)
    std::vector<double> E(H.size());
    for (size_t k = 0; k + 18 <= H.size(); k += 18)
        put_su3(E, k, numerically_stable_matrix_exponential(get_su3(H, k)));
    write_vec(out + "/expH.bin", E);

    // Polyakov loop grid and correlators (Lattice.cpp:869, 886)
    std::vector<complex> grid = precompute_polyakov_grid(U);
    std::vector<double> pg(2 * grid.size());
    for (size_t i = 0; i < grid.size(); ++i) { pg[2 * i] = grid[i].real(); pg[2 * i + 1] = grid[i].imag(); }
    write_vec(out + "/poly_grid.bin", pg);
    std::vector<double> corr;
    for (int r2 = 1; r2 <= 3; ++r2) {
        complex cr = correlator_over_fixed_distance_fast(grid, r2);
        corr.push_back(cr.real()); corr.push_back(cr.imag());
    }
    write_vec(out + "/poly_corr.bin", corr);

    // one trajectory through local_* (Fermions.cpp:967-1028), with H terms
    std::vector<double> Ut = U, Pt = P;
    double h0[3] = {compute_Tr_P2(Pt), compute_action(Ut, beta),
                    field_inner_product_real(phi, solve_X_field(phi, Ut))};
    local_initial_half_step(Pt, beta, phi, Ut, eps);
    local_leapfrog_steps(Pt, beta, phi, Ut, eps, nsteps);
    std::vector<double> Xf = local_final_step(Pt, beta, phi, Ut, eps);
    double h1[3] = {compute_Tr_P2(Pt), compute_action(Ut, beta), field_inner_product_real(phi, Xf)};
    write_vec(out + "/traj_U.bin", Ut);
    write_vec(out + "/traj_P.bin", Pt);
    write_vec(out + "/traj_X.bin", Xf);
    double hh[6] = {h0[0], h0[1], h0[2], h1[0], h1[1], h1[2]};
    write_bin(out + "/traj_H.bin", hh, sizeof(hh));
    return 0;
}

// Reference CPU timing: apply_DDdagger and solve_CG_DDdagger with the
// reference's own OpenMP loops.
static int time_cg(const std::string& indir, int nsolves)
{
    std::vector<double> U = read_bin(indir + "/U.bin");
    std::vector<double> phi = read_bin(indir + "/phi.bin");
    std::vector<double> out(6 * V);
    apply_DDdagger(phi, U, out);  // warm-up
    int napply = 5;
    double t0 = omp_get_wtime();
    for (int i = 0; i < napply; ++i) apply_DDdagger(phi, U, out);
    double t_apply = (omp_get_wtime() - t0) / napply;
    t0 = omp_get_wtime();
    std::vector<double> X;
    for (int i = 0; i < nsolves; ++i) X = solve_CG_DDdagger(phi, U);
    double t_solve = (omp_get_wtime() - t0) / nsolves;
    std::printf("{\"V\": %d, \"mass\": %.17g, \"tol\": %.3g, \"threads\": %d, "
                "\"ddag_s\": %.6e, \"solve_s\": %.6e, \"nsolves\": %d}\n",
                V, fermion_mass, tol, omp_get_max_threads(), t_apply, t_solve, nsolves);
    return 0;
}

// heatbath_update (Lattice.cpp:722-757) nsweeps times from U.bin; writes
// plaq.bin: compute_avg_plaq after every sweep (the reference's generator is
// unseeded, so this is one realisation of its Markov chain)
static int heatbath_run(const std::string& in, const std::string& out, double beta, int nsweeps)
{
    Link_array U = read_bin(in + "/U.bin");
    std::vector<double> plaq;
    for (int k = 0; k < nsweeps; ++k) {
        heatbath_update(U, beta);
        plaq.push_back(compute_avg_plaq(U));
    }
    write_vec(out + "/plaq.bin", plaq);
    return 0;
}

int main(int argc, char** argv)
{
    if (argc >= 6 && std::string(argv[1]) == "heatbath")
        return heatbath_run(argv[2], argv[3], std::atof(argv[4]), std::atoi(argv[5]));
    if (argc >= 7 && std::string(argv[1]) == "run")
        return run(argv[2], argv[3], std::atof(argv[4]), std::atof(argv[5]), std::atoi(argv[6]));
    if (argc >= 4 && std::string(argv[1]) == "time")
        return time_cg(argv[2], std::atoi(argv[3]));
    std::cerr << "usage: ref_harness run <indir> <outdir> <beta> <eps> <nsteps>\n"
                 "       ref_harness time <indir> <nsolves>\n"
                 "       ref_harness heatbath <indir> <outdir> <beta> <nsweeps>\n";
    return 1;
}
