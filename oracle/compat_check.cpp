// compat_check.cpp — runs the reference's own functions and the same-named
// functions of include/sfh_compat.hpp (the GPU library) on identical inputs
// in one process and prints their relative differences as one JSON line.
//
// TEST INFRASTRUCTURE ONLY.  Built by oracle/build_ref.py into oracle/_ref/
// from the reference's unmodified Fermions.cpp, Lattice.cpp,
// SU3_Sampling.cpp and rng.cpp (against a generated Parameters.h and the
// project's Eigen-API subset header), linked with libsfh.so.  The settings
// of the GPU side come from the same Parameters.h through
// SFH_COMPAT_PARAMETERS(), as a reference driver would take them.
//
// usage: compat_check <indir>     inputs: U.bin (72V), P.bin (72V), phi.bin (6V)
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "Fermions.h"
#include "Lattice.h"
#include "Parameters.h"
#include "sfh_compat.hpp"

namespace {

const int V = Spatial_Size * Spatial_Size * Spatial_Size * temporal_size;

std::vector<double> read_bin(const std::string& path)
{
    std::ifstream in(path, std::ios::binary | std::ios::ate);
    if (!in) {
        std::cerr << "cannot read " << path << "\n";
        std::exit(2);
    }
    std::streamsize n = in.tellg();
    in.seekg(0);
    std::vector<double> v(n / sizeof(double));
    in.read(reinterpret_cast<char*>(v.data()), n);
    return v;
}

double rel(const std::vector<double>& a, const std::vector<double>& b)
{
    if (a.size() != b.size()) return 1e300;
    double d = 0.0, m = 0.0;
    for (size_t i = 0; i < a.size(); ++i) {
        d = std::max(d, std::abs(a[i] - b[i]));
        m = std::max(m, std::abs(b[i]));
    }
    return d / std::max(m, 1e-300);
}

double rel(double a, double b) { return std::abs(a - b) / std::max(std::abs(b), 1e-300); }

double rel(const std::vector<std::complex<double>>& a, const std::vector<std::complex<double>>& b)
{
    std::vector<double> x, y;
    for (auto& c : a) { x.push_back(c.real()); x.push_back(c.imag()); }
    for (auto& c : b) { y.push_back(c.real()); y.push_back(c.imag()); }
    return rel(x, y);
}

std::ostringstream js;
bool first = true;

void put(const std::string& k, double v)
{
    js << (first ? "" : ", ") << "\"" << k << "\": " << v;
    first = false;
}

void put_s(const std::string& k, const std::string& v)
{
    std::string e;
    for (char ch : v) e += (ch == '"' || ch == '\\') ? ' ' : ch;
    js << (first ? "" : ", ") << "\"" << k << "\": \"" << e << "\"";
    first = false;
}

// runs f, returns "<exception type>: <message>" or "none"
template <typename F>
std::string thrown(F f)
{
    try {
        f();
    } catch (const std::invalid_argument& e) {
        return std::string("invalid_argument: ") + e.what();
    } catch (const std::runtime_error& e) {
        return std::string("runtime_error: ") + e.what();
    }
    return "none";
}

}  // namespace

int main(int argc, char** argv)
{
    if (argc < 2) {
        std::cerr << "usage: compat_check <indir>\n";
        return 2;
    }
    std::string dir = argv[1];
    const Link_array U = read_bin(dir + "/U.bin");
    const std::vector<double> P = read_bin(dir + "/P.bin");
    const std::vector<double> phi = read_bin(dir + "/phi.bin");
    if ((int)U.size() != 72 * V || (int)P.size() != 72 * V || (int)phi.size() != 6 * V) {
        std::cerr << "input sizes do not match the lattice\n";
        return 2;
    }
    const double beta = 4.2;
    sfh_compat::configure(SFH_COMPAT_PARAMETERS());

    std::vector<double> a(6 * V), b(6 * V);  // the reference writes into a sized field
    apply_DDdagger(phi, U, a);
    sfh_compat::apply_DDdagger(phi, U, b);
    put("apply_DDdagger", rel(b, a));

    std::vector<double> Xr = solve_CG_DDdagger(phi, U), Xg = sfh_compat::solve_CG_DDdagger(phi, U);
    put("solve_CG_DDdagger", rel(Xg, Xr));
    std::vector<double> Yr = solve_Y_field(Xr, U), Yg = sfh_compat::solve_Y_field(Xr, U);
    put("solve_Y_field", rel(Yg, Yr));

    put("compute_full_force_field",
        rel(sfh_compat::compute_full_force_field(Xr, Yr, U, beta), compute_full_force_field(Xr, Yr, U, beta)));
    put("compute_fermion_only_force_field",
        rel(sfh_compat::compute_fermion_only_force_field(Xr, Yr, U), compute_fermion_only_force_field(Xr, Yr, U)));
    put("compute_gauge_only_force_field",
        rel(sfh_compat::compute_gauge_only_force_field(U, beta), compute_gauge_only_force_field(U, beta)));
    put("compute_Tr_P2", rel(sfh_compat::compute_Tr_P2(P), compute_Tr_P2(P)));
    put("compute_action", rel(sfh_compat::compute_action(U, beta), compute_action(U, beta)));
    put("compute_avg_plaq", rel(sfh_compat::compute_avg_plaq(U), compute_avg_plaq(U)));

    {  // production leapfrog stages with the global step size and count
        std::vector<double> Pr = P, Pg = P;
        Link_array Ur = U, Ug = U;
        apply_initial_step_to_conjugate_field(Pr, beta, phi, Ur);
        sfh_compat::apply_initial_step_to_conjugate_field(Pg, beta, phi, Ug);
        put("apply_initial_step_to_conjugate_field.P", rel(Pg, Pr));
        apply_intermediate_update_to_gauge_field_and_conjugate_field(Pr, beta, phi, Ur);
        sfh_compat::apply_intermediate_update_to_gauge_field_and_conjugate_field(Pg, beta, phi, Ug);
        put("apply_intermediate_update.U", rel(Ug, Ur));
        put("apply_intermediate_update.P", rel(Pg, Pr));
        std::vector<double> Xf = apply_final_step(Pr, beta, phi, Ur);
        std::vector<double> Xh = sfh_compat::apply_final_step(Pg, beta, phi, Ug);
        put("apply_final_step.U", rel(Ug, Ur));
        put("apply_final_step.P", rel(Pg, Pr));
        put("apply_final_step.X", rel(Xh, Xf));
    }
    {  // the parameterised copies and their fermion-only / gauge-only variants
        const double eps = 0.03;
        const int n = 3;
        std::vector<double> Pr = P, Pg = P;
        Link_array Ur = U, Ug = U;
        local_initial_half_step(Pr, beta, phi, Ur, eps);
        local_leapfrog_steps(Pr, beta, phi, Ur, eps, n);
        std::vector<double> Xf = local_final_step(Pr, beta, phi, Ur, eps);
        sfh_compat::local_initial_half_step(Pg, beta, phi, Ug, eps);
        sfh_compat::local_leapfrog_steps(Pg, beta, phi, Ug, eps, n);
        std::vector<double> Xh = sfh_compat::local_final_step(Pg, beta, phi, Ug, eps);
        put("local_leapfrog.U", rel(Ug, Ur));
        put("local_leapfrog.P", rel(Pg, Pr));
        put("local_leapfrog.X", rel(Xh, Xf));

        Pr = P, Pg = P, Ur = U, Ug = U;
        local_initial_half_step_fermion(Pr, phi, Ur, eps);
        local_leapfrog_steps_fermion(Pr, phi, Ur, eps, n);
        Xf = local_final_step_fermion(Pr, phi, Ur, eps);
        sfh_compat::local_initial_half_step_fermion(Pg, phi, Ug, eps);
        sfh_compat::local_leapfrog_steps_fermion(Pg, phi, Ug, eps, n);
        Xh = sfh_compat::local_final_step_fermion(Pg, phi, Ug, eps);
        put("local_leapfrog_fermion.U", rel(Ug, Ur));
        put("local_leapfrog_fermion.P", rel(Pg, Pr));
        put("local_leapfrog_fermion.X", rel(Xh, Xf));

        Pr = P, Pg = P, Ur = U, Ug = U;
        local_initial_half_step_gauge(Pr, beta, Ur, eps);
        local_leapfrog_steps_gauge(Pr, beta, Ur, eps, n);
        local_final_step_gauge(Pr, beta, Ur, eps);
        sfh_compat::local_initial_half_step_gauge(Pg, beta, Ug, eps);
        sfh_compat::local_leapfrog_steps_gauge(Pg, beta, Ug, eps, n);
        sfh_compat::local_final_step_gauge(Pg, beta, Ug, eps);
        put("local_leapfrog_gauge.U", rel(Ug, Ur));
        put("local_leapfrog_gauge.P", rel(Pg, Pr));
    }
    {
        std::vector<std::complex<double>> gr = precompute_polyakov_grid(U);
        std::vector<std::complex<double>> gg = sfh_compat::precompute_polyakov_grid(U);
        put("precompute_polyakov_grid", rel(gg, gr));
        double worst = 0.0;
        for (int r2 = 1; r2 <= 3; ++r2) {
            std::complex<double> cr = correlator_over_fixed_distance_fast(gr, r2);
            std::complex<double> cg = sfh_compat::correlator_over_fixed_distance_fast(gr, r2);
            worst = std::max(worst, std::abs(cg - cr) / std::max(std::abs(cr), 1e-300));
        }
        put("correlator_over_fixed_distance_fast", worst);
    }
    {  // the Metropolis update runs on the device; the field stays in SU(3)
        Link_array Ug = U;
        sfh_compat::single_sweep_monte_carlo_update_WITH_FERMIONS(Ug, beta);
        put("single_sweep.plaq_finite", std::isfinite(sfh_compat::compute_avg_plaq(Ug)) ? 1.0 : 0.0);
    }
    {  // error behaviour.  The reference throws from inside its OpenMP loops,
       // which ends the process, so only the library's side runs here; the
       // test compares the exception type and message with the reference's.
        std::vector<double> Pbad = P;
        Pbad[1] += 0.5;  // imaginary part of P_00: no longer Hermitian
        Link_array Ug = U;
        put_s("non_hermitian.compat", thrown([&] {
                  sfh_compat::apply_intermediate_update_to_gauge_field_and_conjugate_field(Pbad, beta, phi, Ug);
              }));
        sfh_compat::Settings s = SFH_COMPAT_PARAMETERS();
        s.max_iter = 2;
        sfh_compat::configure(s);
        put_s("noconv.compat", thrown([&] { sfh_compat::solve_CG_DDdagger(phi, U); }));
        sfh_compat::shutdown();
    }
    std::cout << "{" << js.str() << "}" << std::endl;
    return 0;
}
