// compat.cpp — the reference's field-level C++ functions (include/sfh_compat.hpp)
// on the C ABI.  Each function uploads its inputs, runs on the device and
// downloads its outputs; errors become the reference's exception types.
#include "sfh_compat.hpp"

#include <cmath>
#include <cstdio>
#include <fstream>
#include <iostream>
#include <stdexcept>

namespace sfh_compat {

namespace {

struct ThreadState {
    Settings s;
    sfh_ctx* ctx = nullptr;
    unsigned long long draws = 0;
    int sweeps = 0;  // heatbath sweeps so far (the sweep index of the uniforms)
};

thread_local ThreadState T;

// SplitMix64 (Steele, Lea, Flood 2014): per-draw seeds and the Metropolis uniform
unsigned long long mix64(unsigned long long z)
{
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

unsigned long long next_seed() { return mix64(T.s.seed * 0x100000001B3ull + (++T.draws)); }

double next_uniform() { return (double)(next_seed() >> 11) * (1.0 / 9007199254740992.0); }

[[noreturn]] void raise(int st)
{
    std::string msg = T.ctx ? sfh_last_error(T.ctx) : "";
    if (msg.empty()) msg = sfh_status_string(st);
    // exp(iQ) domain errors are std::invalid_argument (Fermions.cpp:848-857);
    // CG failures and a non-Hermitian momentum std::runtime_error (:574-614, :714-716)
    if (st == SFH_ERR_DOMAIN || st == SFH_ERR_INVALID) throw std::invalid_argument(msg);
    throw std::runtime_error(msg);
}

void check(int st)
{
    if (st != SFH_OK) raise(st);
}

sfh_ctx* ctx()
{
    if (!T.ctx) {
        sfh_params p{};
        for (int k = 0; k < 4; ++k) p.dims[k] = T.s.dims[k];
        p.mass = T.s.mass;
        p.beta = 0.0;
        p.c11 = T.s.c11;
        p.c12 = T.s.c12;
        p.device = T.s.device;
        sfh_ctx* c = nullptr;
        int st = sfh_create(&p, &c);
        if (st != SFH_OK) throw std::runtime_error(std::string("sfh_create: ") + sfh_status_string(st));
        T.ctx = c;
    }
    return T.ctx;
}

size_t volume() { return (size_t)T.s.dims[0] * T.s.dims[1] * T.s.dims[2] * T.s.dims[3]; }

void need(const std::vector<double>& v, size_t n, const char* what)
{
    if (v.size() != n)
        throw std::invalid_argument(std::string(what) + ": expected " + std::to_string(n) + " doubles, got " +
                                    std::to_string(v.size()));
}

void gauge_in(const Link_array& arr)
{
    need(arr, 72 * volume(), "gauge field");
    check(sfh_upload_gauge(ctx(), arr.data()));
}

void gauge_out(Link_array& arr)
{
    arr.resize(72 * volume());
    check(sfh_download_gauge(ctx(), arr.data()));
}

void momenta_in(const std::vector<double>& P)
{
    need(P, 72 * volume(), "conjugate field");
    check(sfh_upload_momenta(ctx(), P.data()));
}

void momenta_out(std::vector<double>& P) { check(sfh_download_momenta(ctx(), P.data())); }

void kick(int forces, const std::vector<double>* phi, double dt, std::vector<double>* X)
{
    if (phi) need(*phi, 6 * volume(), "phi field");
    if (X) X->resize(6 * volume());
    check(sfh_momentum_kick(ctx(), forces, phi ? phi->data() : nullptr, dt, T.s.tol, T.s.max_iter, T.s.precision,
                            X ? X->data() : nullptr, nullptr));
}

void update(double eps, int check_p) { check(sfh_link_update(ctx(), eps, check_p)); }

double dot(const std::vector<double>& a, const std::vector<double>& b)
{
    double s = 0.0;
    for (size_t i = 0; i < a.size(); ++i) s += a[i] * b[i];
    return s;
}

void report(double T0, double T1, double S0, double S1, double F0, double F1)
{
    // the lines Monte_carlo_step prints (Fermions.cpp:794-800)
    std::cout << "Initial Tr(P^2): " << T0 << std::endl;
    std::cout << "Final Tr(P^2): " << T1 << std::endl;
    std::cout << "Initial Gauge Action: " << S0 << std::endl;
    std::cout << "Final Gauge Action: " << S1 << std::endl;
    std::cout << "Initial Fermion Action: " << F0 << std::endl;
    std::cout << "Final Fermion Action: " << F1 << std::endl;
    std::cout << (T0 - T1) + (S0 - S1) + (F0 - F1) << std::endl;
}

}  // namespace

void configure(const Settings& s)
{
    shutdown();
    T.s = s;
    T.draws = 0;
    T.sweeps = 0;
}

const Settings& settings() { return T.s; }

void shutdown()
{
    if (T.ctx) sfh_destroy(T.ctx);
    T.ctx = nullptr;
}

// ---- Fermions.h -------------------------------------------------------------

void apply_DDdagger(const std::vector<double>& in_field, const Link_array& arr, std::vector<double>& out_field)
{
    need(in_field, 6 * volume(), "fermion field");
    gauge_in(arr);
    out_field.resize(6 * volume());
    check(sfh_ddag(ctx(), in_field.data(), out_field.data()));
}

std::vector<double> solve_CG_DDdagger(const std::vector<double>& phi_field, const Link_array& arr)
{
    need(phi_field, 6 * volume(), "phi field");
    gauge_in(arr);
    std::vector<double> X(6 * volume());
    check(sfh_cg_solve(ctx(), phi_field.data(), X.data(), T.s.tol, T.s.max_iter, T.s.precision, nullptr));
    return X;
}

std::vector<double> solve_X_field(const std::vector<double>& phi_field, const Link_array& arr)
{
    return solve_CG_DDdagger(phi_field, arr);
}

std::vector<double> solve_Y_field(const std::vector<double>& X_field, const Link_array& arr)
{
    need(X_field, 6 * volume(), "X field");
    gauge_in(arr);
    std::vector<double> Y(6 * volume());
    check(sfh_dirac(ctx(), 1, X_field.data(), Y.data()));
    return Y;
}

std::vector<double> compute_full_force_field(const std::vector<double>& X_field, const std::vector<double>& Y_field,
                                             const Link_array& arr, double beta)
{
    need(X_field, 6 * volume(), "X field");
    need(Y_field, 6 * volume(), "Y field");
    gauge_in(arr);
    check(sfh_set_beta(ctx(), beta));
    std::vector<double> F(72 * volume());
    check(sfh_full_force(ctx(), X_field.data(), Y_field.data(), F.data()));
    return F;
}

std::vector<double> compute_fermion_only_force_field(const std::vector<double>& X_field,
                                                     const std::vector<double>& Y_field, const Link_array& arr)
{
    need(X_field, 6 * volume(), "X field");
    need(Y_field, 6 * volume(), "Y field");
    gauge_in(arr);
    std::vector<double> F(72 * volume());
    check(sfh_fermion_force(ctx(), X_field.data(), Y_field.data(), F.data()));
    return F;
}

std::vector<double> compute_gauge_only_force_field(const Link_array& arr, double beta)
{
    gauge_in(arr);
    check(sfh_set_beta(ctx(), beta));
    std::vector<double> F(72 * volume());
    check(sfh_gauge_force(ctx(), F.data()));
    return F;
}

double compute_Tr_P2(const std::vector<double>& P_field)
{
    momenta_in(P_field);
    double t = 0.0;
    check(sfh_trp2(ctx(), &t));
    return t;
}

std::vector<double> generate_phi_field(const Link_array& arr)
{
    // phi = D chi, chi complex Gaussian with variance 1/2 per real part (Fermions.cpp:302-314)
    gauge_in(arr);
    std::vector<double> chi(6 * volume()), phi(6 * volume());
    check(sfh_gaussian_spinor(ctx(), next_seed(), 1.0 / std::sqrt(2.0), chi.data()));
    check(sfh_dirac(ctx(), 0, chi.data(), phi.data()));
    return phi;
}

std::vector<double> generate_conjugate_field_configuration()
{
    std::vector<double> P(72 * volume());
    check(sfh_random_momenta(ctx(), next_seed()));
    momenta_out(P);
    return P;
}

void apply_initial_step_to_conjugate_field(std::vector<double>& P_field, double beta,
                                           const std::vector<double>& phi_field, const Link_array& arr)
{
    gauge_in(arr);
    momenta_in(P_field);
    check(sfh_set_beta(ctx(), beta));
    kick(SFH_FORCE_GAUGE | SFH_FORCE_FERMION, &phi_field, 0.5 * T.s.epsilon, nullptr);
    momenta_out(P_field);
}

void apply_intermediate_update_to_gauge_field_and_conjugate_field(std::vector<double>& P_field, double beta,
                                                                  const std::vector<double>& phi_field,
                                                                  Link_array& arr)
{
    gauge_in(arr);
    momenta_in(P_field);
    check(sfh_set_beta(ctx(), beta));
    for (int n = 1; n < T.s.number_of_steps; ++n) {
        update(T.s.epsilon, 1);
        kick(SFH_FORCE_GAUGE | SFH_FORCE_FERMION, &phi_field, T.s.epsilon, nullptr);
    }
    gauge_out(arr);
    momenta_out(P_field);
}

std::vector<double> apply_final_step(std::vector<double>& P_field, double beta,
                                     const std::vector<double>& phi_field, Link_array& arr)
{
    gauge_in(arr);
    momenta_in(P_field);
    check(sfh_set_beta(ctx(), beta));
    update(T.s.epsilon, 1);
    std::vector<double> X;
    kick(SFH_FORCE_GAUGE | SFH_FORCE_FERMION, &phi_field, 0.5 * T.s.epsilon, &X);
    gauge_out(arr);
    momenta_out(P_field);
    return X;
}

void Monte_carlo_step(double initial_Tr_P2, double initial_phi_field_action,
                      const std::vector<double>& P_field_final, const std::vector<double>& phi_field,
                      double gauge_field_initial_action, Link_array& gauge_field_initial,
                      Link_array& gauge_field_final, const std::vector<double>& X_field, double beta)
{
    double r = next_uniform();
    double T1 = compute_Tr_P2(P_field_final);
    double S1 = compute_action(gauge_field_final, beta);
    double F1 = dot(phi_field, X_field);
    report(initial_Tr_P2, T1, gauge_field_initial_action, S1, initial_phi_field_action, F1);
    double d = (initial_Tr_P2 - T1) + (gauge_field_initial_action - S1) + (initial_phi_field_action - F1);
    if (r < std::exp(d)) gauge_field_initial = gauge_field_final;  // Fermions.cpp:805-808
}

void single_sweep_monte_carlo_update_WITH_FERMIONS(Link_array& gauge_field, double beta)
{
    gauge_in(gauge_field);
    check(sfh_set_beta(ctx(), beta));
    sfh_traj_info info;
    check(sfh_hmc_trajectory(ctx(), T.s.epsilon, T.s.number_of_steps, next_seed(), T.s.tol, T.s.max_iter,
                             T.s.precision, &info));
    report(info.H_initial[0], info.H_final[0], info.H_initial[1], info.H_final[1], info.H_initial[2],
           info.H_final[2]);
    gauge_out(gauge_field);  // the accepted or the restored field
}

void local_initial_half_step(std::vector<double>& P_field, double beta, const std::vector<double>& phi_field,
                             const Link_array& arr, double eps)
{
    gauge_in(arr);
    momenta_in(P_field);
    check(sfh_set_beta(ctx(), beta));
    kick(SFH_FORCE_GAUGE | SFH_FORCE_FERMION, &phi_field, 0.5 * eps, nullptr);
    momenta_out(P_field);
}

void local_leapfrog_steps(std::vector<double>& P_field, double beta, const std::vector<double>& phi_field,
                          Link_array& arr, double eps, int n_steps)
{
    gauge_in(arr);
    momenta_in(P_field);
    check(sfh_set_beta(ctx(), beta));
    for (int n = 1; n < n_steps; ++n) {
        update(eps, 0);
        kick(SFH_FORCE_GAUGE | SFH_FORCE_FERMION, &phi_field, eps, nullptr);
    }
    gauge_out(arr);
    momenta_out(P_field);
}

std::vector<double> local_final_step(std::vector<double>& P_field, double beta,
                                     const std::vector<double>& phi_field, Link_array& arr, double eps)
{
    gauge_in(arr);
    momenta_in(P_field);
    check(sfh_set_beta(ctx(), beta));
    update(eps, 0);
    std::vector<double> X;
    kick(SFH_FORCE_GAUGE | SFH_FORCE_FERMION, &phi_field, 0.5 * eps, &X);
    gauge_out(arr);
    momenta_out(P_field);
    return X;
}

void local_initial_half_step_fermion(std::vector<double>& P_field, const std::vector<double>& phi_field,
                                     const Link_array& arr, double eps)
{
    gauge_in(arr);
    momenta_in(P_field);
    kick(SFH_FORCE_FERMION, &phi_field, 0.5 * eps, nullptr);
    momenta_out(P_field);
}

void local_leapfrog_steps_fermion(std::vector<double>& P_field, const std::vector<double>& phi_field,
                                  Link_array& arr, double eps, int n_steps)
{
    gauge_in(arr);
    momenta_in(P_field);
    for (int n = 1; n < n_steps; ++n) {
        update(eps, 0);
        kick(SFH_FORCE_FERMION, &phi_field, eps, nullptr);
    }
    gauge_out(arr);
    momenta_out(P_field);
}

std::vector<double> local_final_step_fermion(std::vector<double>& P_field, const std::vector<double>& phi_field,
                                             Link_array& arr, double eps)
{
    gauge_in(arr);
    momenta_in(P_field);
    update(eps, 0);
    std::vector<double> X;
    kick(SFH_FORCE_FERMION, &phi_field, 0.5 * eps, &X);
    gauge_out(arr);
    momenta_out(P_field);
    return X;
}

void local_initial_half_step_gauge(std::vector<double>& P_field, double beta, const Link_array& arr, double eps)
{
    gauge_in(arr);
    momenta_in(P_field);
    check(sfh_set_beta(ctx(), beta));
    kick(SFH_FORCE_GAUGE, nullptr, 0.5 * eps, nullptr);
    momenta_out(P_field);
}

void local_leapfrog_steps_gauge(std::vector<double>& P_field, double beta, Link_array& arr, double eps,
                                int n_steps)
{
    gauge_in(arr);
    momenta_in(P_field);
    check(sfh_set_beta(ctx(), beta));
    for (int n = 1; n < n_steps; ++n) {
        update(eps, 0);
        kick(SFH_FORCE_GAUGE, nullptr, eps, nullptr);
    }
    gauge_out(arr);
    momenta_out(P_field);
}

void local_final_step_gauge(std::vector<double>& P_field, double beta, Link_array& arr, double eps)
{
    gauge_in(arr);
    momenta_in(P_field);
    check(sfh_set_beta(ctx(), beta));
    update(eps, 0);
    kick(SFH_FORCE_GAUGE, nullptr, 0.5 * eps, nullptr);
    gauge_out(arr);
    momenta_out(P_field);
}

// ---- Lattice.h --------------------------------------------------------------

double compute_action(const Link_array& arr, double beta)
{
    gauge_in(arr);
    check(sfh_set_beta(ctx(), beta));
    double s = 0.0;
    check(sfh_gauge_action(ctx(), &s));
    return s;
}

double compute_avg_plaq(const Link_array& arr)
{
    gauge_in(arr);
    double s = 0.0;
    check(sfh_plaquette(ctx(), &s));
    return s;
}

std::pair<double, double> heatbath_update(Link_array& arr, double beta)
{
    gauge_in(arr);
    check(sfh_set_beta(ctx(), beta));
    double plaq = 0.0, act = 0.0;
    check(sfh_heatbath(ctx(), 1, T.s.seed, T.sweeps++, &plaq, &act));
    gauge_out(arr);
    return {plaq, act};
}

std::vector<std::complex<double>> precompute_polyakov_grid(const Link_array& arr)
{
    gauge_in(arr);
    std::vector<std::complex<double>> grid((size_t)T.s.dims[0] * T.s.dims[1] * T.s.dims[2]);
    check(sfh_polyakov_grid(ctx(), reinterpret_cast<double*>(grid.data())));
    return grid;
}

std::complex<double> correlator_over_fixed_distance_fast(const std::vector<std::complex<double>>& P_grid,
                                                         int r_squared)
{
    if (P_grid.size() != (size_t)T.s.dims[0] * T.s.dims[1] * T.s.dims[2])
        throw std::invalid_argument("P_grid must hold one value per spatial site");
    double out[2];
    check(sfh_polyakov_correlator_grid(ctx(), reinterpret_cast<const double*>(P_grid.data()), r_squared, out));
    return {out[0], out[1]};
}

bool save_lattice_configs(const Link_array* links, int n, const std::string& filename)
{
    std::ofstream out(filename, std::ios::binary);
    if (!out) {
        std::cerr << "Error opening file for writing: " << filename << "\n";
        return false;
    }
    for (int i = 0; i < n; ++i)
        out.write(reinterpret_cast<const char*>(links[i].data()), (std::streamsize)(links[i].size() * sizeof(double)));
    if (!out) {
        std::cerr << "Error writing complete binary data to: " << filename << "\n";
        return false;
    }
    return true;
}

bool load_lattice_configs(Link_array* links, int n, const std::string& filename)
{
    std::ifstream in(filename, std::ios::binary);
    if (!in) {
        std::cerr << "Error opening file for reading: " << filename << "\n";
        return false;
    }
    for (int i = 0; i < n; ++i)
        in.read(reinterpret_cast<char*>(links[i].data()), (std::streamsize)(links[i].size() * sizeof(double)));
    if (!in) {
        std::cerr << "Error reading complete binary data from: " << filename << "\n";
        return false;
    }
    return true;
}

// ---- Smearing.h -------------------------------------------------------------

void Apply_HEX_smearing(Link_array& U_array)
{
    gauge_in(U_array);
    check(sfh_smear_hex(ctx(), T.s.alpha[0], T.s.alpha[1], T.s.alpha[2], 1));
    gauge_out(U_array);
}

void Apply_4HEX_smearing(Link_array& U_array)
{
    gauge_in(U_array);
    check(sfh_smear_hex(ctx(), T.s.alpha[0], T.s.alpha[1], T.s.alpha[2], 4));
    gauge_out(U_array);
}

}  // namespace sfh_compat
