// sfh_compat.hpp — the reference's field-level C++ API on top of the C ABI.
//
// Same names, argument meaning, layouts and error behaviour as the free
// functions of alexanderchasteen/Staggered_Fermions_HMC (Fermions.h:29-145,
// Lattice.h:76-82, Smearing.h:29-31): host std::vector<double> fields in the
// reference's AoS layouts, results returned by value, in-place updates
// through non-const references, std::runtime_error / std::invalid_argument
// on failure.  They live in namespace sfh_compat, so they link beside the
// reference's own definitions; a driver switches by qualifying its calls
// (or `using namespace sfh_compat;` in place of the reference's headers).
//
// The reference fixes lattice size, mass, CG tolerance, step size and step
// count at compile time (Parameters.h); here they are run-time settings,
// given once through configure().  Inside the reference's tree,
// SFH_COMPAT_PARAMETERS() builds the settings from Parameters.h's constants.
//
// Every call uploads its input fields to the device, runs there and
// downloads its outputs; a whole HMC update
// (single_sweep_monte_carlo_update_WITH_FERMIONS) stays on the device from
// start to end.  One device context per thread; not re-entrant per thread.
#ifndef SFH_COMPAT_HPP
#define SFH_COMPAT_HPP

#include <array>
#include <complex>
#include <utility>
#include <string>
#include <vector>

#include "sfh.h"

namespace sfh_compat {

using Link_array = std::vector<double>;  // Lattice.h:12

struct Settings {
    int dims[4] = {4, 4, 4, 4};         // Spatial_Size x3, temporal_size (Parameters.h:9-10)
    double mass = 1.0;                  // fermion_mass (Parameters.h:18)
    double tol = 1e-12;                 // CG relative tolerance (Parameters.h:23)
    int max_iter = 50000;               // Parameters.h:24
    double epsilon = 1e-2;              // MD step (Parameters.h:21)
    int number_of_steps = 100;          // number_of_steps_fermion (Parameters.h:22)
    double c11 = 5.0 / 3.0;             // Parameters.h:51
    double c12 = -1.0 / 12.0;           // Parameters.h:52
    double alpha[3] = {0.95, 0.76, 0.38};  // HEX alpha1..3 (Smearing.h:7-9)
    int precision = SFH_PREC_F64;       // SFH_PREC_F64 runs the reference's own CG
    int device = 0;
    unsigned long long seed = 1;        // pseudofermion / momentum / Metropolis draws
};

// Settings for every later call on this thread (re-creates the device context).
void configure(const Settings& s);
const Settings& settings();
// Releases this thread's device context.
void shutdown();

// ---- Fermions.h -------------------------------------------------------------
void apply_DDdagger(const std::vector<double>& in_field, const Link_array& arr, std::vector<double>& out_field);
std::vector<double> solve_CG_DDdagger(const std::vector<double>& phi_field, const Link_array& arr);
std::vector<double> solve_X_field(const std::vector<double>& phi_field, const Link_array& arr);
std::vector<double> solve_Y_field(const std::vector<double>& X_field, const Link_array& arr);
std::vector<double> compute_full_force_field(const std::vector<double>& X_field, const std::vector<double>& Y_field,
                                             const Link_array& arr, double beta);
std::vector<double> compute_fermion_only_force_field(const std::vector<double>& X_field,
                                                     const std::vector<double>& Y_field, const Link_array& arr);
std::vector<double> compute_gauge_only_force_field(const Link_array& arr, double beta);
double compute_Tr_P2(const std::vector<double>& P_field);

std::vector<double> generate_phi_field(const Link_array& arr);
std::vector<double> generate_conjugate_field_configuration();

void apply_initial_step_to_conjugate_field(std::vector<double>& P_field, double beta,
                                           const std::vector<double>& phi_field, const Link_array& arr);
void apply_intermediate_update_to_gauge_field_and_conjugate_field(std::vector<double>& P_field, double beta,
                                                                  const std::vector<double>& phi_field,
                                                                  Link_array& arr);
std::vector<double> apply_final_step(std::vector<double>& P_field, double beta,
                                     const std::vector<double>& phi_field, Link_array& arr);
void Monte_carlo_step(double initial_Tr_P2, double initial_phi_field_action,
                      const std::vector<double>& P_field_final, const std::vector<double>& phi_field,
                      double gauge_field_initial_action, Link_array& gauge_field_initial,
                      Link_array& gauge_field_final, const std::vector<double>& X_field, double beta);
void single_sweep_monte_carlo_update_WITH_FERMIONS(Link_array& gauge_field, double beta);

void local_initial_half_step(std::vector<double>& P_field, double beta, const std::vector<double>& phi_field,
                             const Link_array& arr, double eps);
void local_leapfrog_steps(std::vector<double>& P_field, double beta, const std::vector<double>& phi_field,
                          Link_array& arr, double eps, int n_steps);
std::vector<double> local_final_step(std::vector<double>& P_field, double beta,
                                     const std::vector<double>& phi_field, Link_array& arr, double eps);
void local_initial_half_step_fermion(std::vector<double>& P_field, const std::vector<double>& phi_field,
                                     const Link_array& arr, double eps);
void local_leapfrog_steps_fermion(std::vector<double>& P_field, const std::vector<double>& phi_field,
                                  Link_array& arr, double eps, int n_steps);
std::vector<double> local_final_step_fermion(std::vector<double>& P_field, const std::vector<double>& phi_field,
                                             Link_array& arr, double eps);
void local_initial_half_step_gauge(std::vector<double>& P_field, double beta, const Link_array& arr, double eps);
void local_leapfrog_steps_gauge(std::vector<double>& P_field, double beta, Link_array& arr, double eps,
                                int n_steps);
void local_final_step_gauge(std::vector<double>& P_field, double beta, Link_array& arr, double eps);

// ---- Lattice.h --------------------------------------------------------------
double compute_action(const Link_array& arr, double beta);
double compute_avg_plaq(const Link_array& arr);
// one heatbath sweep (Lattice.cpp:722-757); returns (average plaquette, action
// per site) after the sweep.  Seeded: the sweeps of a thread draw from the
// settings' seed and a sweep counter.
std::pair<double, double> heatbath_update(Link_array& arr, double beta);
std::vector<std::complex<double>> precompute_polyakov_grid(const Link_array& arr);
std::complex<double> correlator_over_fixed_distance_fast(const std::vector<std::complex<double>>& P_grid,
                                                         int r_squared);

// save_all_lattice_configs / load_all_lattice_configs (Lattice.cpp:806-847):
// the CONFIG link arrays back to back as raw native doubles.
bool save_lattice_configs(const Link_array* links, int n, const std::string& filename);
bool load_lattice_configs(Link_array* links, int n, const std::string& filename);
template <std::size_t N>
bool save_all_lattice_configs(const std::array<Link_array, N>& links, const std::string& filename)
{
    return save_lattice_configs(links.data(), (int)N, filename);
}
template <std::size_t N>
bool load_all_lattice_configs(std::array<Link_array, N>& links, const std::string& filename)
{
    return load_lattice_configs(links.data(), (int)N, filename);
}

// ---- Smearing.h -------------------------------------------------------------
void Apply_HEX_smearing(Link_array& U_array);
void Apply_4HEX_smearing(Link_array& U_array);

}  // namespace sfh_compat

// Settings from the reference's Parameters.h constants (use inside its tree).
#define SFH_COMPAT_PARAMETERS()                                                              \
    ([] {                                                                                    \
        sfh_compat::Settings s_;                                                             \
        s_.dims[0] = s_.dims[1] = s_.dims[2] = Spatial_Size;                                 \
        s_.dims[3] = temporal_size;                                                          \
        s_.mass = fermion_mass;                                                              \
        s_.tol = tol;                                                                        \
        s_.max_iter = max_iter;                                                              \
        s_.epsilon = epsilon;                                                                \
        s_.number_of_steps = number_of_steps_fermion;                                        \
        s_.c11 = c_11;                                                                       \
        s_.c12 = c_12;                                                                       \
        return s_;                                                                           \
    }())

#endif
