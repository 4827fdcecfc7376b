// hmc.cu — C ABI for forces, the link update, observables and the leapfrog /
// HMC trajectory, all on the context's device-resident fields.
//
// The trajectory follows single_sweep_monte_carlo_update_WITH_FERMIONS
// (Fermions.cpp:812-828): S_g, phi = D chi, P, Tr P^2, X0 = (D D^dag)^-1 phi,
// phi.X0, leapfrog (half kick, N-1 x (link update, kick), link update, half
// kick; Fermions.cpp:684-776 / 967-1028), then H_final and the Metropolis
// test of Monte_carlo_step (Fermions.cpp:778-810).  Every force evaluation is
// one CG solve, Y = D^dag X and one fused kernel P -= k (F_gauge + F_fermion).
#include <chrono>
#include <cmath>
#include <cstring>
#include <string>

#include "sfh_internal.h"

namespace sfh {
int set_error(sfh_ctx* c, int code, const std::string& msg);
int cuda_check(sfh_ctx* c, cudaError_t e, const char* what);
}  // namespace sfh

using namespace sfh;

namespace {

size_t spinor_bytes(const sfh_ctx* c) { return (size_t)c->g.V * 6 * sizeof(double); }
size_t link_bytes(const sfh_ctx* c) { return (size_t)c->g.V * 72 * sizeof(double); }

int take_device_error(sfh_ctx* c, const char* what)
{
    int h = 0;
    int st = cuda_check(c, cudaMemcpyAsync(&h, c->derr, sizeof(int), cudaMemcpyDeviceToHost, c->stream), what);
    if (!st) st = cuda_check(c, cudaMemsetAsync(c->derr, 0, sizeof(int), c->stream), what);
    if (!st) st = cuda_check(c, cudaStreamSynchronize(c->stream), what);
    if (st) return st;
    if (h & DEV_ERR_NOT_HERMITIAN)  // Fermions.cpp:714-716
        return set_error(c, SFH_ERR_NOT_HERMITIAN, std::string(what) + ": P_pre is not Hermitian or not traceless");
    if (h & DEV_ERR_DOMAIN)  // Fermions.cpp:848-857
        return set_error(c, SFH_ERR_DOMAIN, std::string(what) + ": exp(iQ) argument outside its domain");
    return SFH_OK;
}

int spinor_in(sfh_ctx* c, const double* host, void* eo)
{
    int st = cuda_check(c, cudaMemcpyAsync(c->stage, host, spinor_bytes(c), cudaMemcpyHostToDevice, c->stream),
                        "spinor upload");
    if (st) return st;
    launch_spinor_aos_to_eo(c->g, (const double*)c->stage, eo, c->stream);
    return SFH_OK;
}

int spinor_out(sfh_ctx* c, const void* eo, double* host)
{
    launch_spinor_eo_to_aos(c->g, eo, (double*)c->stage, c->stream);
    int st = cuda_check(c, cudaMemcpyAsync(host, c->stage, spinor_bytes(c), cudaMemcpyDeviceToHost, c->stream),
                        "spinor download");
    if (st) return st;
    return cuda_check(c, cudaStreamSynchronize(c->stream), "spinor download");
}

int links_out(sfh_ctx* c, const void* eo, double* host)
{
    launch_links_eo_to_aos(c->g, eo, (double*)c->stage, c->stream);
    int st = cuda_check(c, cudaMemcpyAsync(host, c->stage, link_bytes(c), cudaMemcpyDeviceToHost, c->stream),
                        "link field download");
    if (st) return st;
    return cuda_check(c, cudaStreamSynchronize(c->stream), "link field download");
}

int reduce(sfh_ctx* c, int kind, const void* A, const void* B, double* out)
{
    int st = cuda_check(c, launch_reduce(c->g, kind, A, B, c->beta, c->c11, c->c12, c->red, c->red + 2048,
                                         c->stream), "reduction");
    if (st) return st;
    st = cuda_check(c, cudaMemcpyAsync(out, c->red + 2048, sizeof(double), cudaMemcpyDeviceToHost, c->stream),
                    "reduction");
    if (st) return st;
    return cuda_check(c, cudaStreamSynchronize(c->stream), "reduction");
}

}  // namespace

namespace sfh {
int ensure_scratch(sfh_ctx* c, int nfields);
}

namespace {

// ---------------------------------------------------------------------------
// Stout-smeared fermion links (no counterpart in the reference): the fermion
// operator uses V = stout^n(U), the gauge action the thin U.  Scratch link
// fields: levels 0..n (level 0 = the thin field), then G, Gn, W of the chain
// rule.  While a smeared operation runs, U64 holds V (so the solver and the
// operators use it) and level 0 keeps U; smear_out puts U back.
// ---------------------------------------------------------------------------
constexpr int kMaxSmearLevels = 16;

void* scratch_field(sfh_ctx* c, int k) { return (char*)c->smear + (size_t)k * c->g.V * 4 * 9 * 16; }

int ensure_hasen(sfh_ctx* c)
{
    int st = SFH_OK;
    if (!c->hphi) st = cuda_check(c, cudaMalloc(&c->hphi, spinor_bytes(c)), "heavy pseudofermion");
    if (!st && !c->hX) st = cuda_check(c, cudaMalloc(&c->hX, spinor_bytes(c)), "heavy pseudofermion");
    return st;
}

int smear_in(sfh_ctx* c)
{
    int st = ensure_scratch(c, c->fsmear_n + 4);
    if (st) return st;
    void* lev[kMaxSmearLevels + 1];
    for (int k = 0; k <= c->fsmear_n; ++k) lev[k] = scratch_field(c, k);
    st = cuda_check(c, cudaMemcpyAsync(lev[0], c->U64, link_bytes(c), cudaMemcpyDeviceToDevice, c->stream),
                    "smearing");
    if (!st) st = cuda_check(c, launch_stout_levels(c->g, lev, c->fsmear_rho, c->fsmear_n, c->derr, c->stream),
                             "smearing");
    if (!st) st = cuda_check(c, cudaMemcpyAsync(c->U64, lev[c->fsmear_n], link_bytes(c), cudaMemcpyDeviceToDevice,
                                                c->stream), "smearing");
    c->lowp_valid = false;
    if (!st) st = take_device_error(c, "fermion-link smearing");
    return st;
}

int smear_out(sfh_ctx* c)
{
    int st = cuda_check(c, cudaMemcpyAsync(c->U64, scratch_field(c, 0), link_bytes(c), cudaMemcpyDeviceToDevice,
                                           c->stream), "smearing");
    c->lowp_valid = false;
    return st;
}

// ---------------------------------------------------------------------------
// Pseudofermion terms.  One pseudofermion: S_f = phi^dag M(m)^-1 phi with
// M(m) = D(m) D(m)^dag.  With a Hasenbusch heavy mass m_h (no counterpart in
// the reference): S_f = phi_h^dag M(m_h)^-1 phi_h + phi^dag M(m_h) M(m)^-1 phi,
// and since M(m_h) M(m)^-1 = 1 + (m_h^2 - m^2) M(m)^-1 every term is a weight
// times phi_k^dag M(m_k)^-1 phi_k (plus |phi|^2, constant in the MD).  The
// fermion force of a term is compute_fermion_force_at_link (Fermions.cpp:
// 443-515) of X_k = M(m_k)^-1 phi_k, Y_k = D(m_k)^dag X_k, times its weight.
// ---------------------------------------------------------------------------
struct PfTerm {
    const void* phi;
    void* X;
    double mass, weight;
};

int pf_terms(sfh_ctx* c, const void* phi, void* X, PfTerm (&t)[2])
{
    if (c->hasen_mass > 0.0) {
        t[0] = {c->hphi, c->hX, c->hasen_mass, 1.0};
        t[1] = {phi, X, c->mass, c->hasen_mass * c->hasen_mass - c->mass * c->mass};
        return 2;
    }
    t[0] = {phi, X, c->mass, 1.0};
    return 1;
}

// X_k = M(m_k)^-1 phi_k for the pseudofermion terms: a Hasenbusch pair as
// one system with two right-hand sides at their own masses on the same
// links, a single term alone
int solve_terms(sfh_ctx* c, const PfTerm* t, int n, double tol, int maxit, int prec, long* iters, int* solves)
{
    if (n == 2) {
        const void* b[2] = {t[0].phi, t[1].phi};
        void* x[2] = {t[0].X, t[1].X};
        const double ms[2] = {t[0].mass, t[1].mass};
        sfh_cg_info inf[2];
        std::memset(inf, 0, sizeof(inf));
        int st = ctx_solve_pair_device(c, b, x, ms, tol, maxit, prec, inf);
        if (iters) *iters += inf[0].iters + inf[1].iters;
        if (solves) *solves += 2;
        return st;
    }
    const double m = c->mass;
    c->mass = t[0].mass;
    sfh_cg_info inf;
    std::memset(&inf, 0, sizeof(inf));
    int st = ctx_solve_device(c, t[0].phi, t[0].X, tol, maxit, prec, &inf);
    c->mass = m;
    if (iters) *iters += inf.iters;
    if (solves) *solves += 1;
    return st;
}

// Fbuf = sum_k w_k F_f(X_k, Y_k) on the links in U64
int fermion_force_terms(sfh_ctx* c, const void* phi, void* X, void* Y, double tol, int maxit, int prec,
                        long* iters, int* solves)
{
    PfTerm t[2];
    const int n = pf_terms(c, phi, X, t);
    const double m = c->mass;
    int st = cuda_check(c, cudaMemsetAsync(c->Fbuf, 0, link_bytes(c), c->stream), "fermion force");
    if (!st) st = solve_terms(c, t, n, tol, maxit, prec, iters, solves);
    for (int k = 0; k < n && !st; ++k) {
        c->mass = t[k].mass;
        launch_hop(c->g, GP_F64_18, c->U64, SP_F64, t[k].X, SP_F64, Y, t[k].X, t[k].mass, -1.0, 0, 2, c->stream);
        // Fbuf -= (-w) F: the kick form of force_kernel accumulates w F
        st = cuda_check(c, launch_force(c->g, c->U64, t[k].X, Y, c->beta, c->c11, c->c12, 2, nullptr, c->Fbuf,
                                        -t[k].weight, c->stream), "fermion force");
    }
    c->mass = m;
    return st;
}

// the fermion force on the thin links into Fbuf, through the smearing levels
// when the fermion links are smeared
int fermion_force_general(sfh_ctx* c, const void* phi, void* X, void* Y, double tol, int maxit, int prec,
                          long* iters, int* solves)
{
    if (c->fsmear_n == 0) return fermion_force_terms(c, phi, X, Y, tol, maxit, prec, iters, solves);
    int st = smear_in(c);
    if (!st) st = fermion_force_terms(c, phi, X, Y, tol, maxit, prec, iters, solves);
    int st2 = smear_out(c);
    if (st) return st;
    if (st2) return st2;
    void* lev[kMaxSmearLevels + 1];
    for (int k = 0; k <= c->fsmear_n; ++k) lev[k] = scratch_field(c, k);
    const int n = c->fsmear_n;
    st = cuda_check(c, launch_stout_force(c->g, lev, n, c->fsmear_rho, c->Fbuf, scratch_field(c, n + 1),
                                          scratch_field(c, n + 2), scratch_field(c, n + 3), c->derr, c->stream),
                    "stout chain rule");
    if (!st) st = take_device_error(c, "stout chain rule");
    return st;
}

int smeared_fermion_force(sfh_ctx* c, const void* phi, void* X, void* Y, double tol, int maxit, int prec,
                          long* iters, int* solves)
{
    return fermion_force_general(c, phi, X, Y, tol, maxit, prec, iters, solves);
}

// S_f = sum_k w_k phi_k . X_k (+ |phi|^2 for a Hasenbusch pair) with solves on
// the current fermion links (smeared when set)
int fermion_action(sfh_ctx* c, const void* phi, void* X, double tol, int maxit, int prec, double* S, long* iters,
                   int* solves)
{
    PfTerm t[2];
    const int n = pf_terms(c, phi, X, t);
    const double m = c->mass;
    int st = c->fsmear_n > 0 ? smear_in(c) : SFH_OK;
    double sum = 0.0;
    if (!st) st = solve_terms(c, t, n, tol, maxit, prec, iters, solves);
    for (int k = 0; k < n && !st; ++k) {
        double d = 0.0;
        st = reduce(c, RED_DOT, t[k].phi, t[k].X, &d);
        sum += t[k].weight * d;
    }
    c->mass = m;
    if (!st && n == 2) {
        double pp = 0.0;
        st = reduce(c, RED_DOT, phi, phi, &pp);
        sum += pp;
    }
    if (c->fsmear_n > 0) {
        int st2 = smear_out(c);
        if (!st) st = st2;
    }
    *S = sum;
    return st;
}

// one force evaluation and momentum kick: X = (D D^dag)^-1 phi, Y = D^dag X,
// P -= kick (F_g + F_f)  (local_* of Fermions.cpp:967-1028); with smeared
// fermion links or a Hasenbusch pair F_f is the sum over the pseudofermion
// terms, through the smearing chain rule
int force_and_kick(sfh_ctx* c, const void* phi, void* X, void* Y, double kick, double tol, int maxit, int prec,
                   long* iters, int* solves)
{
    if (c->fsmear_n > 0 || c->hasen_mass > 0.0) {
        int st = fermion_force_general(c, phi, X, Y, tol, maxit, prec, iters, solves);
        if (!st) st = cuda_check(c, launch_link_axpy(c->g, c->Pmom, -kick, c->Fbuf, c->stream), "kick");
        if (!st) st = cuda_check(c, launch_force(c->g, c->U64, nullptr, nullptr, c->beta, c->c11, c->c12, 1, nullptr,
                                                 c->Pmom, kick, c->stream), "gauge kick");
        return st;
    }
    sfh_cg_info inf;
    int st = ctx_solve_device(c, phi, X, tol, maxit, prec, &inf);
    if (iters) *iters += inf.iters;
    if (solves) *solves += 1;
    if (st) return st;
    launch_hop(c->g, GP_F64_18, c->U64, SP_F64, X, SP_F64, Y, X, c->mass, -1.0, 0, 2, c->stream);
    return cuda_check(c, launch_force(c->g, c->U64, X, Y, c->beta, c->c11, c->c12, 3, nullptr, c->Pmom, kick,
                                      c->stream), "force");
}

int link_update(sfh_ctx* c, double eps, int check)
{
    int st = cuda_check(c, launch_link_update(c->g, c->U64, c->Pmom, eps, check, c->derr, c->stream), "link update");
    c->lowp_valid = false;
    return st;
}

int leapfrog(sfh_ctx* c, const void* phi, void* X, void* Y, double eps, int nsteps, double tol, int maxit,
             int prec, int check, long* iters, int* solves)
{
    int st = force_and_kick(c, phi, X, Y, 0.5 * eps, tol, maxit, prec, iters, solves);
    for (int n = 1; st == SFH_OK && n < nsteps; ++n) {
        st = link_update(c, eps, check);
        if (!st) st = take_device_error(c, "leapfrog");
        if (!st) st = force_and_kick(c, phi, X, Y, eps, tol, maxit, prec, iters, solves);
    }
    if (!st) st = link_update(c, eps, check);
    if (!st) st = take_device_error(c, "leapfrog");
    if (!st) st = force_and_kick(c, phi, X, Y, 0.5 * eps, tol, maxit, prec, iters, solves);
    return st;
}

}  // namespace

namespace sfh {
// scratch of n FP64 link fields (smearing, staples), grown on demand
int ensure_scratch(sfh_ctx* c, int nfields)
{
    size_t need = (size_t)nfields * c->g.V * 4 * 9 * 16;
    if (c->smear && c->smear_bytes >= need) return SFH_OK;
    if (c->smear) cudaFree(c->smear);
    c->smear = nullptr;
    c->smear_bytes = 0;
    int st = cuda_check(c, cudaMalloc(&c->smear, need), "scratch fields");
    if (!st) c->smear_bytes = need;
    return st;
}
}  // namespace sfh

namespace {

// uniform in [0,1) from a 64-bit seed (SplitMix64 finaliser, Steele et al. 2014)
double uniform_from_seed(unsigned long long s)
{
    unsigned long long z = s + 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

}  // namespace

extern "C" int sfh_staples(sfh_ctx* c, double* A1, double* A2)
{
    if (!c || !A1 || !A2) return SFH_ERR_INVALID;
    cudaSetDevice(c->device);
    int st = ensure_scratch(c, 1);
    if (!st) st = cuda_check(c, launch_staples(c->g, c->U64, c->Fbuf, c->smear, c->stream), "staples");
    if (!st) st = links_out(c, c->Fbuf, A1);
    if (!st) st = links_out(c, c->smear, A2);
    return st;
}

extern "C" int sfh_gauge_force(sfh_ctx* c, double* F)
{
    if (!c || !F) return SFH_ERR_INVALID;
    cudaSetDevice(c->device);
    int st = cuda_check(c, launch_force(c->g, c->U64, nullptr, nullptr, c->beta, c->c11, c->c12, 1, c->Fbuf,
                                        nullptr, 0.0, c->stream), "gauge force");
    if (st) return st;
    return links_out(c, c->Fbuf, F);
}

extern "C" int sfh_fermion_force(sfh_ctx* c, const double* X, const double* Y, double* F)
{
    if (!c || !X || !Y || !F) return SFH_ERR_INVALID;
    cudaSetDevice(c->device);
    int st = spinor_in(c, X, c->spin[1]);
    if (!st) st = spinor_in(c, Y, c->spin[2]);
    if (!st) st = cuda_check(c, launch_force(c->g, c->U64, c->spin[1], c->spin[2], c->beta, c->c11, c->c12, 2,
                                             c->Fbuf, nullptr, 0.0, c->stream), "fermion force");
    if (st) return st;
    return links_out(c, c->Fbuf, F);
}

extern "C" int sfh_full_force(sfh_ctx* c, const double* X, const double* Y, double* F)
{
    if (!c || !X || !Y || !F) return SFH_ERR_INVALID;
    cudaSetDevice(c->device);
    int st = spinor_in(c, X, c->spin[1]);
    if (!st) st = spinor_in(c, Y, c->spin[2]);
    if (!st) st = cuda_check(c, launch_force(c->g, c->U64, c->spin[1], c->spin[2], c->beta, c->c11, c->c12, 3,
                                             c->Fbuf, nullptr, 0.0, c->stream), "full force");
    if (st) return st;
    return links_out(c, c->Fbuf, F);
}

extern "C" int sfh_momentum_kick(sfh_ctx* c, int forces, const double* phi, double dt, double tol, int maxit,
                                 int precision, double* X_out, long* cg_iters)
{
    if (!c || forces < SFH_FORCE_GAUGE || forces > (SFH_FORCE_GAUGE | SFH_FORCE_FERMION)) return SFH_ERR_INVALID;
    const bool ferm = (forces & SFH_FORCE_FERMION) != 0;
    if (ferm && (!phi || !(tol > 0.0) || maxit <= 0)) return SFH_ERR_INVALID;
    if (!valid_precision(precision)) return SFH_ERR_INVALID;
    cudaSetDevice(c->device);
    if (cg_iters) *cg_iters = 0;
    void *X = c->spin[4], *Y = c->spin[2];
    int st = SFH_OK;
    if (ferm && (c->fsmear_n > 0 || c->hasen_mass > 0.0)) {  // smeared links / Hasenbusch: general path
        st = spinor_in(c, phi, c->spin[5]);
        long its = 0;
        if (!st) st = smeared_fermion_force(c, c->spin[5], X, Y, tol, maxit, precision, &its, nullptr);
        if (cg_iters) *cg_iters = its;
        if (!st) st = cuda_check(c, launch_link_axpy(c->g, c->Pmom, -dt, c->Fbuf, c->stream), "momentum kick");
        if (!st && (forces & SFH_FORCE_GAUGE))
            st = cuda_check(c, launch_force(c->g, c->U64, nullptr, nullptr, c->beta, c->c11, c->c12, 1, nullptr,
                                            c->Pmom, dt, c->stream), "momentum kick");
        if (st) return st;
        if (X_out) return spinor_out(c, X, X_out);
        return cuda_check(c, cudaStreamSynchronize(c->stream), "momentum kick");
    }
    if (ferm) {
        sfh_cg_info inf;
        std::memset(&inf, 0, sizeof(inf));
        st = spinor_in(c, phi, c->spin[5]);
        if (!st) st = ctx_solve_device(c, c->spin[5], X, tol, maxit, precision, &inf);
        if (cg_iters) *cg_iters = inf.iters;
        if (st) return st;
        launch_hop(c->g, GP_F64_18, c->U64, SP_F64, X, SP_F64, Y, X, c->mass, -1.0, 0, 2, c->stream);  // Y = D^dag X
    }
    st = cuda_check(c, launch_force(c->g, c->U64, ferm ? X : nullptr, ferm ? Y : nullptr, c->beta, c->c11, c->c12,
                                    forces, nullptr, c->Pmom, dt, c->stream), "momentum kick");
    if (st) return st;
    if (ferm && X_out) return spinor_out(c, X, X_out);
    return cuda_check(c, cudaStreamSynchronize(c->stream), "momentum kick");
}

extern "C" int sfh_heatbath(sfh_ctx* c, int nsweeps, unsigned long long seed, int sweep0, double* plaq,
                            double* action_density)
{
    if (!c || nsweeps < 0 || sweep0 < 0) return SFH_ERR_INVALID;
    for (int k = 0; k < 4; ++k)
        if (c->g.L[k] % 4) return set_error(c, SFH_ERR_INVALID, "heatbath: every extent must be a multiple of 4");
    cudaSetDevice(c->device);
    int st = cuda_check(c, launch_heatbath(c->g, c->U64, c->beta, c->c11, c->c12, seed, sweep0, nsweeps, c->stream),
                        "heatbath");
    c->lowp_valid = false;
    double p = 0.0, a = 0.0;
    if (!st && plaq) st = reduce(c, RED_PLAQ, c->U64, nullptr, &p);
    if (!st && action_density) st = reduce(c, RED_ACTION, c->U64, nullptr, &a);
    if (st) return st;
    const double V = (double)c->g.V;
    if (plaq) *plaq = p / (4.0 * V) / 6.0;  // conventional normalisation: 1 on a cold field
    if (action_density) *action_density = a / V;
    return cuda_check(c, cudaStreamSynchronize(c->stream), "heatbath");
}

extern "C" int sfh_set_hasenbusch(sfh_ctx* c, double heavy_mass, const double* phi_heavy)
{
    if (!c || !(heavy_mass >= 0.0)) return SFH_ERR_INVALID;
    cudaSetDevice(c->device);
    c->hasen_mass = heavy_mass;
    if (heavy_mass == 0.0) return SFH_OK;
    int st = ensure_hasen(c);
    if (!st && phi_heavy) st = spinor_in(c, phi_heavy, c->hphi);
    else if (!st) st = cuda_check(c, cudaMemsetAsync(c->hphi, 0, spinor_bytes(c), c->stream), "heavy pseudofermion");
    if (!st) st = cuda_check(c, cudaStreamSynchronize(c->stream), "heavy pseudofermion");
    return st;
}

extern "C" int sfh_set_fermion_smearing(sfh_ctx* c, double rho, int nlevels)
{
    if (!c || nlevels < 0 || nlevels > kMaxSmearLevels || !(rho >= 0.0)) return SFH_ERR_INVALID;
    c->fsmear_rho = rho;
    c->fsmear_n = nlevels;
    return SFH_OK;
}

extern "C" int sfh_smeared_fermion_force(sfh_ctx* c, const double* phi, double tol, int maxit, int precision,
                                         double* F, double* X_out)
{
    if (!c || !phi || !F || !(tol > 0.0) || maxit <= 0 || c->fsmear_n < 1) return SFH_ERR_INVALID;
    if (!valid_precision(precision)) return SFH_ERR_INVALID;
    cudaSetDevice(c->device);
    void *X = c->spin[4], *Y = c->spin[2];
    int st = spinor_in(c, phi, c->spin[5]);
    if (!st) st = smeared_fermion_force(c, c->spin[5], X, Y, tol, maxit, precision, nullptr, nullptr);
    if (!st) st = links_out(c, c->Fbuf, F);
    if (!st && X_out) st = spinor_out(c, X, X_out);
    return st;
}

extern "C" int sfh_link_update(sfh_ctx* c, double eps, int check)
{
    if (!c) return SFH_ERR_INVALID;
    cudaSetDevice(c->device);
    int st = link_update(c, eps, check);
    if (st) return st;
    return take_device_error(c, "link update");
}

extern "C" int sfh_trp2(sfh_ctx* c, double* out)
{
    if (!c || !out) return SFH_ERR_INVALID;
    cudaSetDevice(c->device);
    return reduce(c, RED_TRP2, c->Pmom, nullptr, out);
}

extern "C" int sfh_gauge_action(sfh_ctx* c, double* out)
{
    if (!c || !out) return SFH_ERR_INVALID;
    cudaSetDevice(c->device);
    return reduce(c, RED_ACTION, c->U64, nullptr, out);
}

extern "C" int sfh_plaquette(sfh_ctx* c, double* out)
{
    if (!c || !out) return SFH_ERR_INVALID;
    cudaSetDevice(c->device);
    double s = 0.0;
    int st = reduce(c, RED_PLAQ, c->U64, nullptr, &s);
    if (st) return st;
    *out = s / (4.0 * (double)c->g.V);  // Lattice.cpp:803
    return SFH_OK;
}

extern "C" int sfh_set_beta(sfh_ctx* c, double beta)
{
    if (!c) return SFH_ERR_INVALID;
    c->beta = beta;
    return SFH_OK;
}

extern "C" int sfh_leapfrog(sfh_ctx* c, const double* phi, double eps, int nsteps, double tol, int maxit,
                            int precision, double* X_out, long* cg_iters)
{
    if (!c || !phi || nsteps < 1 || !(tol > 0.0) || maxit <= 0) return SFH_ERR_INVALID;
    if (!valid_precision(precision)) return SFH_ERR_INVALID;
    cudaSetDevice(c->device);
    int st = spinor_in(c, phi, c->spin[5]);
    if (st) return st;
    long its = 0;
    st = leapfrog(c, c->spin[5], c->spin[4], c->spin[2], eps, nsteps, tol, maxit, precision, 0, &its, nullptr);
    if (cg_iters) *cg_iters = its;
    if (st) return st;
    if (X_out) return spinor_out(c, c->spin[4], X_out);
    return cuda_check(c, cudaStreamSynchronize(c->stream), "leapfrog");
}

extern "C" int sfh_hmc_trajectory(sfh_ctx* c, double eps, int nsteps, unsigned long long seed, double tol,
                                  int maxit, int precision, sfh_traj_info* info)
{
    if (!c || !info || nsteps < 1 || !(tol > 0.0) || maxit <= 0) return SFH_ERR_INVALID;
    if (!valid_precision(precision)) return SFH_ERR_INVALID;
    cudaSetDevice(c->device);
    std::memset(info, 0, sizeof(*info));
    auto t0 = std::chrono::steady_clock::now();
    int st = SFH_OK;
    if (!c->Utrial) st = cuda_check(c, cudaMalloc(&c->Utrial, (size_t)c->g.V * 4 * 9 * 16), "trajectory buffer");
    if (st) return st;
    void *chi = c->spin[0], *phi = c->spin[5], *X = c->spin[4], *Y = c->spin[2];
    double Sg0 = 0, T0 = 0, F0 = 0;
    st = reduce(c, RED_ACTION, c->U64, nullptr, &Sg0);  // Fermions.cpp:813
    // phi = D chi, chi complex Gaussian with variance 1/2 per real part
    // (Fermions.cpp:207-212, 302-314)
    if (!st) st = cuda_check(c, launch_random_spinor(c->g, 1.0 / std::sqrt(2.0), seed, chi, c->stream), "chi");
    const bool smeared = c->fsmear_n > 0;  // the fermion operator on stout links
    const bool hasen = c->hasen_mass > 0.0;
    if (!st && hasen) st = ensure_hasen(c);
    if (!st && smeared) st = smear_in(c);
    if (!st && !hasen) {
        launch_hop(c->g, GP_F64_18, c->U64, SP_F64, chi, SP_F64, phi, chi, c->mass, 1.0, 0, 2, c->stream);
    } else if (!st) {
        // heavy: phi_h = D(m_h) chi_h; ratio: phi = D(m) D(m_h)^-1 chi = D(m) D(m_h)^dag M(m_h)^-1 chi
        const double m = c->mass, mh = c->hasen_mass;
        st = cuda_check(c, launch_random_spinor(c->g, 1.0 / std::sqrt(2.0), seed + 3, c->hX, c->stream), "chi_h");
        if (!st) launch_hop(c->g, GP_F64_18, c->U64, SP_F64, c->hX, SP_F64, c->hphi, c->hX, mh, 1.0, 0, 2, c->stream);
        sfh_cg_info inf;
        std::memset(&inf, 0, sizeof(inf));
        c->mass = mh;
        if (!st) st = ctx_solve_device(c, chi, X, tol, maxit, precision, &inf);
        c->mass = m;
        info->cg_iters += inf.iters;
        info->solves += 1;
        if (!st) {
            launch_hop(c->g, GP_F64_18, c->U64, SP_F64, X, SP_F64, Y, X, mh, -1.0, 0, 2, c->stream);
            launch_hop(c->g, GP_F64_18, c->U64, SP_F64, Y, SP_F64, phi, Y, m, 1.0, 0, 2, c->stream);
        }
    }
    if (smeared) {
        int st2 = smear_out(c);
        if (!st) st = st2;
    }
    if (!st) st = cuda_check(c, launch_random_momenta(c->g, seed + 1, c->Pmom, c->stream), "momenta");
    if (!st) st = reduce(c, RED_TRP2, c->Pmom, nullptr, &T0);
    if (!st) st = fermion_action(c, phi, X, tol, maxit, precision, &F0, &info->cg_iters, &info->solves);
    if (!st) st = cuda_check(c, cudaMemcpyAsync(c->Utrial, c->U64, (size_t)c->g.V * 4 * 9 * 16,
                                                cudaMemcpyDeviceToDevice, c->stream), "gauge backup");
    if (!st) st = leapfrog(c, phi, X, Y, eps, nsteps, tol, maxit, precision, 1, &info->cg_iters, &info->solves);
    double T1 = 0, Sg1 = 0, F1 = 0;
    if (!st) st = reduce(c, RED_TRP2, c->Pmom, nullptr, &T1);
    if (!st) st = reduce(c, RED_ACTION, c->U64, nullptr, &Sg1);
    if (!st && !hasen) st = reduce(c, RED_DOT, phi, X, &F1);  // X of the last force evaluation
    if (!st && hasen) st = fermion_action(c, phi, X, tol, maxit, precision, &F1, &info->cg_iters, &info->solves);
    if (st) {  // leave the field as it was before the trajectory
        cudaMemcpyAsync(c->U64, c->Utrial, (size_t)c->g.V * 4 * 9 * 16, cudaMemcpyDeviceToDevice, c->stream);
        cudaStreamSynchronize(c->stream);
        c->lowp_valid = false;
        info->status = st;
        return st;
    }
    info->H_initial[0] = T0;
    info->H_initial[1] = Sg0;
    info->H_initial[2] = F0;
    info->H_final[0] = T1;
    info->H_final[1] = Sg1;
    info->H_final[2] = F1;
    // Fermions.cpp:794-809: accept if u < exp(H_initial - H_final)
    double d = (T0 - T1) + (Sg0 - Sg1) + (F0 - F1);
    info->dH = -d;
    info->uniform = uniform_from_seed(seed + 2);
    info->accepted = info->uniform < std::exp(d) ? 1 : 0;
    if (!info->accepted) {
        st = cuda_check(c, cudaMemcpyAsync(c->U64, c->Utrial, (size_t)c->g.V * 4 * 9 * 16, cudaMemcpyDeviceToDevice,
                                           c->stream), "gauge restore");
        c->lowp_valid = false;
    }
    double s = 0.0;
    if (!st) st = reduce(c, RED_PLAQ, c->U64, nullptr, &s);
    info->plaquette = s / (4.0 * (double)c->g.V);
    info->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    info->status = st;
    return st;
}

extern "C" int sfh_smear_stout(sfh_ctx* c, double rho, int nlevels)
{
    if (!c || nlevels < 0) return SFH_ERR_INVALID;
    cudaSetDevice(c->device);
    int st = ensure_scratch(c, 1);
    if (!st) st = cuda_check(c, launch_stout(c->g, c->U64, c->smear, rho, nlevels, c->derr, c->stream), "stout");
    c->lowp_valid = false;
    if (st) return st;
    return take_device_error(c, "stout smearing");
}

// Device time of one launch of an HMC kernel on the context's fields (CUDA
// events on the context's stream, nrep timed launches after two untimed
// ones).  Inputs are whatever the context holds; the kick forms use a zero
// step, the link update runs on a scratch copy of the links, so the
// context's gauge field and momenta are unchanged.
extern "C" int sfh_kernel_timing(sfh_ctx* c, int kernel, int nrep, double* ms)
{
    if (!c || !ms || nrep < 1 || kernel < 0 || kernel > SFH_KERNEL_PLAQUETTE) return SFH_ERR_INVALID;
    cudaSetDevice(c->device);
    int st = ensure_scratch(c, 5);
    if (st) return st;
    void* s0 = scratch_field(c, 0);
    void* s1 = scratch_field(c, 1);
    void* lev[2] = {s0, s1};
    void* lev_u[2] = {c->U64, s1};  // one stout level of the context's links into scratch
    if (kernel == SFH_KERNEL_LINK_UPDATE || kernel == SFH_KERNEL_STOUT_FORCE)
        st = cuda_check(c, cudaMemcpyAsync(s0, c->U64, link_bytes(c), cudaMemcpyDeviceToDevice, c->stream), "timing");
    if (!st && kernel == SFH_KERNEL_STOUT_FORCE)
        st = cuda_check(c, launch_stout_levels(c->g, lev, 0.125, 1, c->derr, c->stream), "timing");
    if (st) return st;
    auto launch = [&]() -> cudaError_t {
        switch (kernel) {
        case SFH_KERNEL_GAUGE_FORCE:
            return launch_force(c->g, c->U64, nullptr, nullptr, c->beta, c->c11, c->c12, 1, nullptr, c->Pmom, 0.0,
                                c->stream);
        case SFH_KERNEL_FERMION_FORCE:
            return launch_force(c->g, c->U64, c->spin[0], c->spin[1], c->beta, c->c11, c->c12, 2, nullptr, c->Pmom,
                                0.0, c->stream);
        case SFH_KERNEL_STAPLES:
            return launch_staples(c->g, c->U64, c->Fbuf, s1, c->stream);
        case SFH_KERNEL_LINK_UPDATE:
            return launch_link_update(c->g, s0, c->Pmom, 1e-3, 0, c->derr, c->stream);
        case SFH_KERNEL_STOUT_LEVEL:
            return launch_stout_levels(c->g, lev_u, 0.125, 1, c->derr, c->stream);
        case SFH_KERNEL_STOUT_FORCE:
            return launch_stout_force(c->g, lev, 1, 0.125, c->Fbuf, scratch_field(c, 2), scratch_field(c, 3),
                                      scratch_field(c, 4), c->derr, c->stream);
        case SFH_KERNEL_ACTION:
            return launch_reduce(c->g, RED_ACTION, c->U64, nullptr, c->beta, c->c11, c->c12, c->red, c->red + 2048,
                                 c->stream);
        default:
            return launch_reduce(c->g, RED_PLAQ, c->U64, nullptr, c->beta, c->c11, c->c12, c->red, c->red + 2048,
                                 c->stream);
        }
    };
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaError_t e = cudaSuccess;
    for (int k = 0; k < 2 && e == cudaSuccess; ++k) e = launch();
    if (e == cudaSuccess) e = cudaEventRecord(e0, c->stream);
    for (int k = 0; k < nrep && e == cudaSuccess; ++k) e = launch();
    if (e == cudaSuccess) e = cudaEventRecord(e1, c->stream);
    if (e == cudaSuccess) e = cudaEventSynchronize(e1);
    float t = 0.f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&t, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    st = cuda_check(c, e, "kernel timing");
    if (st) return st;
    *ms = (double)t / nrep;
    return take_device_error(c, "kernel timing");
}

extern "C" int sfh_hex_staples(sfh_ctx* c, int level, const double* in, double* out)
{
    if (!c || !in || !out || level < 1 || level > 3) return SFH_ERR_INVALID;
    cudaSetDevice(c->device);
    const size_t V = (size_t)c->g.V;
    const size_t nin = (level == 1 ? 4 : (level == 2 ? 64 : 16)) * V * 18 * sizeof(double);
    const size_t nout = (level == 1 ? 64 : (level == 2 ? 16 : 4)) * V * 18 * sizeof(double);
    void *din = nullptr, *dout = nullptr;
    cudaError_t e = cudaMalloc(&din, nin);
    if (e == cudaSuccess) e = cudaMalloc(&dout, nout);
    if (e == cudaSuccess) e = cudaMemcpyAsync(din, in, nin, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = launch_hex_gamma(c->g, level, din, dout, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, dout, nout, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (din) cudaFree(din);
    if (dout) cudaFree(dout);
    return cuda_check(c, e, "hex staples");
}

extern "C" int sfh_smear_hex(sfh_ctx* c, double alpha1, double alpha2, double alpha3, int npasses)
{
    if (!c || npasses < 0) return SFH_ERR_INVALID;
    cudaSetDevice(c->device);
    int st = ensure_scratch(c, 6);
    if (!st)
        st = cuda_check(c, launch_hex(c->g, c->U64, c->smear, alpha1, alpha2, alpha3, npasses, c->derr, c->stream),
                        "hex");
    c->lowp_valid = false;
    if (st) return st;
    return take_device_error(c, "HEX smearing");
}
