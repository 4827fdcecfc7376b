/*
 * sfh_oracle.h — CPU oracle for the staggered-fermion HMC hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference
 * algorithms (alexanderchasteen/Staggered_Fermions_HMC) used as the checker
 * for the CUDA path.  Only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg may load it.  The product library never calls it.
 *
 * Parity pin: the restatement is checked against fixtures produced by the
 * reference's own sources (tests/golden/, generated by
 * tests/golden/make_golden.py from binaries that oracle/build_ref.py builds
 * from the unmodified reference files) and
 * against the reference's analytic known-answer tests (cold-start staples
 * 6I / 18I, cold action, cold plaquette, unitarity).
 *
 * Conventions (all identical to the reference):
 *   dims[4] = {Lx, Ly, Lz, Lt}; site s = ((x*Ly + y)*Lz + z)*Lt + t.
 *   Gauge / momentum / force field: [site][mu(4)][row(3)][col(3)][re,im]
 *   = 72 doubles per site.  Spinor: [site][color(3)][re,im] = 6 doubles.
 *   Spatial directions periodic; time direction anti-periodic for fermions.
 */
#ifndef SFH_ORACLE_H
#define SFH_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

enum {
    ORC_OK = 0,
    ORC_ERR_NOCONV = 1,     /* CG did not reach tol in maxit iterations   */
    ORC_ERR_BREAKDOWN = 2,  /* CG p.Ap non-finite/zero or alpha/beta NaN  */
    ORC_ERR_DOMAIN = 3,     /* exp(iQ) called with Q outside its domain   */
    ORC_ERR_NOT_HERMITIAN = 4
};

/* Neighbour tables, Fermions.cpp:20-96 (LatticeTables).  Each array 4*V. */
void orc_tables(const int dims[4], int* up, int* dn, int* bc_up, int* bc_dn,
                int* eta);

/* Full-lattice staggered operator, Fermions.cpp:218-283.
 * sign=+1: out = D psi = (m + K) psi;  sign=-1: out = D^dag psi = (m - K) psi */
void orc_dirac(const int dims[4], double mass, int sign, const double* U,
               const double* in, double* out);

/* out = D D^dag in (via a temporary D^dag in), Fermions.cpp:530-547 */
void orc_ddag(const int dims[4], double mass, const double* U,
              const double* in, double* out);

/* Real part of <a,b> over n doubles, Fermions.cpp:521-528 */
double orc_dot(long n, const double* a, const double* b);

/* Plain CG on D D^dag X = phi, X0 = 0, Fermions.cpp:553-617.
 * iters = number of D D^dag applications.  Returns ORC_* status. */
int orc_cg(const int dims[4], double mass, const double* U, const double* phi,
           double tol, int maxit, double* X, int* iters, double* final_rsq);

/* Per-link staple sums, Lattice.cpp:249-313 (A1) and 315-499 (A2). Each 4V*18 */
void orc_staples(const int dims[4], const double* U, double* A1, double* A2);

/* Gauge force, Fermions.cpp:372-384 with Lattice.cpp:502-507.  F: 4V*18 */
void orc_gauge_force(const int dims[4], double beta, double c11, double c12,
                     const double* U, double* F);

/* Fermion force, Fermions.cpp:443-515.  F: 4V*18 */
void orc_fermion_force(const int dims[4], const double* U, const double* X,
                       const double* Y, double* F);

/* Total force gauge + fermion, Fermions.cpp:640-659 */
void orc_full_force(const int dims[4], double beta, double c11, double c12,
                    const double* U, const double* X, const double* Y,
                    double* F);

/* exp(iQ) for one Hermitian traceless 3x3 (18 doubles), Fermions.cpp:834-902 */
int orc_expiq(const double* Q, double* out);

/* U <- exp(i eps P) U on every link, Fermions.cpp:984-994 */
int orc_link_update(const int dims[4], double eps, const double* P, double* U);

/* Sum over links of Re Tr P^2, Fermions.cpp:662-678 */
double orc_trp2(const int dims[4], const double* P);

/* Symanzik gauge action, Lattice.cpp:759-781 */
double orc_action(const int dims[4], double beta, double c11, double c12,
                  const double* U);

/* Average plaquette (reference normalisation, 6.0 on a cold start),
 * Lattice.cpp:784-804 */
double orc_avg_plaq(const int dims[4], const double* U);

/* One leapfrog trajectory with explicit eps and n_steps, following
 * local_initial_half_step / local_leapfrog_steps / local_final_step,
 * Fermions.cpp:967-1028.  P and U are updated in place; X (6V) receives the
 * solution of the last solve.  cg_iters_total (may be NULL) sums CG iters. */
int orc_leapfrog(const int dims[4], double mass, double beta, double c11,
                 double c12, double eps, int n_steps, double tol, int maxit,
                 const double* phi, double* P, double* U, double* X,
                 long* cg_iters_total);

/* Polyakov loop grid P(x,y,z) = Tr prod_t U_t (un-normalised),
 * Lattice.cpp:849-882.  out: Lx*Ly*Lz complex as (re,im) pairs. */
void orc_polyakov_grid(const int dims[4], const double* U, double* out);

/* Polyakov correlator at squared distance r2, Lattice.cpp:886-948 (cubic
 * spatial volume).  Writes (re,im) into out2. */
void orc_polyakov_corr(const int dims[4], const double* grid, int r2,
                       double* out2);

/* One stout level: U' = exp(proj(rho * C U^dag)) U with C the plaquette
 * staple sum running from x to x+mu.  The map is the single-level analogue of
 * the reference's HEX steps (Smearing.cpp:132-155); applied n_levels times. */
int orc_stout(const int dims[4], double rho, int n_levels, double* U);

/* One HEX smearing pass, Smearing.cpp:76-311, with the documented fixes:
 * exp(A) evaluated as exp(i * (-iA)), Gamma_3 zero-initialised.
 * alphas = {alpha1, alpha2, alpha3} as in Smearing.h:7-9. */
int orc_hex(const int dims[4], const double alphas[3], double* U);

/* The staple steps of HEX on their own, in the reference's flat tensor
 * layouts (combo * V + site, 18 doubles per matrix): G1 = apply_step_1(U)
 * [64][V] (Smearing.cpp:76-123), G2 = apply_step_3(V1) [16][V] from V1
 * [64][V] (Smearing.cpp:157-211), G3 = apply_step_5(V2) [4][V] from V2 [16][V]
 * (Smearing.cpp:236-275, Gamma_3 starting at zero). */
void orc_hex_gamma1(const int dims[4], const double* U, double* G1);
void orc_hex_gamma2(const int dims[4], const double* V1, double* G2);
void orc_hex_gamma3(const int dims[4], const double* V2, double* G3);

/* nsweeps heatbath sweeps (single_link_heatbath, Lattice.cpp:722-757, in
 * colour order; seeded Philox uniforms), sweep indices sweep0.. */
int orc_heatbath(const int dims[4], double beta, double c11, double c12, unsigned long long seed, int sweep0,
                 int nsweeps, double* U);

/* Thin-link force of an action on n_levels stout-smeared links (rho), given
 * the force F_top on the smeared links (same convention as
 * orc_fermion_force).  No counterpart in the reference. */
int orc_stout_force(const int dims[4], double rho, int n_levels, const double* U_thin, const double* F_top,
                    double* F_thin);

/* U[i] = exp(i eps H[i]) for n matrices (used to build seeded gauge fields). */
int orc_exp_field(long n, double eps, const double* H, double* U);

/* Seeded generators: the library's Philox-4x32-10 + Box-Muller fields on the
 * CPU, keyed like the device generators (counter (id, id >> 32, pair, stream),
 * key = seed).  Gauge: U = exp(i eps H) per link, H traceless Hermitian with
 * N(0,1) entries (Lattice.cpp:1001-1033); spinor: N(0, sigma^2) per real;
 * momenta: 1/2 sum_a p_a lambda_a (Fermions.cpp:342-360).  AoS layouts. */
void orc_philox4x32_10(const unsigned ctr[4], const unsigned key[2], unsigned out[4]);
void orc_gen_normals(unsigned long long seed, unsigned stream, unsigned long long id, int n, double* z);
int orc_gen_gauge(const int dims[4], double eps, unsigned long long seed, double* U);
void orc_gen_spinor(const int dims[4], double sigma, unsigned long long seed, double* out);
void orc_gen_momenta(const int dims[4], unsigned long long seed, double* P);

#ifdef __cplusplus
}
#endif
#endif
