/*
 * sfh.h — C ABI of the B200 staggered-fermion HMC hot path.
 *
 * Plain C: opaque handles, host pointers in the reference's layouts, int
 * status codes, no exceptions cross this boundary.  Every entry point names
 * the reference function (alexanderchasteen/Staggered_Fermions_HMC,
 * file:line) it replaces.
 *
 * Host layouts (identical to the reference):
 *   gauge links, momenta, forces: double[V][4][3][3][2]   (Lattice.cpp:135-168)
 *   spinors (pseudofermion, X, Y): double[V][3][2]         (Fermions.cpp:99-116)
 *   site index s = ((x*Ly + y)*Lz + z)*Lt + t              (Fermions.cpp:42)
 * All four dimensions must be even (even-odd decomposition).
 *
 * Threading: one CUDA stream per context (or batch); calls on one handle are
 * not re-entrant.  Separate handles may be used from separate threads.
 */
#ifndef SFH_H
#define SFH_H

#ifdef __cplusplus
extern "C" {
#endif

/* status codes (the reference throws std::runtime_error / invalid_argument) */
#define SFH_OK 0
#define SFH_ERR_NOCONV 1        /* CG not converged (Fermions.cpp:609-614)          */
#define SFH_ERR_BREAKDOWN 2     /* CG p.Ap or alpha/beta non-finite (:574-600)       */
#define SFH_ERR_DOMAIN 3        /* exp(iQ) input outside its domain (:848-857)       */
#define SFH_ERR_NOT_HERMITIAN 4 /* momentum not Hermitian/traceless (:714-716)       */
#define SFH_ERR_TIMEOUT 5       /* a bounded device wait gave up                     */
#define SFH_ERR_CUDA 6          /* CUDA runtime error (message in sfh_last_error)    */
#define SFH_ERR_INVALID 7       /* invalid argument                                  */
#define SFH_ERR_NOMEM 8         /* device allocation failed                          */
#define SFH_ERR_IO 9            /* checkpoint file could not be read or written      */

/* solver precisions */
#define SFH_PREC_F64 0   /* plain FP64 CG, FP64 links and vectors                     */
#define SFH_PREC_F32 1   /* FP32 12-real links, FP32 vectors, FP64 reliable updates   */
#define SFH_PREC_F16 2   /* FP16 12-real links, FP16+per-site-scale vectors; hop
                            products in packed FP16 (half2), each neighbour's product
                            accumulated in FP32; FP64 reliable updates                */
#define SFH_PREC_F32_18 3 /* FP32 18-real links (no reconstruction), FP32 vectors,
                             FP64 reliable updates                                     */
#define SFH_PREC_BF16 4  /* BF16 12-real links, BF16+per-site-scale vectors, FP32 math,
                            FP64 reliable updates                                      */

typedef struct sfh_ctx sfh_ctx;
typedef struct sfh_batch sfh_batch;

typedef struct {
    int dims[4];   /* Lx, Ly, Lz, Lt (Parameters.h:9-10 Spatial_Size, temporal_size) */
    double mass;   /* staggered mass (Parameters.h:18 fermion_mass)                   */
    double beta;   /* gauge coupling                                                 */
    double c11;    /* Symanzik plaquette coefficient (Parameters.h:51), 0 => 5/3      */
    double c12;    /* Symanzik rectangle coefficient (Parameters.h:52), 0 => -1/12    */
    int device;    /* CUDA device ordinal                                            */
} sfh_params;

typedef struct {
    int status;            /* SFH_OK or an error code                                 */
    int iters;             /* Krylov iterations (operator applications)               */
    int iters_parity[2];   /* per parity system in the even-odd solve                  */
    int reliable_updates;  /* FP64 residual recomputations                             */
    double rsq_rel;        /* final |r|^2 / |b|^2 of the solver's own residual          */
    double true_resid;     /* |b - D D^dag x| / |b| recomputed in FP64                  */
} sfh_cg_info;

/* ---- library / context --------------------------------------------------- */
int sfh_version(void);
const char* sfh_status_string(int status);

/* Replaces the compile-time lattice of Parameters.h:9-31 and the static
 * LatticeTables (Fermions.cpp:20-96) with a runtime context. */
int sfh_create(const sfh_params* params, sfh_ctx** ctx);
int sfh_destroy(sfh_ctx* ctx);
const char* sfh_last_error(const sfh_ctx* ctx);
int sfh_set_stream(sfh_ctx* ctx, void* cuda_stream);
void* sfh_get_stream(sfh_ctx* ctx);
int sfh_set_mass(sfh_ctx* ctx, double mass);
int sfh_synchronize(sfh_ctx* ctx);

/* gauge field in, out (Lattice.cpp:135-168 get_SU3_at_link / set_link_SU3) */
int sfh_upload_gauge(sfh_ctx* ctx, const double* links);
int sfh_download_gauge(sfh_ctx* ctx, double* links);

/* Seeded generators (the reference seeds from std::random_device, rng.cpp:7-15,
 * and is not reproducible).  Gauge: U = exp(i eps H) per link, H traceless
 * Hermitian with N(0,1) entries (the distribution of Lattice.cpp:1001-1033;
 * replaces hot_start_array, Lattice.cpp:198).  Spinor: N(0, sigma^2) per real
 * component (generateGaussianComplex, Fermions.cpp:207-212, has sigma = 1/sqrt2).
 * Momenta: P = sum_a 1/2 p_a lambda_a (generate_conjugate_field_configuration,
 * Fermions.cpp:342-360). */
int sfh_random_gauge(sfh_ctx* ctx, double eps, unsigned long long seed);
int sfh_gaussian_spinor(sfh_ctx* ctx, unsigned long long seed, double sigma, double* out);
int sfh_random_momenta(sfh_ctx* ctx, unsigned long long seed);
int sfh_upload_momenta(sfh_ctx* ctx, const double* P);
int sfh_download_momenta(sfh_ctx* ctx, double* P);

/* ---- operators ------------------------------------------------------------ */
/* out = D in (dagger=0) or D^dag in (dagger=1) on the full lattice:
 * apply_dirac_operator_at_site_s / apply_dirac_dagger_at_site_s
 * (Fermions.cpp:218-283); dagger=1 is also solve_Y_field (Fermions.cpp:623-633). */
int sfh_dirac(sfh_ctx* ctx, int dagger, const double* in, double* out);

/* out = D D^dag in: apply_DDdagger (Fermions.cpp:530-547) */
int sfh_ddag(sfh_ctx* ctx, const double* in, double* out);

/* Device time of one even-odd hop (V/2 output sites, the hopping part of
 * Fermions.cpp:218-283) in a storage format: 0 FP64 18-real, 1 FP32 12-real,
 * 2 FP16 12-real with per-site spinor scale, 3 FP32 18-real, 4 BF16 12-real
 * with per-site spinor scale, 5 FP64 12-real; 6 and 7 the storages of 2 and 4
 * with each block's time and z neighbours staged in shared memory by one
 * bulk asynchronous (TMA) copy along the time direction (results identical
 * to 2 and 4; SFH_ERR_INVALID for Lt above 2816).  Benchmark aid; the input
 * is all zeros, so the value of the output is meaningless. */
int sfh_dslash_timing(sfh_ctx* ctx, int storage, int nrep, double* ms_per_hop);
/* out = K in (the hopping term of D = m + K, Fermions.cpp:218-247, both
 * parities, reference AoS layout) computed by the same Dslash kernel in a
 * storage format (0..7 as above): the input rounded to the format's vectors
 * and the links to its links; the result returned in FP64.  The numerical
 * check of the kernels sfh_dslash_timing times. */
int sfh_dslash_storage(sfh_ctx* ctx, int storage, const double* in, double* out);
/* Test hook of the time-staged Dslash (storages 6 and 7), for checking its
 * bounded waits without a GPU fault: each block announces extra_bytes (a
 * multiple of 16, at most 65536) more on its barrier than its bulk copy
 * delivers, so the copy lands but the barrier never completes, every
 * staging wait runs out after its bound (about 0.1 s, twice per block), the
 * blocks read their neighbours from global memory (same result) and the
 * call returns SFH_ERR_TIMEOUT.  0, the default, turns it off.  No
 * counterpart in the reference. */
int sfh_set_staging_fault(sfh_ctx* ctx, int extra_bytes);

/* ---- solver --------------------------------------------------------------- */
/* X = (D D^dag)^{-1} phi to |r| < tol |phi|: solve_CG_DDdagger / solve_X_field
 * (Fermions.cpp:553-621).  SFH_PREC_F64 runs the reference's full-lattice CG
 * (one set of CG scalars over both parities); the mixed precisions solve the
 * two parity blocks as independent systems and stop on the FP64 true
 * residual.  info may be NULL. */
int sfh_cg_solve(sfh_ctx* ctx, const double* phi, double* X, double tol, int maxit,
                 int precision, sfh_cg_info* info);

/* The schedule of the context's mixed-precision solves (sfh_cg_solve, the
 * trajectory's solves), as sfh_batch_set_schedule: RHS-block width, tiles per
 * block, link staging 0..7 (3: the whole solve in one persistent launch).
 * Default 0, 0, 0; the FP64 CG keeps its own (default tiles per block).  No
 * counterpart in the reference. */
int sfh_set_schedule(sfh_ctx* ctx, int width, int tiles_per_block, int stage_links);

/* ---- forces, link update, observables (context's device fields) --------- */
/* Per-link staple sums A1 (plaquette) and A2 (rectangle):
 * compute_staple_sum_at_link / compute_rectangle_staple_sum_at_link
 * (Lattice.cpp:249-499).  A1, A2: link-field layout. */
int sfh_staples(sfh_ctx* ctx, double* A1, double* A2);
/* Symanzik gauge force on every link: compute_gauge_force_at_link
 * (Fermions.cpp:372-384), as compute_gauge_only_force_field (Fermions.cpp:1278). */
int sfh_gauge_force(sfh_ctx* ctx, double* F);
/* Fermion force: compute_fermion_force_at_link (Fermions.cpp:443-515) on every
 * link, as compute_fermion_only_force_field (Fermions.cpp:1114-1134). */
int sfh_fermion_force(sfh_ctx* ctx, const double* X, const double* Y, double* F);
/* Gauge + fermion force: compute_full_force_field (Fermions.cpp:640-659). */
int sfh_full_force(sfh_ctx* ctx, const double* X, const double* Y, double* F);
/* P <- P - dt F on the context's momenta, F the force selected by `forces`
 * (SFH_FORCE_GAUGE: compute_gauge_only_force_field, Fermions.cpp:1278;
 * SFH_FORCE_FERMION: X = (D D^dag)^{-1} phi, Y = D^dag X,
 * compute_fermion_only_force_field, Fermions.cpp:1114-1134; both:
 * compute_full_force_field, Fermions.cpp:640-659).  This is the momentum
 * update of apply_initial_step_to_conjugate_field / the intermediate and
 * final steps (Fermions.cpp:690-695, 730-735, 767-773).  X_out (may be NULL)
 * receives the solve, cg_iters (may be NULL) its iterations. */
#define SFH_FORCE_GAUGE 1
#define SFH_FORCE_FERMION 2
int sfh_momentum_kick(sfh_ctx* ctx, int forces, const double* phi, double dt, double tol, int maxit,
                      int precision, double* X_out, long* cg_iters);
/* nsweeps heatbath sweeps of the context's gauge field at its beta:
 * heatbath_update (Lattice.cpp:722-757) with single_link_heatbath's
 * Cabibbo-Marinari SU(2) subgroups and the sampler of SU3_Sampling.cpp:17-199.
 * The reference sweeps lexicographically with an unseeded generator; here one
 * direction and one of eight colours of mutually independent links per launch,
 * with Philox uniforms from (seed, link, sweep index), sweep indices sweep0..
 * Every extent must be a multiple of 4.  plaq / action_density (may be NULL)
 * receive the average plaquette (1 on a cold field, the normalisation
 * heatbath_update returns) and the Symanzik action per site after the sweeps
 * (the reference accumulates them during its sweep). */
int sfh_heatbath(sfh_ctx* ctx, int nsweeps, unsigned long long seed, int sweep0, double* plaq,
                 double* action_density);

/* Stout-smeared fermion links (no counterpart in the reference, which has no
 * smeared-link HMC): with nlevels > 0 the fermion operator of sfh_leapfrog,
 * sfh_hmc_trajectory and sfh_momentum_kick uses V = stout^nlevels(U) with
 * parameter rho (plaquette staples, as sfh_smear_stout); the gauge action
 * stays on U, and the fermion force reaches U by the chain rule through the
 * levels (Morningstar & Peardon, Phys. Rev. D 69 (2004) 054501).
 * nlevels = 0 (the default) restores thin links.  At most 16 levels. */
int sfh_set_fermion_smearing(sfh_ctx* ctx, double rho, int nlevels);
/* Hasenbusch mass splitting (no counterpart in the reference): with
 * heavy_mass > 0 the fermion action of sfh_leapfrog, sfh_hmc_trajectory and
 * sfh_momentum_kick is phi_h^dag M(m_h)^{-1} phi_h + phi^dag M(m_h) M(m)^{-1} phi,
 * M(m) = D(m) D(m)^dag, m the context's mass (both terms on the smeared links
 * when sfh_set_fermion_smearing is on).  phi is the caller's pseudofermion (or
 * the trajectory's own); phi_heavy (may be NULL: zero, or what the last
 * trajectory drew) is the heavy one.  heavy_mass = 0 restores one
 * pseudofermion. */
int sfh_set_hasenbusch(sfh_ctx* ctx, double heavy_mass, const double* phi_heavy);
/* The fermion force on the thin links under that smearing: X = (D D^dag)^{-1}
 * phi and Y = D^dag X with V, compute_fermion_force_at_link (Fermions.cpp:443-515)
 * on V, then the chain rule.  F: link-field layout; X_out may be NULL. */
int sfh_smeared_fermion_force(sfh_ctx* ctx, const double* phi, double tol, int maxit, int precision,
                              double* F, double* X_out);
/* U <- exp(i eps P) U with the context's momenta (Fermions.cpp:699-723 with
 * check = 1, which rejects a non-Hermitian P as the reference does;
 * Fermions.cpp:984-994 with check = 0). */
int sfh_link_update(sfh_ctx* ctx, double eps, int check);
/* Device time (ms per launch, CUDA events on the context's stream) of one HMC
 * kernel on the context's current fields, a measurement aid with no
 * counterpart in the reference: the gauge force with the momentum kick
 * (compute_gauge_force_at_link, Fermions.cpp:372-384), the fermion force
 * (Fermions.cpp:443-515) of the context's spinor work fields, the plaquette
 * and rectangle staple sums (Lattice.cpp:249-499), the link update
 * U <- exp(i eps P) U (Fermions.cpp:699-723) on a scratch copy, one stout level
 * (rho 0.125), one level of the stout chain-rule force, the Symanzik action
 * (Lattice.cpp:759-781) and the plaquette (Lattice.cpp:784-804).  Kicks use a
 * zero step: the context's links and momenta are left as they were. */
#define SFH_KERNEL_GAUGE_FORCE 0
#define SFH_KERNEL_FERMION_FORCE 1
#define SFH_KERNEL_STAPLES 2
#define SFH_KERNEL_LINK_UPDATE 3
#define SFH_KERNEL_STOUT_LEVEL 4
#define SFH_KERNEL_STOUT_FORCE 5
#define SFH_KERNEL_ACTION 6
#define SFH_KERNEL_PLAQUETTE 7
int sfh_kernel_timing(sfh_ctx* ctx, int kernel, int nrep, double* ms);
/* sum over links of Re Tr P^2: compute_Tr_P2 (Fermions.cpp:662-678) */
int sfh_trp2(sfh_ctx* ctx, double* out);
/* Symanzik gauge action: compute_action (Lattice.cpp:759-781) */
int sfh_gauge_action(sfh_ctx* ctx, double* out);
/* average plaquette in the reference's normalisation (6.0 on a cold field):
 * compute_avg_plaq (Lattice.cpp:784-804) */
int sfh_plaquette(sfh_ctx* ctx, double* out);
int sfh_set_beta(sfh_ctx* ctx, double beta);

/* ---- molecular dynamics ---------------------------------------------------- */
typedef struct {
    int status;
    int accepted;          /* Metropolis outcome                                   */
    int solves;            /* CG solves in the trajectory                          */
    int pad;
    long cg_iters;         /* summed CG iterations                                 */
    double dH;             /* H_final - H_initial                                  */
    double H_initial[3];   /* Tr P^2, S_gauge, phi.X                               */
    double H_final[3];
    double uniform;        /* the Metropolis uniform                               */
    double plaquette;      /* after the accept / reject                            */
    double seconds;
} sfh_traj_info;

/* One leapfrog trajectory on the context's gauge field and momenta with
 * explicit step size and count: local_initial_half_step, local_leapfrog_steps,
 * local_final_step (Fermions.cpp:967-1028).  X_out (may be NULL) receives the
 * last solve; cg_iters (may be NULL) the summed CG iterations. */
int sfh_leapfrog(sfh_ctx* ctx, const double* phi, double eps, int nsteps, double tol, int maxit,
                 int precision, double* X_out, long* cg_iters);
/* A full HMC update: single_sweep_monte_carlo_update_WITH_FERMIONS
 * (Fermions.cpp:812-828) with seeded phi = D chi, momenta and Metropolis
 * uniform (Monte_carlo_step, Fermions.cpp:778-810). */
int sfh_hmc_trajectory(sfh_ctx* ctx, double eps, int nsteps, unsigned long long seed, double tol, int maxit,
                       int precision, sfh_traj_info* info);

/* ---- observables and checkpoints ------------------------------------------ */
/* Polyakov loops Tr prod_t U_t(x,y,z,t) on the spatial grid, (re, im) pairs in
 * (x*Ly + y)*Lz + z order: precompute_polyakov_grid (Lattice.cpp:869-882). */
int sfh_polyakov_grid(sfh_ctx* ctx, double* out);
/* <P(m) conj(P(m+d))> over |d|^2 = r2: correlator_over_fixed_distance_fast
 * (Lattice.cpp:886-948).  out2 = (re, im). */
int sfh_polyakov_correlator(sfh_ctx* ctx, int r2, double* out2);
/* The same correlator from a given Polyakov grid (as precompute_polyakov_grid
 * returns it), so callers holding a grid need no gauge field:
 * correlator_over_fixed_distance_fast(P_grid, r2) (Lattice.cpp:886-948).
 * The spatial sizes are the context's. */
int sfh_polyakov_correlator_grid(sfh_ctx* ctx, const double* grid, int r2, double* out2);
/* Raw gauge checkpoint in the reference layout (save_all_lattice_configs /
 * load_all_lattice_configs for one coupling, Lattice.cpp:810-847). */
int sfh_save_gauge(sfh_ctx* ctx, const char* path);
int sfh_load_gauge(sfh_ctx* ctx, const char* path);

/* ---- smearing ------------------------------------------------------------- */
/* nlevels stout levels U <- exp(rho proj(C U^dag)) U with plaquette staples
 * (the single-level analogue of the HEX steps of Smearing.cpp:132-155). */
int sfh_smear_stout(sfh_ctx* ctx, double rho, int nlevels);
/* The staple steps of HEX on their own, on host fields in the reference's
 * flat tensor layouts (combo * V + s, 18 doubles per matrix):
 *   level 1: apply_step_1 (Smearing.cpp:76-123): in = gauge links (link-field
 *            layout), out = Gamma1 [64][V], combo (4 mu + nu) 4 + rho;
 *   level 2: apply_step_3 (Smearing.cpp:157-211): in = V1 [64][V], out =
 *            Gamma2 [16][V], combo 4 mu + nu;
 *   level 3: apply_step_5 (Smearing.cpp:236-275): in = V2 [16][V], out =
 *            Gamma3 [4][V] (summed from zero).
 * The fused smearing below keeps only the decorated links the next level
 * uses; this is its checking path against the reference's own steps. */
int sfh_hex_staples(sfh_ctx* ctx, int level, const double* in, double* out);
/* npasses HEX passes: Apply_HEX_smearing (Smearing.cpp:304-311); npasses = 4
 * is Apply_4HEX_smearing (Smearing.cpp:313-318).  Alphas as Smearing.h:7-9. */
int sfh_smear_hex(sfh_ctx* ctx, double alpha1, double alpha2, double alpha3, int npasses);

/* ---- batched solver (many lattices, masses and right-hand sides) --------- */
typedef struct {
    int dims[4];
    double mass;
    int nrhs;
} sfh_system_desc;

#define SFH_BATCH_FULL_LATTICE 1  /* one CG per RHS over both parities, as the
                                     reference's solve_CG_DDdagger               */

/* No reference counterpart: the reference solves one system at a time
 * (Fermions.cpp:553).  All systems of a batch advance together: every CG
 * iteration of every lane is the same three grid-wide kernels (t = K p;
 * v = m^2 p - K t with the CG sums; the x, r, p update), replayed as CUDA
 * graphs of 16 iterations, with the lanes' scalars advanced on the device. */
int sfh_batch_create(int device, int nsys, const sfh_system_desc* systems, int precision,
                     int flags, sfh_batch** batch);
int sfh_batch_destroy(sfh_batch* batch);
const char* sfh_batch_last_error(const sfh_batch* batch);
int sfh_batch_set_stream(sfh_batch* batch, void* cuda_stream);
void* sfh_batch_get_stream(sfh_batch* batch);
/* RHS-block width for the fused hop (0 = automatic); the autotuner sets it */
int sfh_batch_set_rhs_block(sfh_batch* batch, int width);
/* RHS-block widths of the two hop kernels separately (0 = automatic; 1, 2,
 * 4, 8): the first hop (t = K p) can serve wider groups than the second,
 * whose CG sums take registers.  sfh_batch_set_rhs_block and
 * sfh_batch_set_schedule set both to one width.  No counterpart in the
 * reference. */
int sfh_batch_set_hop_widths(sfh_batch* batch, int hop1_width, int hop2_width);
int sfh_batch_get_hop_widths(sfh_batch* batch, int* hop1_width, int* hop2_width);
/* Autotuner: time probe_iters capped iterations for every RHS-block width
 * (1, 2, 4, 8; FP64: 1, 2), tiles-per-block count (1, 2, 4) and link staging
 * (0 to 7 as below; FP64: 0; 6 for FP16 only), and for the lane-list stages
 * (4 to 7) also hop widths 4 and 2, on the batch's current inputs and keep
 * the fastest.
 * The schedule never changes the results.  No counterpart in the reference
 * (its solver has no schedule). */
int sfh_batch_autotune(sfh_batch* batch, int probe_iters, int* best_width);
/* The schedule directly: RHS-block width (0 = automatic), 256-site tiles per
 * block of the iteration kernels (0 = 2, or 1 where two would give the first
 * hop fewer than four work items per SM), and the hop kernels' link staging:
 * 0 links read directly per RHS group; 1 staged in shared memory per work
 * item with asynchronous copies; 2 system-blocked: one block per tile serves
 * every RHS of its system in groups of the RHS-block width, the tile's links
 * read once into shared memory (FP16 unpacked), the tiles per block fixed at
 * 1, and the FP64 reliable-update hops in two kernels of their own; 3
 * persistent: the same per-tile work in one cooperative launch for the whole
 * solve, its phases separated by a grid barrier whose waits are bounded (a
 * wait that gives up fails the solve with SFH_ERR_TIMEOUT); the solutions
 * equal those of 2 bit for bit.  2 and 3 serve FP16, BF16 and FP32 12-real
 * storage (FP32 18-real takes 1).  4 and 5: 0 and 1 with the FP64
 * reliable-update hops taken out of the hop kernels into two kernels that
 * walk a device list of the lanes due for one (as 2 and 3 always do).
 * 6 (FP16; the other precisions run 4): 4 with each tile's time and z
 * neighbour vectors staged in shared memory, one bulk asynchronous (TMA)
 * copy per RHS of the tile's range [i0 - Lt/2, i0 + 256 + Lt/2) of the other
 * parity, double-buffered across the work item's tiles (RHS groups of at
 * most 4; a staging wait that gives up fails the solve with SFH_ERR_TIMEOUT,
 * the thread reading that tile from global memory).  7: 4 with the two hop
 * kernels on grids of as many blocks as fit on the GPU at once, each block
 * taking work items in turn from a device counter (no partial last wave;
 * FP64 runs 0).  Staging applies to the reduced precisions only.  And its
 * current values. */
int sfh_batch_set_schedule(sfh_batch* batch, int width, int tiles_per_block, int stage_links);
/* Bound on each grid-barrier wait of the persistent schedule (3), in polls
 * of about 128 ns (0 = the default, about 4 s): a wait that runs out fails
 * the solve with SFH_ERR_TIMEOUT and leaves the batch usable.  No
 * counterpart in the reference. */
int sfh_batch_set_barrier_polls(sfh_batch* batch, long long polls);
/* Reliable-update threshold of the mixed precisions (default 0.1 for
 * the 16-bit storages, 0.01 for the FP32 ones): an FP64
 * update (x_hi += x_lo, r = b - M x_hi) when the iterated residual has dropped
 * by this factor below its largest value since the last update.  No
 * counterpart in the reference (its CG is FP64 only). */
int sfh_batch_set_reliable_delta(sfh_batch* batch, double delta);
int sfh_batch_get_schedule(sfh_batch* batch, int* width, int* tiles_per_block, int* stage_links);
int sfh_batch_set_gauge(sfh_batch* batch, int sys, const double* links);
int sfh_batch_set_rhs(sfh_batch* batch, int sys, int rhs, const double* phi);
/* The mass of one right-hand side (default: its system's), so that the RHS of
 * a system can be solved at several masses on the same links (a Hasenbusch
 * pair, a multi-mass set): they share the system's link loads.  No
 * counterpart in the reference (one mass per program, Parameters.h:18). */
int sfh_batch_set_rhs_mass(sfh_batch* batch, int sys, int rhs, double mass);
int sfh_batch_solve(sfh_batch* batch, double tol, int maxit);
int sfh_batch_get_solution(sfh_batch* batch, int sys, int rhs, double* X);
int sfh_batch_get_info(sfh_batch* batch, int sys, int rhs, sfh_cg_info* info);
/* seeded device generators and read-back for the batch's inputs */
int sfh_batch_random_gauge(sfh_batch* batch, int sys, double eps, unsigned long long seed);
int sfh_batch_random_rhs(sfh_batch* batch, int sys, int rhs, unsigned long long seed, double sigma);
int sfh_batch_get_gauge(sfh_batch* batch, int sys, double* links);
int sfh_batch_get_rhs(sfh_batch* batch, int sys, int rhs, double* phi);
/* number of kernels the last sfh_batch_solve launched (init + graph chunks) */
int sfh_batch_kernel_launches(sfh_batch* batch, long* n);
/* sfh_batch_solve with the iteration kernels launched one by one between CUDA
 * events on the batch's stream (no graph replay): ms / n (SFH_TIMED_KERNELS
 * entries) receive the summed device time and launch count of each kernel:
 * t = K p; v = m^2 p - K t with the CG sums; the x, r, p update; with the
 * system-blocked schedule the two FP64 reliable-update kernels (zero
 * otherwise: the hop kernels do those hops); and with the persistent schedule
 * the one cooperative launch (the others zero).  Same kernels, same results;
 * a measurement aid with no counterpart in the reference. */
#define SFH_TIMED_KERNELS 6
int sfh_batch_solve_timed(sfh_batch* batch, double tol, int maxit, double* ms, long* n);
/* FP64 |b - D D^dag x| / |b| for one solution (diagnostic) */
int sfh_batch_true_residual(sfh_batch* batch, int sys, int rhs, double* rel);

/* ---- allocation-free solve ------------------------------------------------ */
/* No counterpart in the reference.  An FP64 CG solve of D D^dag X = phi (the
 * reference's full-lattice algorithm, as sfh_cg_solve with SFH_PREC_F64; there
 * is no mixed-precision variant) that allocates no device or host memory, for
 * callers that cannot call cudaMalloc: host runtimes that own all device
 * memory through their own pool and forbid allocations outside it, and
 * trajectory loops that must not allocate after start-up.  The solver's work
 * vectors live in a fixed array inside the library (about 12.6 MB, reserved
 * on every GPU that loads the library until the process exits), so the
 * lattice may have at most SFH_NOALLOC_MAX_SITES sites; larger lattices return
 * SFH_ERR_INVALID.
 *
 * All pointers are device pointers in the library's even-odd layout (site
 * index i = s >> 1 within parity p = (x+y+z+t) & 1, s as above):
 *   links_eo: double2 [p][mu][row*3+col][i]   (4*V*9 double2 = 72*V doubles)
 *   phi_eo, x_eo: double2 [p][color][i]       (6*V doubles)
 * The call runs on cuda_stream (0 = legacy default stream) of the current
 * device, copies the solver's status back to the host and waits for the
 * stream before returning; info may be NULL.  info->true_resid is -1 (not
 * computed: no array is spare for the extra operator application);
 * info->rsq_rel is the recurrence's |r|^2 / |b|^2.  The first call on a device
 * looks up the array's device address, which can load the library's device
 * code on that device: make that first call before any stream capture.  Every
 * call uses the same array, so calls whose work overlaps on the GPU (other
 * threads, other streams) race and must be serialised by the caller. */
#define SFH_NOALLOC_MAX_SITES 65536
int sfh_cg_solve_noalloc(const int dims[4], double mass, const void* links_eo, const void* phi_eo,
                         void* x_eo, double tol, int maxit, void* cuda_stream, sfh_cg_info* info);

#ifdef __cplusplus
}
#endif
#endif
