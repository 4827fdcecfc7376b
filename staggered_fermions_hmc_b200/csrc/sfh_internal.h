// sfh_internal.h — host-side context shared by the library's translation
// units.  Not part of the public C ABI (include/sfh.h).
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "../../include/sfh.h"
#include "sfh_core.cuh"

namespace sfh {
struct CgWorkspace;
constexpr int kNumPrecisions = SFH_PREC_BF16 + 1;  // the solver precisions of include/sfh.h
}

struct sfh_ctx {
    sfh::Geom g;
    double mass = 0.0, beta = 0.0, c11 = 5.0 / 3.0, c12 = -1.0 / 12.0;
    int device = 0;
    int num_sms = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;

    // device fields (even-odd SoA, see sfh_core.cuh)
    void* U64 = nullptr;       // gauge FP64 18-real
    void* U32 = nullptr;       // gauge FP32 12-real (derived)
    void* U16 = nullptr;       // gauge FP16 12-real (derived)
    void* Ubf16 = nullptr;     // gauge BF16 12-real (derived)
    void* U64_12 = nullptr;    // gauge FP64 12-real (derived on use by the standalone Dslash)
    void* U32_18 = nullptr;    // gauge FP32 18-real (derived)
    bool lowp_valid = false;   // derived copies match U64
    void* Pmom = nullptr;      // momenta FP64 18-real
    void* Fbuf = nullptr;      // force scratch FP64 18-real
    void* stage = nullptr;     // device staging for host AoS transfers (72V doubles)
    void* spin[6] = {};        // FP64 spinor work fields (6V doubles each)
    double* red = nullptr;     // reduction partials / scalars
    int* derr = nullptr;       // device error flags (DeviceErr bits)
    void* pinned = nullptr;    // pinned host staging (72V doubles)
    size_t pinned_bytes = 0;

    sfh::CgWorkspace* ws[sfh::kNumPrecisions] = {};  // cached solver workspaces per precision
    double ws_mass[sfh::kNumPrecisions] = {};
    int sched_nb = 0, sched_tpi = 0, sched_stage = 0;  // schedule of the context's mixed-precision solves
    unsigned stage_extra_tx = 0;  // test hook of the time-staged Dslash (sfh_set_staging_fault)
    sfh::CgWorkspace* ws_pair[sfh::kNumPrecisions] = {};  // two systems on the links (Hasenbusch pair)
    double ws_pair_mass[sfh::kNumPrecisions][2] = {};
    void* Utrial = nullptr;        // gauge backup for the Metropolis step
    void* smear = nullptr;         // scratch link fields (smearing, staples)
    size_t smear_bytes = 0;
    double fsmear_rho = 0.0;       // stout smearing of the fermion links (HMC)
    int fsmear_n = 0;              // levels; 0 = thin links
    double hasen_mass = 0.0;       // Hasenbusch heavy mass (0 = one pseudofermion)
    void* hphi = nullptr;          // heavy pseudofermion and its solution (FP64 spinors)
    void* hX = nullptr;

    std::string last_error;
};

namespace sfh {

// error helpers
int set_error(sfh_ctx* c, int code, const std::string& msg);
int cuda_check(sfh_ctx* c, cudaError_t e, const char* what);

// launch helpers implemented in layout.cu / dslash.cu
void launch_spinor_aos_to_eo(const Geom& g, const double* aos, void* eo, cudaStream_t s);
void launch_spinor_eo_to_aos(const Geom& g, const void* eo, double* aos, cudaStream_t s);
// even-odd FP64 vectors to storage format sp (to_fmt) or back, both parities
void launch_spinor_convert(const Geom& g, int sp, bool to_fmt, const void* src, void* dst, cudaStream_t s);
void launch_links_aos_to_eo(const Geom& g, const double* aos, void* eo, cudaStream_t s);
void launch_links_eo_to_aos(const Geom& g, const void* eo, double* aos, cudaStream_t s);
void launch_make_lowp_gauge(const Geom& g, const void* U64, void* U32, void* U16, cudaStream_t s,
                            void* U32_18 = nullptr, void* Ubf16 = nullptr);

// the solver precisions of include/sfh.h
inline bool valid_precision(int p) { return p >= SFH_PREC_F64 && p <= SFH_PREC_BF16; }

// out_q = a*self_q + b*K_{q,1-q} in  for q in [q0, q0+nq); precisions by enum
void launch_hop(const Geom& g, int gauge_prec, const void* gauge, int in_prec, const void* in,
                int out_prec, void* out, const void* self, double a, double b, int q0, int nq,
                cudaStream_t s);

// launch_hop for the 16-bit storages (gauge_prec GP_F16_12 or GP_BF16_12,
// vectors of the matching format) with the neighbours staged along the time
// direction; a bounded staging wait that gives up sets DEV_ERR_TIMEOUT in
// *err, and the thread reads its neighbours from global memory instead.
// extra_tx: a test hook, normally 0 (bytes announced beyond each copy's, so
// that every staging wait runs out).
// hop_tstaged_fits: the staged range of a 256-site tile fits the default
// 48 KB of shared memory (Lt <= 2816).
bool hop_tstaged_fits(const Geom& g);
void launch_hop_tstaged(const Geom& g, int gauge_prec, const void* gauge, const void* in, void* out,
                        const void* self, double a, double b, int q0, int nq, int* err, unsigned extra_tx,
                        cudaStream_t s);

cudaError_t launch_random_gauge(const Geom& g, double eps, unsigned long long seed, void* U, int* d_err,
                                cudaStream_t s);
cudaError_t launch_random_spinor(const Geom& g, double sigma, unsigned long long seed, void* out,
                                 cudaStream_t s);
cudaError_t launch_random_momenta(const Geom& g, unsigned long long seed, void* P, cudaStream_t s);

Geom make_geom(const int dims[4]);
bool dims_ok(const int dims[4]);
int ctx_cg_solve(sfh_ctx* c, const double* phi, double* X, double tol, int maxit, int prec,
                 sfh_cg_info* info);
int ctx_solve_device(sfh_ctx* c, const void* b_eo, void* x_eo, double tol, int maxit, int prec,
                     sfh_cg_info* info);
// two solves on the context's links at two masses, as one batch of two systems
int ctx_solve_pair_device(sfh_ctx* c, const void* const b_eo[2], void* const x_eo[2], const double mass[2],
                          double tol, int maxit, int prec, sfh_cg_info info[2]);
void workspace_free(CgWorkspace* w);
int ensure_scratch(sfh_ctx* c, int nfields);

// gauge.cu
cudaError_t launch_force(const Geom& g, const void* U, const void* X, const void* Y, double beta, double c11,
                         double c12, int what, void* out, void* mom, double kick, cudaStream_t s);
cudaError_t launch_staples(const Geom& g, const void* U, void* A1, void* A2, cudaStream_t s);
cudaError_t launch_link_update(const Geom& g, void* U, const void* P, double eps, int check, int* err,
                               cudaStream_t s);
enum { RED_TRP2 = 0, RED_ACTION = 1, RED_PLAQ = 2, RED_DOT = 3 };
// smear.cu
cudaError_t launch_stout(const Geom& g, void* U, void* tmp, double rho, int n, int* err, cudaStream_t s);
cudaError_t launch_stout_levels(const Geom& g, void* const* levels, double rho, int n, int* err, cudaStream_t s);
cudaError_t launch_stout_force(const Geom& g, void* const* levels, int n, double rho, void* F, void* G, void* Gn,
                               void* W, int* err, cudaStream_t s);
cudaError_t launch_link_axpy(const Geom& g, void* Y, double a, const void* X, cudaStream_t s);
cudaError_t launch_heatbath(const Geom& g, void* U, double beta, double c11, double c12, unsigned long long seed,
                            int sweep0, int nsweeps, cudaStream_t s);
cudaError_t launch_hex(const Geom& g, void* U, void* scratch, double a1, double a2, double a3, int n, int* err,
                       cudaStream_t s);
cudaError_t launch_hex_gamma(const Geom& g, int level, const void* in, void* out, cudaStream_t s);
cudaError_t launch_reduce(const Geom& g, int kind, const void* A, const void* B, double beta, double c11,
                          double c12, double* partial, double* out, cudaStream_t s);

}  // namespace sfh
