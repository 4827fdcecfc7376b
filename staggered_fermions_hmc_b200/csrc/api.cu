// api.cu — C ABI: context lifetime, field transfer, operators, solver entry.
//
// Host buffers use the reference's AoS layouts; conversion to the device
// even-odd SoA layout happens on the device right after the copy.
#include <cstring>
#include <string>

#include "sfh_internal.h"

namespace sfh {

int set_error(sfh_ctx* c, int code, const std::string& msg)
{
    if (c) c->last_error = msg;
    return code;
}

int cuda_check(sfh_ctx* c, cudaError_t e, const char* what)
{
    if (e == cudaSuccess) return SFH_OK;
    return set_error(c, e == cudaErrorMemoryAllocation ? SFH_ERR_NOMEM : SFH_ERR_CUDA,
                     std::string(what) + ": " + cudaGetErrorString(e));
}

bool dims_ok(const int dims[4])
{
    long V = 1;
    for (int k = 0; k < 4; ++k) {
        if (dims[k] < 2 || (dims[k] & 1)) return false;
        V *= dims[k];
    }
    return V <= (1L << 28);
}

Geom make_geom(const int dims[4])
{
    Geom g;
    for (int k = 0; k < 4; ++k) g.L[k] = dims[k];
    g.V = dims[0] * dims[1] * dims[2] * dims[3];
    g.Vh = g.V / 2;
    g.dLt = FastDiv((uint32_t)dims[3]);
    g.dLz = FastDiv((uint32_t)dims[2]);
    g.dLy = FastDiv((uint32_t)dims[1]);
    return g;
}

}  // namespace sfh

using namespace sfh;

extern "C" int sfh_version(void) { return 1; }

extern "C" const char* sfh_status_string(int s)
{
    switch (s) {
        case SFH_OK: return "ok";
        case SFH_ERR_NOCONV: return "CG did not converge";
        case SFH_ERR_BREAKDOWN: return "CG breakdown (non-finite or zero p.Ap, alpha or beta)";
        case SFH_ERR_DOMAIN: return "exp(iQ) argument outside its domain";
        case SFH_ERR_NOT_HERMITIAN: return "momentum field is not Hermitian and traceless";
        case SFH_ERR_TIMEOUT: return "bounded device wait timed out";
        case SFH_ERR_CUDA: return "CUDA error";
        case SFH_ERR_INVALID: return "invalid argument";
        case SFH_ERR_NOMEM: return "device allocation failed";
        case SFH_ERR_IO: return "checkpoint file could not be read or written";
        default: return "unknown status";
    }
}

extern "C" int sfh_create(const sfh_params* p, sfh_ctx** out)
{
    if (!p || !out) return SFH_ERR_INVALID;
    *out = nullptr;
    if (!dims_ok(p->dims)) return SFH_ERR_INVALID;
    sfh_ctx* c = new sfh_ctx();
    c->g = make_geom(p->dims);
    c->mass = p->mass;
    c->beta = p->beta;
    c->c11 = p->c11 != 0.0 ? p->c11 : 5.0 / 3.0;
    c->c12 = p->c12 != 0.0 ? p->c12 : -1.0 / 12.0;
    c->device = p->device;
    cudaError_t e = cudaSetDevice(c->device);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, c->device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete c;
        return SFH_ERR_CUDA;
    }
    c->own_stream = true;
    const size_t V = (size_t)c->g.V;
    const size_t links64 = V * 4 * 9 * 16;
    e = cudaMalloc(&c->U64, links64);
    if (e == cudaSuccess) e = cudaMalloc(&c->U32, V * 4 * 3 * 16);
    if (e == cudaSuccess) e = cudaMalloc(&c->U16, V * 4 * 3 * 8);
    if (e == cudaSuccess) e = cudaMalloc(&c->Ubf16, V * 4 * 3 * 8);
    if (e == cudaSuccess) e = cudaMalloc(&c->U32_18, V * 4 * 9 * 8);
    if (e == cudaSuccess) e = cudaMalloc(&c->Pmom, links64);
    if (e == cudaSuccess) e = cudaMalloc(&c->Fbuf, links64);
    if (e == cudaSuccess) e = cudaMalloc(&c->stage, V * 72 * sizeof(double));
    for (int k = 0; k < 6 && e == cudaSuccess; ++k) e = cudaMalloc(&c->spin[k], V * 6 * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc((void**)&c->red, 4096 * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc((void**)&c->derr, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(c->derr, 0, sizeof(int));
    if (e != cudaSuccess) {
        sfh_destroy(c);
        return SFH_ERR_NOMEM;
    }
    // cold start until a field is uploaded
    e = cudaMemset(c->U64, 0, links64);
    *out = c;
    return SFH_OK;
}

extern "C" int sfh_destroy(sfh_ctx* c)
{
    if (!c) return SFH_OK;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    for (int k = 0; k < kNumPrecisions; ++k) {
        if (c->ws[k]) workspace_free(c->ws[k]);
        if (c->ws_pair[k]) workspace_free(c->ws_pair[k]);
    }
    void* ptrs[] = {c->U64, c->U32, c->U16, c->Ubf16, c->U32_18, c->U64_12, c->Pmom, c->Fbuf, c->stage, c->red, c->derr, c->Utrial,
                    c->smear, c->hphi, c->hX};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    for (void* p : c->spin)
        if (p) cudaFree(p);
    if (c->pinned) cudaFreeHost(c->pinned);
    if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return SFH_OK;
}

extern "C" const char* sfh_last_error(const sfh_ctx* c) { return c ? c->last_error.c_str() : "null context"; }

extern "C" int sfh_set_stream(sfh_ctx* c, void* s)
{
    if (!c) return SFH_ERR_INVALID;
    cudaSetDevice(c->device);
    if (c->own_stream && c->stream) {
        cudaStreamSynchronize(c->stream);
        cudaStreamDestroy(c->stream);
    }
    c->stream = (cudaStream_t)s;
    c->own_stream = false;
    return SFH_OK;
}

extern "C" void* sfh_get_stream(sfh_ctx* c) { return c ? (void*)c->stream : nullptr; }

extern "C" int sfh_set_mass(sfh_ctx* c, double m)
{
    if (!c) return SFH_ERR_INVALID;
    c->mass = m;
    return SFH_OK;
}

extern "C" int sfh_synchronize(sfh_ctx* c)
{
    if (!c) return SFH_ERR_INVALID;
    return cuda_check(c, cudaStreamSynchronize(c->stream), "synchronize");
}

extern "C" int sfh_upload_gauge(sfh_ctx* c, const double* links)
{
    if (!c || !links) return SFH_ERR_INVALID;
    cudaSetDevice(c->device);
    size_t n = (size_t)c->g.V * 72 * sizeof(double);
    int st = cuda_check(c, cudaMemcpyAsync(c->stage, links, n, cudaMemcpyHostToDevice, c->stream), "gauge upload");
    if (st) return st;
    launch_links_aos_to_eo(c->g, (const double*)c->stage, c->U64, c->stream);
    c->lowp_valid = false;
    return cuda_check(c, cudaStreamSynchronize(c->stream), "gauge upload");
}

extern "C" int sfh_download_gauge(sfh_ctx* c, double* links)
{
    if (!c || !links) return SFH_ERR_INVALID;
    cudaSetDevice(c->device);
    size_t n = (size_t)c->g.V * 72 * sizeof(double);
    launch_links_eo_to_aos(c->g, c->U64, (double*)c->stage, c->stream);
    int st = cuda_check(c, cudaMemcpyAsync(links, c->stage, n, cudaMemcpyDeviceToHost, c->stream), "gauge download");
    if (st) return st;
    return cuda_check(c, cudaStreamSynchronize(c->stream), "gauge download");
}

static int spinor_in(sfh_ctx* c, const double* host, void* eo)
{
    size_t n = (size_t)c->g.V * 6 * sizeof(double);
    int st = cuda_check(c, cudaMemcpyAsync(c->stage, host, n, cudaMemcpyHostToDevice, c->stream), "spinor upload");
    if (st) return st;
    launch_spinor_aos_to_eo(c->g, (const double*)c->stage, eo, c->stream);
    return SFH_OK;
}

static int spinor_out(sfh_ctx* c, const void* eo, double* host)
{
    size_t n = (size_t)c->g.V * 6 * sizeof(double);
    launch_spinor_eo_to_aos(c->g, eo, (double*)c->stage, c->stream);
    int st = cuda_check(c, cudaMemcpyAsync(host, c->stage, n, cudaMemcpyDeviceToHost, c->stream), "spinor download");
    if (st) return st;
    return cuda_check(c, cudaStreamSynchronize(c->stream), "spinor download");
}

extern "C" int sfh_dirac(sfh_ctx* c, int dagger, const double* in, double* out)
{
    if (!c || !in || !out) return SFH_ERR_INVALID;
    cudaSetDevice(c->device);
    int st = spinor_in(c, in, c->spin[0]);
    if (st) return st;
    launch_hop(c->g, GP_F64_18, c->U64, SP_F64, c->spin[0], SP_F64, c->spin[1], c->spin[0], c->mass,
               dagger ? -1.0 : 1.0, 0, 2, c->stream);
    st = cuda_check(c, cudaGetLastError(), "dirac");
    if (st) return st;
    return spinor_out(c, c->spin[1], out);
}

extern "C" int sfh_ddag(sfh_ctx* c, const double* in, double* out)
{
    if (!c || !in || !out) return SFH_ERR_INVALID;
    cudaSetDevice(c->device);
    int st = spinor_in(c, in, c->spin[0]);
    if (st) return st;
    // temp = D^dag in; out = D temp  (Fermions.cpp:530-547)
    launch_hop(c->g, GP_F64_18, c->U64, SP_F64, c->spin[0], SP_F64, c->spin[1], c->spin[0], c->mass, -1.0,
               0, 2, c->stream);
    launch_hop(c->g, GP_F64_18, c->U64, SP_F64, c->spin[1], SP_F64, c->spin[2], c->spin[1], c->mass, 1.0,
               0, 2, c->stream);
    st = cuda_check(c, cudaGetLastError(), "ddag");
    if (st) return st;
    return spinor_out(c, c->spin[2], out);
}

extern "C" int sfh_cg_solve(sfh_ctx* c, const double* phi, double* X, double tol, int maxit,
                            int precision, sfh_cg_info* info)
{
    if (!c || !phi || !X || !(tol > 0.0) || maxit <= 0) return SFH_ERR_INVALID;
    if (!valid_precision(precision)) return SFH_ERR_INVALID;
    cudaSetDevice(c->device);
    return ctx_cg_solve(c, phi, X, tol, maxit, precision, info);
}

// Device error flags raised by kernels (never a trap): read and clear.
static int take_device_error(sfh_ctx* c, const char* what)
{
    int h = 0;
    int st = cuda_check(c, cudaMemcpyAsync(&h, c->derr, sizeof(int), cudaMemcpyDeviceToHost, c->stream), what);
    if (!st) st = cuda_check(c, cudaMemsetAsync(c->derr, 0, sizeof(int), c->stream), what);
    if (!st) st = cuda_check(c, cudaStreamSynchronize(c->stream), what);
    if (st) return st;
    if (h & DEV_ERR_DOMAIN) return set_error(c, SFH_ERR_DOMAIN, std::string(what) + ": exp(iQ) domain error");
    if (h & DEV_ERR_NOT_HERMITIAN)
        return set_error(c, SFH_ERR_NOT_HERMITIAN, std::string(what) + ": P_pre is not Hermitian or not traceless");
    if (h & DEV_ERR_TIMEOUT) return set_error(c, SFH_ERR_TIMEOUT, std::string(what) + ": device wait timed out");
    return SFH_OK;
}

extern "C" int sfh_random_gauge(sfh_ctx* c, double eps, unsigned long long seed)
{
    if (!c) return SFH_ERR_INVALID;
    cudaSetDevice(c->device);
    int st = cuda_check(c, launch_random_gauge(c->g, eps, seed, c->U64, c->derr, c->stream), "random gauge");
    if (st) return st;
    c->lowp_valid = false;
    return take_device_error(c, "random gauge");
}

extern "C" int sfh_gaussian_spinor(sfh_ctx* c, unsigned long long seed, double sigma, double* out)
{
    if (!c || !out) return SFH_ERR_INVALID;
    cudaSetDevice(c->device);
    int st = cuda_check(c, launch_random_spinor(c->g, sigma, seed, c->spin[0], c->stream), "gaussian spinor");
    if (st) return st;
    return spinor_out(c, c->spin[0], out);
}

extern "C" int sfh_random_momenta(sfh_ctx* c, unsigned long long seed)
{
    if (!c) return SFH_ERR_INVALID;
    cudaSetDevice(c->device);
    int st = cuda_check(c, launch_random_momenta(c->g, seed, c->Pmom, c->stream), "random momenta");
    if (st) return st;
    return cuda_check(c, cudaStreamSynchronize(c->stream), "random momenta");
}

extern "C" int sfh_upload_momenta(sfh_ctx* c, const double* P)
{
    if (!c || !P) return SFH_ERR_INVALID;
    cudaSetDevice(c->device);
    size_t n = (size_t)c->g.V * 72 * sizeof(double);
    int st = cuda_check(c, cudaMemcpyAsync(c->stage, P, n, cudaMemcpyHostToDevice, c->stream), "momenta upload");
    if (st) return st;
    launch_links_aos_to_eo(c->g, (const double*)c->stage, c->Pmom, c->stream);
    return cuda_check(c, cudaStreamSynchronize(c->stream), "momenta upload");
}

extern "C" int sfh_download_momenta(sfh_ctx* c, double* P)
{
    if (!c || !P) return SFH_ERR_INVALID;
    cudaSetDevice(c->device);
    size_t n = (size_t)c->g.V * 72 * sizeof(double);
    launch_links_eo_to_aos(c->g, c->Pmom, (double*)c->stage, c->stream);
    int st = cuda_check(c, cudaMemcpyAsync(P, c->stage, n, cudaMemcpyDeviceToHost, c->stream), "momenta download");
    if (st) return st;
    return cuda_check(c, cudaStreamSynchronize(c->stream), "momenta download");
}

// The links, gauge format and vector format of a standalone-Dslash storage:
// 0 FP64 18-real, 1 FP32 12-real, 2 FP16 12-real + scale, 3 FP32 18-real,
// 4 BF16 12-real + scale, 5 FP64 12-real (derived from U64 on each call,
// in a buffer allocated on first use).
// storages 6 and 7: the links and vectors of 2 (FP16) and 4 (BF16), the
// Dslash with its time and z neighbours staged in shared memory
static bool storage_tstaged(int storage) { return storage == 6 || storage == 7; }

static int storage_links(sfh_ctx* c, int storage, const void** U, int* gp, int* sp)
{
    static const int gps[6] = {GP_F64_18, GP_F32_12, GP_F16_12, GP_F32_18, GP_BF16_12, GP_F64_12};
    static const int sps[6] = {SP_F64, SP_F32, SP_F16, SP_F32, SP_BF16, SP_F64};
    if (storage_tstaged(storage)) {
        if (!hop_tstaged_fits(c->g)) return set_error(c, SFH_ERR_INVALID, "time-staged Dslash: Lt above 2816");
        storage = storage == 6 ? 2 : 4;
    }
    if (storage < 0 || storage > 5) return SFH_ERR_INVALID;
    if (!c->lowp_valid) {
        launch_make_lowp_gauge(c->g, c->U64, c->U32, c->U16, c->stream, c->U32_18, c->Ubf16);
        c->lowp_valid = true;
    }
    if (storage == 5) {
        const size_t Vh = (size_t)c->g.Vh;
        if (!c->U64_12) {
            int st = cuda_check(c, cudaMalloc(&c->U64_12, (size_t)c->g.V * 4 * 6 * 16), "FP64 12-real links");
            if (st) return st;
        }
        for (int pm = 0; pm < 8; ++pm) {  // rows 0 and 1: the first 6 of the 9 elements of each (p, mu)
            int st = cuda_check(c,
                                cudaMemcpyAsync((char*)c->U64_12 + pm * 6 * Vh * 16, (const char*)c->U64 + pm * 9 * Vh * 16,
                                                6 * Vh * 16, cudaMemcpyDeviceToDevice, c->stream),
                                "FP64 12-real links");
            if (st) return st;
        }
    }
    const void* const Us[6] = {c->U64, c->U32, c->U16, c->U32_18, c->Ubf16, c->U64_12};
    *U = Us[storage];
    *gp = gps[storage];
    *sp = sps[storage];
    return SFH_OK;
}

// one standalone Dslash, out = K in over parities [q0, q0 + nq), in a
// storage format (0..7)
static void storage_hop(sfh_ctx* c, int storage, const void* U, int gp, int sp, const void* in, void* out, int q0,
                        int nq)
{
    if (storage_tstaged(storage))
        launch_hop_tstaged(c->g, gp, U, in, out, nullptr, 0.0, 1.0, q0, nq, c->derr, c->stage_extra_tx, c->stream);
    else
        launch_hop(c->g, gp, U, sp, in, sp, out, nullptr, 0.0, 1.0, q0, nq, c->stream);
}

// out = K in (the hopping term of D = m + K, Fermions.cpp:218-247, both
// parities) computed by the standalone Dslash kernel in a storage format
// (0..7 as storage_links): the input rounded to the format's vectors, the
// links to its links, the result returned in FP64.  The check of the
// kernels that sfh_dslash_timing times.
extern "C" int sfh_dslash_storage(sfh_ctx* c, int storage, const double* in, double* out)
{
    if (!c || !in || !out) return SFH_ERR_INVALID;
    cudaSetDevice(c->device);
    const void* U = nullptr;
    int gp = 0, sp = 0;
    int st = storage_links(c, storage, &U, &gp, &sp);
    if (st) return st;
    const size_t n = (size_t)c->g.V * 6 * sizeof(double);
    st = cuda_check(c, cudaMemcpyAsync(c->stage, in, n, cudaMemcpyHostToDevice, c->stream), "dslash input");
    if (st) return st;
    launch_spinor_aos_to_eo(c->g, (const double*)c->stage, c->spin[0], c->stream);
    launch_spinor_convert(c->g, sp, true, c->spin[0], c->spin[1], c->stream);
    storage_hop(c, storage, U, gp, sp, c->spin[1], c->spin[2], 0, 2);
    launch_spinor_convert(c->g, sp, false, c->spin[2], c->spin[3], c->stream);
    launch_spinor_eo_to_aos(c->g, c->spin[3], (double*)c->stage, c->stream);
    st = cuda_check(c, cudaMemcpyAsync(out, c->stage, n, cudaMemcpyDeviceToHost, c->stream), "dslash output");
    if (st) return st;
    st = cuda_check(c, cudaStreamSynchronize(c->stream), "dslash storage");
    if (st) return st;
    return take_device_error(c, "dslash storage");
}

// Test hook of the time-staged Dslash (storages 6, 7): each block announces
// extra_bytes more on its barrier than its bulk copy delivers, so the copy
// lands but the barrier's phase never completes, every staging wait runs out
// after its bound, the blocks read their neighbours from global memory, and
// the call reports SFH_ERR_TIMEOUT.  0 (the default) turns it off.
extern "C" int sfh_set_staging_fault(sfh_ctx* c, int extra_bytes)
{
    if (!c || extra_bytes < 0 || (extra_bytes & 15) || extra_bytes > (1 << 16)) return SFH_ERR_INVALID;
    c->stage_extra_tx = (unsigned)extra_bytes;
    return SFH_OK;
}

// Device time of one even-odd hop (V/2 output sites) in a storage format
// (0..5 as storage_links).  Uses the context's gauge field and a zero input
// (the memory traffic and arithmetic do not depend on the values); nrep
// timed hops after three untimed ones, measured with CUDA events on the
// context's stream.
extern "C" int sfh_dslash_timing(sfh_ctx* c, int storage, int nrep, double* ms_per_hop)
{
    if (!c || !ms_per_hop || nrep < 1) return SFH_ERR_INVALID;
    cudaSetDevice(c->device);
    const void* U = nullptr;
    int gp = 0, sp = 0;
    int st = storage_links(c, storage, &U, &gp, &sp);
    if (st) return st;
    void* in = c->spin[0];
    void* out = c->spin[1];
    cudaMemsetAsync(in, 0, (size_t)c->g.V * 48, c->stream);
    cudaMemsetAsync(out, 0, (size_t)c->g.V * 48, c->stream);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    for (int k = 0; k < 3; ++k) storage_hop(c, storage, U, gp, sp, in, out, 0, 1);
    cudaEventRecord(e0, c->stream);
    for (int k = 0; k < nrep; ++k) storage_hop(c, storage, U, gp, sp, in, out, 0, 1);
    cudaEventRecord(e1, c->stream);
    st = cuda_check(c, cudaEventSynchronize(e1), "dslash timing");
    float ms = 0.f;
    if (!st) st = cuda_check(c, cudaEventElapsedTime(&ms, e0, e1), "dslash timing");
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st) return st;
    *ms_per_hop = (double)ms / nrep;
    return take_device_error(c, "dslash timing");
}
