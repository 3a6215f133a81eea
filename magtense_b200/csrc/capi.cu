// extern "C" entry points of libmagtense_b200.so (declared in include/magtense_b200.h).
//
// A handle replaces the process-wide state of the reference's CUDA shim
// (MagTenseCudaBlas.cu:29-92): it owns the device copy of the demag tensor,
// the per-cell material vectors and the integrator workspace.  The caller owns
// every m / H / output device buffer.
#include <cuda_runtime.h>
#include <math.h>
#include <float.h>
#include <stdint.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <algorithm>
#include <chrono>
#include <thread>
#include <mutex>
#include <string>
#include <vector>
#include <memory>
#include <map>

#include "../../include/magtense_b200.h"
#include "common.cuh"
#include "fields.cuh"
#include "integrate.cuh"
#include "llg.cuh"
#include "batch.cuh"
#include "gemm_tc.cuh"
#include "sparse.cuh"
#include <cudaTypedefs.h>

namespace {

thread_local std::string g_last_error;

int fail(int code, const char* fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

#define CUDA_TRY(expr)                                                                              \
    do {                                                                                            \
        cudaError_t _e = (expr);                                                                    \
        if (_e != cudaSuccess)                                                                      \
            return fail(_e == cudaErrorMemoryAllocation ? MT_ERR_NOMEM : MT_ERR_CUDA, "%s: %s (%s:%d)", \
                        #expr, cudaGetErrorString(_e), __FILE__, __LINE__);                         \
    } while (0)

const double kMu0 = 4.0 * 3.141592653589793 * 1e-7;   // (4*pi)*1e-7 as the reference evaluates it

template <typename T>
cudaError_t dalloc(T** p, size_t count)
{
    *p = nullptr;
    if (count == 0) count = 1;
    return cudaMalloc((void**)p, sizeof(T) * count);
}

}  // namespace

struct mt_handle {
    int nx = 0, ny = 0, nz = 0, n = 0, ldk = 0;
    double L[3] = {0, 0, 0}, d[3] = {0, 0, 0};
    int device = 0, num_sms = 0;
    // material
    double* Jfact = nullptr; double* Kfact = nullptr; float* Mfact = nullptr; double* A6 = nullptr;
    bool have_material = false;
    // dynamics
    int solver = 2; double gamma = 0.0, alpha0 = 0.0; int hext_row = 0; int renorm = 0;
    double* hext = nullptr; int nt_hext = 0; double* alpha_tab = nullptr; int nt_alpha = 0;
    int cap_hext = 0, cap_alpha = 0;   // allocated rows: tables of the same size keep their device address
    bool have_dynamics = false;
    // tensor
    float* K = nullptr; bool have_K = false;
    // thresholded-sparse demag built from K (sparse.cu); nullptr: the dense product
    int* sp_rowptr = nullptr; int* sp_col = nullptr; float* sp_val = nullptr;
    long long sp_nnz = 0; float sp_thr = 0.f;
    // scratch
    float* m32 = nullptr;
    double* vjp_buf = nullptr;   // [lam (3n) | g_Ms (n)]
    double* vjp_z = nullptr;     // Jfact g_he (3n)
    float* vjp_v32 = nullptr;    // Ms g_he, FP32 [3][ldk] (padding stays 0)
    // row shards of one instance (shard_world > 1): this rank's cells and tensor rows only
    int shard_rank = 0, shard_world = 1, shard_cell0 = 0, shard_ncell = 0;
    unsigned char* shard_region = nullptr;          // this rank's exchange region
    void* shard_peer[kMaxShards] = {};              // every rank's region, this rank's included
    bool shard_ipc[kMaxShards] = {};                // mapped here by cudaIpcOpenMemHandle
    bool shard_peers_set = false, shard_broken = false;
    double shard_timeout_s = 10.0;                  // bound on one cross-rank wait (build_link)
    std::chrono::steady_clock::time_point shard_broken_at;   // when a run of this rank gave up
    ShardLink* shard_link = nullptr;                // device copy of the link
    long long shard_xseq = 0, shard_rseq = 0;       // barrier and reduction counts after the last run
    // device buffers of an integration, kept between calls (one integration at a time)
    unsigned char* integ_arena = nullptr;
    size_t integ_arena_bytes = 0;
    bool integ_arena_busy = false;
};

namespace {

void free_ptr(void* p)
{
    if (p) cudaFree(p);
}

void axis_setup(int nn, double L, double* d)
{
    *d = (nn > 1) ? L / nn : L;
}

// Fraction of a dense tensor of `bytes` that the streaming demag loads mark L2 evict_last:
// enough of it to fill 80 % of one die's half of L2, so that the lines kept survive the
// evaluation's sweep over the rest; 0 when that is under 5 % of the tensor.
float l2_keep_fraction(int device, double bytes)
{
    int l2 = 0;
    if (cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, device) != cudaSuccess || l2 <= 0 || bytes <= 0.0) {
        cudaGetLastError();
        return 0.f;
    }
    const double f = std::min(1.0, 0.8 * 0.5 * (double)l2 / bytes);
    return f < 0.05 ? 0.f : (float)f;
}

DevProb make_prob(const mt_handle* h)
{
    DevProb P;
    memset(&P, 0, sizeof(P));
    P.n = h->n; P.nx = h->nx; P.ny = h->ny; P.nz = h->nz; P.ldk = h->ldk;
    P.K = h->K;
    P.krow0 = h->shard_cell0;
    const int nn[3] = {h->nx, h->ny, h->nz};
    for (int a = 0; a < 3; ++a) {
        const double d2 = h->d[a] * h->d[a];
        P.lapc[a] = 1.0 / d2;
        P.diag_b[a] = nn[a] > 1 ? -1.0 / d2 : 0.0;
        P.diag_i[a] = nn[a] > 1 ? -2.0 / d2 : 0.0;
    }
    P.Jfact = h->Jfact; P.Kfact = h->Kfact; P.Mfact = h->Mfact; P.A6 = h->A6;
    P.solver = h->solver; P.hext_row = h->hext_row; P.nt_hext = h->nt_hext; P.nt_alpha = h->nt_alpha;
    P.hext = h->hext; P.alpha_tab = h->alpha_tab;
    P.gamma = h->gamma; P.alpha0 = h->alpha0;
    P.sp_rowptr = h->sp_rowptr; P.sp_col = h->sp_col; P.sp_val = h->sp_val;
    P.l2_keep = l2_keep_fraction(h->device, 24.0 * (double)(h->shard_world > 1 ? h->shard_ncell : h->n) * h->ldk);
    return P;
}

int check_ready(const mt_handle* h, bool need_material, bool need_dynamics)
{
    if (!h) return fail(MT_ERR_ARG, "null handle");
    if (!h->have_K) return fail(MT_ERR_STATE, "no demag tensor: call mt_assemble_demag or mt_load_demag_colmajor first");
    if (need_material && !h->have_material) return fail(MT_ERR_STATE, "no material: call mt_set_material first");
    if (need_dynamics && !h->have_dynamics) return fail(MT_ERR_STATE, "no dynamics: call mt_set_dynamics first");
    return MT_OK;
}

bool sharded(const mt_handle* h) { return h && h->shard_world > 1; }

// a run of this row shard gave up: no further runs, and mt_destroy keeps the region a while
void mark_broken(mt_handle* h)
{
    if (!sharded(h) || h->shard_broken) return;
    h->shard_broken = true;
    h->shard_broken_at = std::chrono::steady_clock::now();
}

int refuse_sharded(const mt_handle* h, const char* what)
{
    if (sharded(h)) return fail(MT_ERR_UNSUPPORTED, "%s: the handle is a row shard (only mt_integrate runs it)", what);
    return MT_OK;
}

// tensor rows the handle holds
int tensor_rows(const mt_handle* h) { return sharded(h) ? h->shard_ncell : h->n; }

int ensure_tensor(mt_handle* h)
{
    if (h->K) return MT_OK;
    const size_t cnt = (size_t)tensor_rows(h) * 6 * (size_t)h->ldk;
    CUDA_TRY(dalloc(&h->K, cnt));
    return MT_OK;
}

int ensure_m32(mt_handle* h)
{
    if (h->m32) return MT_OK;
    CUDA_TRY(dalloc(&h->m32, 3 * (size_t)h->ldk));
    return MT_OK;
}

}  // namespace

extern "C" {

const char* mt_last_error(void) { return g_last_error.c_str(); }
const char* mt_version(void) { return "magtense_b200 0.1 (sm_100a)"; }

int mt_create(const mt_grid* g, mt_handle** out)
{
    if (!g || !out) return fail(MT_ERR_ARG, "null argument");
    *out = nullptr;
    if (g->nx < 1 || g->ny < 1 || g->nz < 1) return fail(MT_ERR_ARG, "grid counts must be >= 1");
    const long long n = (long long)g->nx * g->ny * g->nz;
    if (n > 200000) return fail(MT_ERR_ARG, "n = %lld cells exceeds the dense-tensor limit", n);
    if (!(g->Lx > 0 && g->Ly > 0 && g->Lz > 0)) return fail(MT_ERR_ARG, "grid extents must be > 0");
    mt_handle* h = new mt_handle();
    h->nx = g->nx; h->ny = g->ny; h->nz = g->nz; h->n = (int)n;
    h->ldk = (int)((n + 3) & ~3LL);
    h->L[0] = g->Lx; h->L[1] = g->Ly; h->L[2] = g->Lz;
    axis_setup(g->nx, g->Lx, &h->d[0]);
    axis_setup(g->ny, g->Ly, &h->d[1]);
    axis_setup(g->nz, g->Lz, &h->d[2]);
    cudaError_t e = cudaGetDevice(&h->device);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&h->num_sms, cudaDevAttrMultiProcessorCount, h->device);
    if (e == cudaSuccess) e = integrate_upload_tables();
    if (e != cudaSuccess) {
        delete h;
        return fail(MT_ERR_CUDA, "CUDA init: %s", cudaGetErrorString(e));
    }
    *out = h;
    return MT_OK;
}

int mt_destroy(mt_handle* h)
{
    if (!h) return MT_OK;
    if (h->shard_broken && h->shard_region) {
        // A rank of another process may still store into this region after a run gave up:
        // until its next cross-rank barrier sees the abort word, or, if it waits on this
        // rank, until its own wait runs out and it raises the abort words.  Both end within
        // two timeouts of the failure, so the region is freed no earlier than that.
        bool remote = false;
        for (int p = 0; p < kMaxShards; ++p) remote = remote || h->shard_ipc[p];
        if (remote) {
            const auto until = h->shard_broken_at + std::chrono::milliseconds(
                                   (long long)(1000.0 * (2.0 * h->shard_timeout_s + 1.0)));
            std::this_thread::sleep_until(until);
        }
    }
    free_ptr(h->Jfact); free_ptr(h->Kfact); free_ptr(h->Mfact); free_ptr(h->A6);
    free_ptr(h->hext); free_ptr(h->alpha_tab); free_ptr(h->K); free_ptr(h->m32);
    free_ptr(h->vjp_buf); free_ptr(h->vjp_z); free_ptr(h->vjp_v32);
    free_ptr(h->sp_rowptr); free_ptr(h->sp_col); free_ptr(h->sp_val);
    for (int p = 0; p < kMaxShards; ++p)
        if (h->shard_ipc[p]) cudaIpcCloseMemHandle(h->shard_peer[p]);
    free_ptr(h->shard_region); free_ptr(h->shard_link);
    free_ptr(h->integ_arena);
    delete h;
    return MT_OK;
}

int mt_set_material(mt_handle* h, double A0, const double* Ms, const double* K0, const double* u_ea)
{
    if (!h || !Ms || !K0 || !u_ea) return fail(MT_ERR_ARG, "null argument");
    const int n = h->n;
    std::vector<double> jf(n), kf(n), a6(6 * (size_t)n);
    std::vector<float> mf(n);
    for (int i = 0; i < n; ++i) {
        if (!(Ms[i] != 0.0) || !std::isfinite(Ms[i])) return fail(MT_ERR_ARG, "Ms[%d] must be finite and nonzero", i);
        jf[i] = A0 / (kMu0 * Ms[i]);
        kf[i] = K0[i] / (kMu0 * Ms[i]);
        mf[i] = (float)Ms[i];
        const double ux = u_ea[i * 3 + 0], uy = u_ea[i * 3 + 1], uz = u_ea[i * 3 + 2];
        a6[0 * (size_t)n + i] = ux * ux; a6[1 * (size_t)n + i] = ux * uy; a6[2 * (size_t)n + i] = ux * uz;
        a6[3 * (size_t)n + i] = uy * uy; a6[4 * (size_t)n + i] = uy * uz; a6[5 * (size_t)n + i] = uz * uz;
    }
    if (!h->Jfact) {
        CUDA_TRY(dalloc(&h->Jfact, n)); CUDA_TRY(dalloc(&h->Kfact, n));
        CUDA_TRY(dalloc(&h->Mfact, n)); CUDA_TRY(dalloc(&h->A6, 6 * (size_t)n));
    }
    CUDA_TRY(cudaMemcpy(h->Jfact, jf.data(), sizeof(double) * n, cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(h->Kfact, kf.data(), sizeof(double) * n, cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(h->Mfact, mf.data(), sizeof(float) * n, cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(h->A6, a6.data(), sizeof(double) * 6 * (size_t)n, cudaMemcpyHostToDevice));
    h->have_material = true;
    return MT_OK;
}

int mt_set_dynamics(mt_handle* h, int solver, double gamma, double alpha0, const double* alpha_tab, int nt_alpha,
                    const double* hext, int nt_hext, int hext_row, int renormalize)
{
    if (!h) return fail(MT_ERR_ARG, "null handle");
    if (solver != 1 && solver != 2) return fail(MT_ERR_UNSUPPORTED, "solver %d: only explicit (1) and dynamic (2)", solver);
    if (nt_hext < 0 || nt_alpha < 0) return fail(MT_ERR_ARG, "negative table length");
    if (nt_hext > 0 && !hext) return fail(MT_ERR_ARG, "null hext table");
    if (nt_alpha > 0 && !alpha_tab) return fail(MT_ERR_ARG, "null alpha table");
    if (solver == 1 && (hext_row < 0 || hext_row >= nt_hext))
        return fail(MT_ERR_ARG, "hext_row %d outside the table (%d rows)", hext_row, nt_hext);
    if (!h->hext || h->cap_hext < std::max(nt_hext, 1)) {
        free_ptr(h->hext); h->hext = nullptr;
        CUDA_TRY(dalloc(&h->hext, 4 * (size_t)std::max(nt_hext, 1)));
        h->cap_hext = std::max(nt_hext, 1);
    }
    if (!h->alpha_tab || h->cap_alpha < std::max(nt_alpha, 1)) {
        free_ptr(h->alpha_tab); h->alpha_tab = nullptr;
        CUDA_TRY(dalloc(&h->alpha_tab, 2 * (size_t)std::max(nt_alpha, 1)));
        h->cap_alpha = std::max(nt_alpha, 1);
    }
    CUDA_TRY(cudaMemset(h->hext, 0, sizeof(double) * 4 * std::max(nt_hext, 1)));
    CUDA_TRY(cudaMemset(h->alpha_tab, 0, sizeof(double) * 2 * std::max(nt_alpha, 1)));
    if (nt_hext > 0) CUDA_TRY(cudaMemcpy(h->hext, hext, sizeof(double) * 4 * nt_hext, cudaMemcpyHostToDevice));
    if (nt_alpha > 0) CUDA_TRY(cudaMemcpy(h->alpha_tab, alpha_tab, sizeof(double) * 2 * nt_alpha, cudaMemcpyHostToDevice));
    h->solver = solver; h->gamma = gamma; h->alpha0 = alpha0; h->nt_alpha = nt_alpha; h->nt_hext = nt_hext;
    h->hext_row = hext_row; h->renorm = renormalize ? 1 : 0;
    h->have_dynamics = true;
    return MT_OK;
}

// a new dense tensor replaces the sparse one built from the old (call mt_set_demag_threshold again)
static void drop_sparse(mt_handle* h)
{
    free_ptr(h->sp_rowptr); free_ptr(h->sp_col); free_ptr(h->sp_val);
    h->sp_rowptr = nullptr; h->sp_col = nullptr; h->sp_val = nullptr;
    h->sp_nnz = 0; h->sp_thr = 0.f;
}

int mt_assemble_demag(mt_handle* h, void* stream)
{
    if (!h) return fail(MT_ERR_ARG, "null handle");
    drop_sparse(h);
    int rc = ensure_tensor(h);
    if (rc) return rc;
    CUDA_TRY(launch_assemble(h->nx, h->ny, h->nz, h->L, h->d, h->n, h->ldk, h->shard_cell0, tensor_rows(h), h->K,
                             (cudaStream_t)stream));
    h->have_K = true;
    return MT_OK;
}

// FindThresholdFraction (DemagAuxFunctions.f90:353-428) on the positive entries of the
// six blocks: bisection in single precision between the smallest and the largest
// positive entry until the count of positive entries <= f_middle lies within +-0.01 of
// frac times their number (the bounds in double, as the literal 0.01 is a default
// real of the 8-byte-real build), at most 1000 steps; frac >= 1 removes everything.
static int threshold_fraction(mt_handle* h, float frac, float* thr_out, cudaStream_t s)
{
    if (frac >= 1.0f) { *thr_out = FLT_MAX; return MT_OK; }
    unsigned* mm = nullptr;
    unsigned long long* cnt = nullptr;
    CUDA_TRY(dalloc(&mm, 2));
    struct FreeU { unsigned* p; ~FreeU() { cudaFree(p); } } fm{mm};
    CUDA_TRY(dalloc(&cnt, 2));
    struct FreeC { unsigned long long* p; ~FreeC() { cudaFree(p); } } fcn{cnt};
    CUDA_TRY(sparse_positive_minmax(h->K, h->n, h->ldk, mm, s));
    unsigned mmh[2];
    CUDA_TRY(cudaMemcpyAsync(mmh, mm, sizeof(mmh), cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    if (mmh[1] == 0u) { *thr_out = 0.f; return MT_OK; }   // no positive entry
    float f_small, f_large;
    memcpy(&f_small, &mmh[0], 4);
    memcpy(&f_large, &mmh[1], 4);
    unsigned long long ch[2] = {0, 0};
    float f_middle = f_small;
    for (int k_do = 1;; ++k_do) {
        f_middle = (f_large - f_small) / 2.0f + f_small;
        CUDA_TRY(sparse_count_positive(h->K, h->n, h->ldk, f_middle, cnt, s));
        CUDA_TRY(cudaMemcpyAsync(ch, cnt, sizeof(ch), cudaMemcpyDeviceToHost, s));
        CUDA_TRY(cudaStreamSynchronize(s));
        const unsigned long long n_pos = ch[0], count_middle = ch[1];
        if ((float)count_middle > frac * (float)n_pos) f_large = f_middle;
        else f_small = f_middle;
        const double c = (double)count_middle, np = (double)n_pos;
        if (c >= ((double)frac - 0.01) * np && c <= ((double)frac + 0.01) * np) break;
        if (k_do > 1000) break;
    }
    *thr_out = f_middle;
    return MT_OK;
}

int mt_set_demag_threshold(mt_handle* h, int approx, double value, long long* nnz_out, float* thr_out, void* stream)
{
    if (!h) return fail(MT_ERR_ARG, "null handle");
    if (int rc = refuse_sharded(h, "mt_set_demag_threshold")) return rc;
    if (!h->have_K) return fail(MT_ERR_STATE, "no demag tensor: assemble or load it first");
    cudaStream_t s = (cudaStream_t)stream;
    drop_sparse(h);
    if (approx == 1) return MT_OK;   // the dense product
    if (approx != 2 && approx != 4)
        return fail(MT_ERR_UNSUPPORTED, "demag approximation %d: 1 (none), 2 (threshold), 4 (threshold fraction)", approx);
    if (!(value >= 0.0)) return fail(MT_ERR_ARG, "threshold %g must be >= 0", value);
    float thr = (float)value;
    if (approx == 4) {
        int rc = threshold_fraction(h, (float)value, &thr, s);
        if (rc) return rc;
    }
    const int n = h->n, rows = 3 * n;
    std::vector<int> counts(rows), rowptr(rows + 1);
    int* d_counts = nullptr;
    CUDA_TRY(dalloc(&d_counts, (size_t)rows));
    struct Free { int* p; ~Free() { cudaFree(p); } } fc{d_counts};
    CUDA_TRY(sparse_count_rows(h->K, n, h->ldk, thr, d_counts, s));
    CUDA_TRY(cudaMemcpyAsync(counts.data(), d_counts, sizeof(int) * rows, cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    long long nnz = 0;
    for (int r = 0; r < rows; ++r) { rowptr[r] = (int)nnz; nnz += counts[r]; }
    if (nnz > INT32_MAX) return fail(MT_ERR_UNSUPPORTED, "%lld kept entries exceed 32-bit CSR indices", nnz);
    rowptr[rows] = (int)nnz;
    CUDA_TRY(dalloc(&h->sp_rowptr, (size_t)rows + 1));
    CUDA_TRY(dalloc(&h->sp_col, (size_t)std::max(nnz, 1LL)));
    CUDA_TRY(dalloc(&h->sp_val, (size_t)std::max(nnz, 1LL)));
    CUDA_TRY(cudaMemcpyAsync(h->sp_rowptr, rowptr.data(), sizeof(int) * (rows + 1), cudaMemcpyHostToDevice, s));
    CUDA_TRY(sparse_fill_rows(h->K, n, h->ldk, thr, h->sp_rowptr, h->sp_col, h->sp_val, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    h->sp_nnz = nnz;
    h->sp_thr = thr;
    if (nnz_out) *nnz_out = nnz;
    if (thr_out) *thr_out = thr;
    return MT_OK;
}

int mt_load_demag_colmajor(mt_handle* h, const float* Kxx, const float* Kxy, const float* Kxz, const float* Kyy,
                           const float* Kyz, const float* Kzz)
{
    if (h) drop_sparse(h);
    if (!h || !Kxx || !Kxy || !Kxz || !Kyy || !Kyz || !Kzz) return fail(MT_ERR_ARG, "null argument");
    if (int rc = refuse_sharded(h, "mt_load_demag_colmajor")) return rc;
    int rc = ensure_tensor(h);
    if (rc) return rc;
    const float* blocks[6] = {Kxx, Kxy, Kxz, Kyy, Kyz, Kzz};
    float* tmp = nullptr;
    const size_t nn = (size_t)h->n * h->n;
    CUDA_TRY(dalloc(&tmp, nn));
    for (int c = 0; c < 6; ++c) {
        cudaError_t e = cudaMemcpy(tmp, blocks[c], sizeof(float) * nn, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = launch_colmajor_to_rows(tmp, c, h->n, h->ldk, h->K, 0);
        if (e == cudaSuccess) e = cudaDeviceSynchronize();
        if (e != cudaSuccess) { cudaFree(tmp); return fail(MT_ERR_CUDA, "tensor upload: %s", cudaGetErrorString(e)); }
    }
    cudaFree(tmp);
    h->have_K = true;
    return MT_OK;
}

int mt_get_demag_colmajor(mt_handle* h, float* Kxx, float* Kxy, float* Kxz, float* Kyy, float* Kyz, float* Kzz)
{
    if (!h || !Kxx || !Kxy || !Kxz || !Kyy || !Kyz || !Kzz) return fail(MT_ERR_ARG, "null argument");
    if (int rc = refuse_sharded(h, "mt_get_demag_colmajor")) return rc;
    if (!h->have_K) return fail(MT_ERR_STATE, "no demag tensor");
    float* blocks[6] = {Kxx, Kxy, Kxz, Kyy, Kyz, Kzz};
    float* tmp = nullptr;
    const size_t nn = (size_t)h->n * h->n;
    CUDA_TRY(dalloc(&tmp, nn));
    for (int c = 0; c < 6; ++c) {
        cudaError_t e = launch_rows_to_colmajor(h->K, c, h->n, h->ldk, tmp, 0);
        if (e == cudaSuccess) e = cudaMemcpy(blocks[c], tmp, sizeof(float) * nn, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) { cudaFree(tmp); return fail(MT_ERR_CUDA, "tensor download: %s", cudaGetErrorString(e)); }
    }
    cudaFree(tmp);
    return MT_OK;
}

int mt_demag_field(mt_handle* h, const double* m_dev, double* H_dev, void* stream)
{
    int rc = check_ready(h, true, false);
    if (rc) return rc;
    if ((rc = refuse_sharded(h, "mt_demag_field"))) return rc;
    if (!m_dev || !H_dev) return fail(MT_ERR_ARG, "null device pointer");
    if ((rc = ensure_m32(h))) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    DevProb P = make_prob(h);
    CUDA_TRY(launch_m_to_f32(m_dev, h->n, h->ldk, h->m32, s));
    CUDA_TRY(launch_field(0, P, m_dev, h->m32, 0.0, H_dev, nullptr, nullptr, nullptr, nullptr, 0.f, h->num_sms, s));
    return MT_OK;
}

int mt_fields(mt_handle* h, double t, const double* m_dev, double* Hj, double* Hh, double* Hk, double* Hm, void* stream)
{
    int rc = check_ready(h, true, true);
    if (rc) return rc;
    if ((rc = refuse_sharded(h, "mt_fields"))) return rc;
    if (!m_dev || !Hj || !Hh || !Hk || !Hm) return fail(MT_ERR_ARG, "null device pointer");
    if ((rc = ensure_m32(h))) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    DevProb P = make_prob(h);
    CUDA_TRY(launch_m_to_f32(m_dev, h->n, h->ldk, h->m32, s));
    CUDA_TRY(launch_field(1, P, m_dev, h->m32, t, Hj, Hh, Hk, Hm, nullptr, 0.f, h->num_sms, s));
    return MT_OK;
}

int mt_rhs(mt_handle* h, double t, const double* m_dev, double* dmdt_dev, void* stream)
{
    int rc = check_ready(h, true, true);
    if (rc) return rc;
    if ((rc = refuse_sharded(h, "mt_rhs"))) return rc;
    if (!m_dev || !dmdt_dev) return fail(MT_ERR_ARG, "null device pointer");
    if ((rc = ensure_m32(h))) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    DevProb P = make_prob(h);
    CUDA_TRY(launch_m_to_f32(m_dev, h->n, h->ldk, h->m32, s));
    CUDA_TRY(launch_field(2, P, m_dev, h->m32, t, dmdt_dev, nullptr, nullptr, nullptr, nullptr, 0.f, h->num_sms, s));
    return MT_OK;
}

int mt_rhs_vjp(mt_handle* h, double t, const double* m_dev, const double* lam_dev, double* gm_dev, double* ghe_dev,
               double* gms_dev, void* stream)
{
    int rc = check_ready(h, true, true);
    if (rc) return rc;
    if ((rc = refuse_sharded(h, "mt_rhs_vjp"))) return rc;
    if (!m_dev || !lam_dev || !gm_dev || !ghe_dev || !gms_dev) return fail(MT_ERR_ARG, "null device pointer");
    if ((rc = ensure_m32(h))) return rc;
    const size_t n = (size_t)h->n;
    if (!h->vjp_buf) {
        CUDA_TRY(dalloc(&h->vjp_buf, 4 * n));
        CUDA_TRY(dalloc(&h->vjp_z, 3 * n));
        CUDA_TRY(dalloc(&h->vjp_v32, 3 * (size_t)h->ldk));
        CUDA_TRY(cudaMemset(h->vjp_v32, 0, sizeof(float) * 3 * (size_t)h->ldk));
    }
    cudaStream_t s = (cudaStream_t)stream;
    DevProb P = make_prob(h);
    CUDA_TRY(launch_m_to_f32(m_dev, h->n, h->ldk, h->m32, s));
    CUDA_TRY(cudaMemcpyAsync(h->vjp_buf, lam_dev, sizeof(double) * 3 * n, cudaMemcpyDeviceToDevice, s));
    CUDA_TRY(launch_field(4, P, m_dev, h->m32, t, gm_dev, h->vjp_z, ghe_dev, h->vjp_buf, h->vjp_v32, 0.f, h->num_sms, s));
    CUDA_TRY(launch_field(5, P, m_dev, h->vjp_v32, t, gm_dev, h->vjp_z, nullptr, nullptr, nullptr, 0.f, h->num_sms, s));
    CUDA_TRY(cudaMemcpyAsync(gms_dev, h->vjp_buf + 3 * n, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
    return MT_OK;
}

// ---------------------------------------------------------------------------
// integration driver
// ---------------------------------------------------------------------------
}  // extern "C"

namespace {

// Device buffers of one call.  Bound to a handle (bind), they come from the handle's
// arena, kept between calls; what does not fit is allocated separately, and the arena is
// grown to the whole amount when the call ends, so repeated calls allocate nothing.  A
// handle lends its arena to one integration at a time.
struct IntegAlloc {
    std::vector<void*> ptrs;
    mt_handle* h = nullptr;
    size_t used = 0, want = 0;
    void bind(mt_handle* hh)
    {
        if (hh->integ_arena_busy) return;
        hh->integ_arena_busy = true;
        h = hh;
    }
    template <typename T>
    cudaError_t get(T** p, size_t count)
    {
        if (count == 0) count = 1;
        const size_t bytes = (sizeof(T) * count + 255) & ~(size_t)255;
        want += bytes;
        if (h && used + bytes <= h->integ_arena_bytes) {
            *p = reinterpret_cast<T*>(h->integ_arena + used);
            used += bytes;
            return cudaSuccess;
        }
        cudaError_t e = dalloc(p, count);
        if (e == cudaSuccess) ptrs.push_back((void*)*p);
        return e;
    }
    ~IntegAlloc()
    {
        for (void* p : ptrs) cudaFree(p);
        if (!h) return;
        if (!ptrs.empty()) {   // grow the arena for the next call (the device is idle: cudaFree synchronised)
            free_ptr(h->integ_arena);
            h->integ_arena = nullptr;
            h->integ_arena_bytes = 0;
            if (cudaMalloc((void**)&h->integ_arena, want) == cudaSuccess) h->integ_arena_bytes = want;
            else cudaGetLastError();
        }
        h->integ_arena_busy = false;
    }
};

}  // namespace

extern "C" {

}  // extern "C"

namespace {

// One instance's integration state on the device: RKSUITE buffers, parameters and outputs.
struct IntegRun {
    IntegAlloc A;
    IntegBufs B;
    IntegParams Q;
    DevProb P;
    double* d_tout = nullptr;
    int* d_flags = nullptr;
    int grid = 0;
    size_t smem = 0;
};

// setup_r1 checks, merged output/convergence times, buffers and the initial RKSUITE
// state of one instance, to be integrated by a group of `grid` CTAs
int integ_prepare(mt_handle* h, const double* t, int nt, const double* m0_dev, double tol, double thres,
                  const double* t_conv, int nt_conv, double conv_tol, double* y_out_dev, int grid, IntegRun& R,
                  mt_stats* stats, cudaStream_t s)
{
    memset(stats, 0, sizeof(*stats));
    stats->converged_at = -1;
    const int n = h->n, n3 = 3 * n;

    // ---- setup_r1 checks and initial state (RKSuitef90.f90:596-856) ----
    const double eps = 2.220446049250313e-16;
    const double round_off = 10.0 * eps, sqrrmc = sqrt(eps), cubrmc = pow(eps, 1.0 / 3.0);
    const double sqtiny = sqrt(2.2250738585072014e-308);
    const double cdiff = 1.0 / 18.0;   // min nonzero |c_i - c_j| of the pair (2/9 - 1/6)
    const double toosml = round_off / cdiff;
    const double t_start = t[0], t_end = t[nt - 1];
    if (t_start == t_end) { stats->status = 911; return fail(MT_ERR_ARG, "T_START = T_END"); }
    if (tol > 0.01 || tol < round_off) { stats->status = 911; return fail(MT_ERR_ARG, "tol %g outside (%g, 0.01)", tol, round_off); }
    if (thres < sqtiny) { stats->status = 911; return fail(MT_ERR_ARG, "threshold %g below %g", thres, sqtiny); }
    const double hmin0 = std::max(sqtiny, toosml * std::max(fabs(t_start), fabs(t_end)));
    if (fabs(t_end - t_start) < hmin0) { stats->status = 911; return fail(MT_ERR_ARG, "T_END and T_START not distinguishable"); }

    // ---- merged output / convergence times (ODE_Solvers.f90:183-193) ----
    std::vector<double> comb;
    comb.reserve(nt + nt_conv);
    for (int i = 0; i < nt + nt_conv; ++i) {
        const double v = (i < nt) ? t[i] : t_conv[i - nt];
        bool dup = (i > 0 && v == 0.0);   // simple_unique compares with its zero-filled output
        for (double c : comb) if (c == v) { dup = true; break; }
        if (i == 0 || !dup) comb.push_back(v);
    }
    std::sort(comb.begin(), comb.end());
    std::vector<int> cflags(comb.size(), 0);
    for (size_t k = 0; k < comb.size(); ++k) {
        for (int q = 0; q < nt; ++q) if (t[q] == comb[k]) { cflags[k] |= 1; break; }
        for (int q = 0; q < nt_conv; ++q) if (t_conv[q] == comb[k]) { cflags[k] |= 2; break; }
    }

    // ---- buffers ----
    IntegAlloc& A = R.A;
    A.bind(h);
    IntegBufs& B = R.B;
    memset(&B, 0, sizeof(B));
    if (sharded(h)) {   // stage arguments and partials in the exchange region, which peers write into
        const ShardLayout lay = shard_layout(n, h->ldk, h->shard_world);
        for (int k = 0; k < 4; ++k) {
            B.pool[k] = reinterpret_cast<double*>(h->shard_region + lay.pool) + (size_t)k * n3;
            B.pool32[k] = reinterpret_cast<float*>(h->shard_region + lay.pool32) + (size_t)k * 3 * h->ldk;
        }
        CUDA_TRY(cudaMemsetAsync(B.pool32[0], 0, sizeof(float) * 4 * 3 * (size_t)h->ldk, s));
        B.partials = reinterpret_cast<double*>(h->shard_region + lay.partials);
        B.link = h->shard_link;
    } else {
        for (int k = 0; k < 4; ++k) {
            CUDA_TRY(A.get(&B.pool[k], n3));
            CUDA_TRY(A.get(&B.pool32[k], 3 * (size_t)h->ldk));
            CUDA_TRY(cudaMemsetAsync(B.pool32[k], 0, sizeof(float) * 3 * h->ldk, s));
        }
    }
    for (int k = 0; k < 3; ++k) CUDA_TRY(A.get(&B.deriv[k], n3));
    for (int k = 2; k <= 11; ++k) if (k != 8) CUDA_TRY(A.get(&B.stg[k], n3));
    for (int k = 1; k <= 5; ++k) CUDA_TRY(A.get(&B.p[k], n3));
    CUDA_TRY(A.get(&B.errest, n3));
    CUDA_TRY(A.get(&B.weights, n3));
    CUDA_TRY(A.get(&B.ylast, n3));
    CUDA_TRY(A.get(&B.ystep, n3));
    B.y_out = y_out_dev;
    if (!sharded(h)) CUDA_TRY(A.get(&B.partials, 2 * (size_t)grid * 4));
    CUDA_TRY(A.get(&B.gs, 1));
    CUDA_TRY(A.get(&B.state, 1));
    double* d_comb = nullptr; int* d_cflags = nullptr;
    double*& d_tout = R.d_tout;
    int*& d_flags = R.d_flags;
    CUDA_TRY(A.get(&d_comb, comb.size()));
    CUDA_TRY(A.get(&d_cflags, comb.size()));
    CUDA_TRY(A.get(&d_tout, nt));
    CUDA_TRY(A.get(&d_flags, nt));
    CUDA_TRY(cudaMemcpyAsync(d_comb, comb.data(), sizeof(double) * comb.size(), cudaMemcpyHostToDevice, s));
    CUDA_TRY(cudaMemcpyAsync(d_cflags, cflags.data(), sizeof(int) * comb.size(), cudaMemcpyHostToDevice, s));
    CUDA_TRY(cudaMemsetAsync(d_tout, 0, sizeof(double) * nt, s));
    CUDA_TRY(cudaMemsetAsync(d_flags, 0, sizeof(int) * nt, s));
    // y <- m0 (with its FP32 shadow), first sample, convergence reference
    CUDA_TRY(cudaMemcpyAsync(B.pool[0], m0_dev, sizeof(double) * n3, cudaMemcpyDeviceToDevice, s));
    CUDA_TRY(launch_m_to_f32(m0_dev, n, h->ldk, B.pool32[0], s));
    CUDA_TRY(cudaMemcpyAsync(y_out_dev, m0_dev, sizeof(double) * n3, cudaMemcpyDeviceToDevice, s));
    CUDA_TRY(cudaMemcpyAsync(B.ylast, m0_dev, sizeof(double) * n3, cudaMemcpyDeviceToDevice, s));
    CUDA_TRY(cudaMemsetAsync(B.weights, 0, sizeof(double) * n3, s));

    RKS st;
    memset(&st, 0, sizeof(st));
    st.t = t_start; st.t_old = t_start; st.t_start = t_start; st.t_end = t_end;
    st.dir = (t_end - t_start) >= 0 ? 1.0 : -1.0;
    st.tol = tol;
    st.h = std::max(fabs(t_end - t_start) / 8.0, hmin0);
    st.at_t_start = 1; st.phase2 = 1;
    st.iy = 0; st.iyold = 1; st.ia0 = 2; st.ia1 = 3;
    st.dyp = 0; st.dypold = 1; st.d8 = 2;
    st.ci = 1; st.ko = 1;
    st.converged_at = -1;
    st.xseq = h->shard_xseq; st.rseq = h->shard_rseq;
    CUDA_TRY(cudaMemcpyAsync(B.state, &st, sizeof(st), cudaMemcpyHostToDevice, s));

    IntegParams& Q = R.Q;
    memset(&Q, 0, sizeof(Q));
    Q.thres = thres; Q.round_off = round_off; Q.sqrrmc = sqrrmc; Q.cubrmc = cubrmc; Q.sqtiny = sqtiny;
    Q.toosml = toosml; Q.conv_tol = conv_tol;
    Q.comb_t = d_comb; Q.comb_flags = d_cflags; Q.ncomb = (int)comb.size(); Q.nt = nt;
    Q.t_out = d_tout; Q.flags_out = d_flags;
    Q.renorm = h->renorm;
    // cells the grid's CTAs share; for row shards the largest rank's, so that every
    // rank gets the same evaluation budget per launch and they stop together
    const int cells = sharded(h) ? (n + h->shard_world - 1) / h->shard_world : n;
    {   // about 0.25 s of work per launch
        const double bytes = 24.0 * (double)cells * (double)h->ldk;
        const double t_eval = bytes / 3.0e12 + 15e-6;
        long long b = (long long)(0.25 / t_eval);
        Q.evals_per_launch = std::min(100000LL, std::max(64LL, b));
    }
    // co-residency of the persistent grid
    const size_t smem = integrate_smem_bytes(cells, h->ldk, grid);
    R.smem = smem;
    if (smem > 227 * 1024) return fail(MT_ERR_UNSUPPORTED, "integrator shared memory %zu exceeds 227 KB", smem);
    R.P = make_prob(h);
    R.grid = grid;
    return MT_OK;
}

// outputs and statistics of a finished instance
int integ_finish(IntegRun& R, const RKS& hs, const double* t, int nt, double* t_out, int* flags, mt_stats* stats)
{
    std::vector<int> fl(nt);
    const double* d_tout = R.d_tout;
    const int* d_flags = R.d_flags;
    CUDA_TRY(cudaMemcpy(t_out, d_tout, sizeof(double) * nt, cudaMemcpyDeviceToHost));
    CUDA_TRY(cudaMemcpy(fl.data(), d_flags, sizeof(int) * nt, cudaMemcpyDeviceToHost));
    t_out[0] = t[0];
    fl[0] = 0;
    if (flags) memcpy(flags, fl.data(), sizeof(int) * nt);
    stats->f_evals = hs.full_f_count + hs.f_count;
    stats->steps = hs.step_count;
    stats->bad_steps = hs.bad_step_count;
    stats->n_flag3 = hs.n_flag3;
    stats->n_flag4 = hs.n_flag4;
    stats->n_out = hs.ko;
    stats->status = hs.status;
    stats->converged_at = hs.converged_at;
    if (hs.status != 0) return fail(MT_ERR_SOLVER, "integrator stopped with RKSUITE flag %d", hs.status);
    return MT_OK;
}

// ---- row shards ----

int shard_ready(const mt_handle* h)
{
    if (!h->shard_region) return fail(MT_ERR_STATE, "row shard: call mt_shard_region first");
    if (!h->shard_peers_set) return fail(MT_ERR_STATE, "row shard: the peers' regions are not set");
    if (h->shard_broken) return fail(MT_ERR_STATE, "row shard: an earlier run gave up; destroy the ranks' handles");
    return MT_OK;
}

// CTAs per rank: the same on every rank (from the largest rank's cells)
int shard_grid(const mt_handle* h, int sms)
{
    return std::min(kShardMaxCtas, integrate_grid_size((h->n + h->shard_world - 1) / h->shard_world, sms));
}

// the device link of this rank for a launch of `grid` CTAs per rank
int build_link(mt_handle* h, int grid)
{
    const ShardLayout lay = shard_layout(h->n, h->ldk, h->shard_world);
    ShardLink L;
    memset(&L, 0, sizeof(L));
    L.rank = h->shard_rank; L.world = h->shard_world;
    L.cell0 = h->shard_cell0; L.ncell = h->shard_ncell;
    L.cta_base = h->shard_rank * grid; L.cta_total = h->shard_world * grid;
    // ranks may enter a run some time apart: 10 s by default, MAGTENSE_B200_SHARD_TIMEOUT_S overrides
    double tmo_s = 10.0;
    if (const char* e = getenv("MAGTENSE_B200_SHARD_TIMEOUT_S")) {
        const double v = atof(e);
        if (v > 0.0 && v <= 600.0) tmo_s = v;
    }
    L.timeout_ns = (unsigned long long)(tmo_s * 1e9);
    h->shard_timeout_s = tmo_s;
    for (int p = 0; p < h->shard_world; ++p) {
        unsigned char* base = static_cast<unsigned char*>(h->shard_peer[p]);
        for (int k = 0; k < 4; ++k) {
            L.pool[p][k] = reinterpret_cast<double*>(base + lay.pool) + (size_t)k * 3 * h->n;
            L.pool32[p][k] = reinterpret_cast<float*>(base + lay.pool32) + (size_t)k * 3 * h->ldk;
        }
        L.partials[p] = reinterpret_cast<double*>(base + lay.partials);
        L.flags[p] = reinterpret_cast<unsigned*>(base + lay.flags);
    }
    if (!h->shard_link) CUDA_TRY(dalloc(&h->shard_link, 1));
    CUDA_TRY(cudaMemcpy(h->shard_link, &L, sizeof(L), cudaMemcpyHostToDevice));
    return MT_OK;
}

// Barrier and RKSUITE state of a CTA group after a launch.
struct GroupBack { GridSync gs; RKS st; };

// Integrates prepared runs as CTA groups of one cooperative launch on one device,
// relaunched until every group has finished (replayed from a CUDA graph when
// `graph`).  runs[k]->grid CTAs go to group k.  back receives each group's final
// barrier and state.
// Relaunch planning of a ragged batch: after a launch in which instances finished, their
// CTAs go to the unfinished groups, one at a time to the group with the most demag work
// (n^2) per CTA, up to cap CTAs each; a group never shrinks, so its shared-memory need
// stays within the first plan's.  CTAs left over join a finished instance's group, which
// returns at once.  An instance's trajectory does not depend on its group size.
struct GroupPlan {
    std::vector<int> cap;
    std::vector<double> work;
    double launch_s = 0.25;   // target device time of one launch per group
};

int run_groups(const std::vector<IntegRun*>& runs, bool graph, cudaStream_t cs, std::vector<GroupBack>& back_out,
               long long& launches, double& kernel_ms, const GroupPlan* plan)
{
    const int ninst = (int)runs.size();
    size_t smem = 0;
    int used = 0;
    for (IntegRun* r : runs) { smem = std::max(smem, r->smem); used += r->grid; }
    std::vector<RaggedInst> tab(ninst);
    std::vector<int> cta_inst(used);
    for (int k = 0, c0 = 0; k < ninst; ++k) {
        tab[k].P = runs[k]->P; tab[k].B = runs[k]->B; tab[k].Q = runs[k]->Q;
        tab[k].cta0 = c0; tab[k].ncta = runs[k]->grid;
        for (int j = 0; j < runs[k]->grid; ++j) cta_inst[c0 + j] = k;
        c0 += runs[k]->grid;
    }
    IntegAlloc A;
    RaggedInst* d_tab = nullptr;
    int* d_cta = nullptr;
    CUDA_TRY(A.get(&d_tab, (size_t)ninst));
    CUDA_TRY(A.get(&d_cta, (size_t)used));
    CUDA_TRY(cudaMemcpyAsync(d_tab, tab.data(), sizeof(RaggedInst) * ninst, cudaMemcpyHostToDevice, cs));
    CUDA_TRY(cudaMemcpyAsync(d_cta, cta_inst.data(), sizeof(int) * used, cudaMemcpyHostToDevice, cs));
    // pinned read-back of every group's barrier and RKSUITE state after a launch
    GroupBack* back = nullptr;
    CUDA_TRY(cudaMallocHost((void**)&back, sizeof(GroupBack) * ninst));
    struct HostFree { void* p; ~HostFree() { cudaFreeHost(p); } } hf{back};
    // private stream (the caller's may be the legacy default stream, which cannot be captured)
    cudaStream_t s = nullptr;
    CUDA_TRY(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    struct StreamGuard { cudaStream_t s; ~StreamGuard() { cudaStreamDestroy(s); } } sg{s};
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, evc = nullptr;
    CUDA_TRY(cudaEventCreate(&ev0));
    CUDA_TRY(cudaEventCreate(&ev1));
    CUDA_TRY(cudaEventCreateWithFlags(&evc, cudaEventDisableTiming));
    struct EvGuard { cudaEvent_t a, b, c; ~EvGuard() { cudaEventDestroy(a); cudaEventDestroy(b); cudaEventDestroy(c); } }
        evg{ev0, ev1, evc};
    CUDA_TRY(cudaEventRecord(evc, cs));
    CUDA_TRY(cudaStreamWaitEvent(s, evc, 0));
    auto enqueue = [&]() -> cudaError_t {
        cudaError_t e = cudaSuccess;
        for (int k = 0; k < ninst && e == cudaSuccess; ++k) e = cudaMemsetAsync(runs[k]->B.gs, 0, sizeof(GridSync), s);
        if (e == cudaSuccess) e = launch_integrate_ragged(d_tab, d_cta, used, smem, s);
        for (int k = 0; k < ninst && e == cudaSuccess; ++k) {
            e = cudaMemcpyAsync(&back[k].gs, runs[k]->B.gs, sizeof(GridSync), cudaMemcpyDeviceToHost, s);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(&back[k].st, runs[k]->B.state, sizeof(RKS), cudaMemcpyDeviceToHost, s);
        }
        return e;
    };
    cudaGraphExec_t gexec = nullptr;
    struct GraphGuard { cudaGraphExec_t g; ~GraphGuard() { if (g) cudaGraphExecDestroy(g); } } gg{nullptr};
    if (graph) {
        cudaGraph_t gr = nullptr;
        CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        cudaError_t e = enqueue();
        cudaError_t e2 = cudaStreamEndCapture(s, &gr);
        if (e != cudaSuccess || e2 != cudaSuccess) {
            if (gr) cudaGraphDestroy(gr);
            cudaGetLastError();
            return fail(MT_ERR_CUDA, "capturing the group launch: %s", cudaGetErrorString(e != cudaSuccess ? e : e2));
        }
        e = cudaGraphInstantiate(&gexec, gr, 0);
        cudaGraphDestroy(gr);
        if (e != cudaSuccess) return fail(MT_ERR_CUDA, "instantiating the group launch: %s", cudaGetErrorString(e));
        gg.g = gexec;
    }
    kernel_ms = 0.0;
    launches = 0;
    std::vector<long long> last(ninst, -1);
    back_out.assign(ninst, GroupBack());
    for (;;) {
        CUDA_TRY(cudaEventRecord(ev0, s));
        if (gexec) CUDA_TRY(cudaGraphLaunch(gexec, s));
        else CUDA_TRY(enqueue());
        CUDA_TRY(cudaEventRecord(ev1, s));
        CUDA_TRY(cudaStreamSynchronize(s));
        float ms = 0.f;
        CUDA_TRY(cudaEventElapsedTime(&ms, ev0, ev1));
        kernel_ms += ms;
        launches++;
        bool all = true, progress = false;
        for (int k = 0; k < ninst; ++k) {
            const GroupBack& bk = back[k];
            back_out[k] = bk;
            if (bk.gs.err != 0 || bk.gs.abort)
                return fail(MT_ERR_TIMEOUT, "group %d: barrier gave up (code %d at %d)", k, bk.gs.err, bk.gs.err_where);
            if (!bk.st.finished) all = false;
            const long long sig = bk.st.full_f_count + bk.st.f_count + bk.st.ci;
            if (sig != last[k]) progress = true;
            last[k] = sig;
        }
        if (all) break;
        if (!progress) return fail(MT_ERR_SOLVER, "grouped integrator made no progress");
        if (plan) {
            // re-plan when an instance with CTAs of its own has finished
            bool freed = false;
            for (int k = 0; k < ninst; ++k)
                if (back[k].st.finished && tab[k].ncta > 0 && runs[k]->grid > 0) freed = true;
            if (freed) {
                std::vector<int> nc(ninst, 0);
                int given = 0;
                for (int k = 0; k < ninst; ++k)
                    if (!back[k].st.finished) { nc[k] = runs[k]->grid; given += nc[k]; }
                for (; given < used; ++given) {
                    int j = -1;
                    double best = 0.0;
                    for (int k = 0; k < ninst; ++k)
                        if (!back[k].st.finished && nc[k] < plan->cap[k] && plan->work[k] / nc[k] > best) {
                            best = plan->work[k] / nc[k];
                            j = k;
                        }
                    if (j < 0) break;
                    nc[j]++;
                }
                int idle_k = -1;
                for (int k = 0; k < ninst && idle_k < 0; ++k)
                    if (back[k].st.finished) idle_k = k;
                nc[idle_k] += used - given;   // some instance has finished, so idle_k >= 0
                for (int k = 0, c0 = 0; k < ninst; ++k) {
                    tab[k].cta0 = c0;
                    tab[k].ncta = nc[k];
                    for (int j = 0; j < nc[k]; ++j) cta_inst[c0 + j] = k;
                    c0 += nc[k];
                    if (!back[k].st.finished && nc[k] != runs[k]->grid) {
                        const double t_eval = plan->work[k] * 24.0 / (nc[k] * 30.0e9) + 15e-6;
                        tab[k].Q.evals_per_launch =
                            std::min(100000LL, std::max(plan->launch_s < 0.25 ? 1LL : 64LL, (long long)(plan->launch_s / t_eval)));
                    }
                    runs[k]->grid = back[k].st.finished ? 0 : nc[k];
                }
                CUDA_TRY(cudaMemcpyAsync(d_tab, tab.data(), sizeof(RaggedInst) * ninst, cudaMemcpyHostToDevice, s));
                CUDA_TRY(cudaMemcpyAsync(d_cta, cta_inst.data(), sizeof(int) * used, cudaMemcpyHostToDevice, s));
            }
        }
    }
    CUDA_TRY(cudaEventRecord(evc, s));
    CUDA_TRY(cudaStreamWaitEvent(cs, evc, 0));
    return MT_OK;
}



}  // namespace

extern "C" {

static int integrate_single(mt_handle* h, const double* t, int nt, const double* m0_dev, double tol, double thres,
                            const double* t_conv, int nt_conv, double conv_tol, double* t_out, double* y_out_dev,
                            int* flags, mt_stats* stats, void* stream);

int mt_integrate(mt_handle* h, const double* t, int nt, const double* m0_dev, double tol, double thres,
                 const double* t_conv, int nt_conv, double conv_tol, double* t_out, double* y_out_dev, int* flags,
                 mt_stats* stats, void* stream)
{
    const int rc = integrate_single(h, t, nt, m0_dev, tol, thres, t_conv, nt_conv, conv_tol, t_out, y_out_dev, flags,
                                    stats, stream);
    // a row shard whose run failed past the argument checks (CUDA error, timeout, no progress)
    // may have left peers mid-run: it takes no further runs
    if (rc != MT_OK && rc != MT_ERR_ARG && rc != MT_ERR_STATE) mark_broken(h);
    return rc;
}

static int integrate_single(mt_handle* h, const double* t, int nt, const double* m0_dev, double tol, double thres,
                            const double* t_conv, int nt_conv, double conv_tol, double* t_out, double* y_out_dev,
                            int* flags, mt_stats* stats, void* stream)
{
    int rc = check_ready(h, true, true);
    if (rc) return rc;
    if (!t || nt < 2 || !m0_dev || !t_out || !y_out_dev || !stats) return fail(MT_ERR_ARG, "bad argument (nt >= 2 required)");
    if (nt_conv < 0 || (nt_conv > 0 && !t_conv)) return fail(MT_ERR_ARG, "bad convergence-time list");
    cudaStream_t s = (cudaStream_t)stream;
    int grid0 = integrate_grid_size(h->n, h->num_sms);
    if (sharded(h)) {   // this rank's part of a row-sharded instance; the peers run theirs at the same time
        if ((rc = shard_ready(h))) return rc;
        grid0 = shard_grid(h, h->num_sms);
        if ((rc = build_link(h, grid0))) return rc;
    }
    IntegRun R;
    int prc = integ_prepare(h, t, nt, m0_dev, tol, thres, t_conv, nt_conv, conv_tol, y_out_dev, grid0, R, stats, s);
    if (prc) return prc;
    DevProb P = R.P;
    // the tensor lines kept in L2 (evict_last) return to normal priority when the run ends
    struct L2Reset { bool on; ~L2Reset() { if (on) cudaCtxResetPersistingL2Cache(); } } l2r{P.l2_keep > 0.f};
    IntegBufs& B = R.B;
    IntegParams& Q = R.Q;
    const int grid = R.grid;
    RKS hs;
    long long last_evals = -1;
    int last_ci = -1;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    CUDA_TRY(cudaEventCreate(&ev0));
    CUDA_TRY(cudaEventCreate(&ev1));
    struct EvGuard { cudaEvent_t a, b; ~EvGuard() { cudaEventDestroy(a); cudaEventDestroy(b); } } evg{ev0, ev1};
    double kernel_ms = 0.0;
    long long launches = 0;
    for (;;) {
        CUDA_TRY(cudaMemsetAsync(B.gs, 0, sizeof(GridSync), s));
        CUDA_TRY(cudaEventRecord(ev0, s));
        CUDA_TRY(launch_integrate(P, B, Q, grid, s));
        CUDA_TRY(cudaEventRecord(ev1, s));
        GridSync gs_h;
        CUDA_TRY(cudaMemcpyAsync(&gs_h, B.gs, sizeof(gs_h), cudaMemcpyDeviceToHost, s));
        CUDA_TRY(cudaMemcpyAsync(&hs, B.state, sizeof(hs), cudaMemcpyDeviceToHost, s));
        CUDA_TRY(cudaStreamSynchronize(s));
        float ms = 0.f;
        CUDA_TRY(cudaEventElapsedTime(&ms, ev0, ev1));
        kernel_ms += ms;
        launches++;
        stats->launches = launches;
        stats->kernel_ms = kernel_ms;
        if (gs_h.err != 0 || gs_h.abort) {
            mark_broken(h);
            return fail(MT_ERR_TIMEOUT, "integrator %s barrier gave up (code %d at %d)",
                        gs_h.err == KERR_PEER_TIMEOUT ? "cross-rank"
                        : gs_h.err == KERR_PEER_ABORT ? "cross-rank (another rank gave up)" : "grid",
                        gs_h.err, gs_h.err_where);
        }
        if (hs.finished) break;
        const long long evals = hs.full_f_count + hs.f_count;
        if (evals == last_evals && hs.ci == last_ci) {
            mark_broken(h);
            return fail(MT_ERR_SOLVER, "integrator made no progress");
        }
        last_evals = evals;
        last_ci = hs.ci;
    }
    h->shard_xseq = hs.xseq;
    h->shard_rseq = hs.rseq;
    return integ_finish(R, hs, t, nt, t_out, flags, stats);
}


int mt_integrate_ragged(mt_handle* const* hs, int ninst, const double* t, int nt, const double* const* m0_dev,
                        double tol, double thres, double* t_out, double* const* y_out_dev, int* flags, mt_stats* stats,
                        int options, void* stream)
{
    if (!hs || ninst < 1 || !t || nt < 2 || !m0_dev || !t_out || !y_out_dev || !stats)
        return fail(MT_ERR_ARG, "bad argument (ninst >= 1, nt >= 2 required)");
    int rc;
    for (int k = 0; k < ninst; ++k) {
        if (!hs[k] || !m0_dev[k] || !y_out_dev[k]) return fail(MT_ERR_ARG, "null handle or buffer of instance %d", k);
        if ((rc = check_ready(hs[k], true, true))) return rc;
        if ((rc = refuse_sharded(hs[k], "mt_integrate_ragged"))) return rc;
        if (hs[k]->device != hs[0]->device) return fail(MT_ERR_ARG, "all instances must live on one device");
    }
    const int G = hs[0]->num_sms;
    if (ninst > G) return fail(MT_ERR_UNSUPPORTED, "%d instances exceed the %d SMs of one launch", ninst, G);
    // CTA groups for the demag work n^2 per evaluation (at least one CTA, at most n/8): one
    // CTA each, then every further CTA to the group with the most work per CTA, which
    // minimises the slowest group's time per evaluation
    std::vector<double> w(ninst);
    for (int k = 0; k < ninst; ++k) w[k] = (double)hs[k]->n * (double)hs[k]->n;
    std::vector<int> ncta(ninst, 1), cap(ninst);
    for (int k = 0; k < ninst; ++k) cap[k] = integrate_grid_size(hs[k]->n, G);
    for (int used = ninst; used < G; ++used) {
        int j = -1;
        double best = 0.0;
        for (int k = 0; k < ninst; ++k)
            if (ncta[k] < cap[k] && w[k] / ncta[k] > best) { best = w[k] / ncta[k]; j = k; }
        if (j < 0) break;
        ncta[j]++;
    }
    cudaStream_t cs = (cudaStream_t)stream;
    std::vector<std::unique_ptr<IntegRun>> runs(ninst);
    std::vector<IntegRun*> rp(ninst);
    for (int k = 0; k < ninst; ++k) {
        runs[k].reset(new IntegRun());
        rp[k] = runs[k].get();
        // the reduction slots for the largest group the instance may get (cap CTAs); the group
        // starts with ncta CTAs and the shared memory those need
        if ((rc = integ_prepare(hs[k], t, nt, m0_dev[k], tol, thres, nullptr, 0, 0.0, y_out_dev[k], cap[k], *runs[k],
                                &stats[k], cs)))
            return rc;
        runs[k]->grid = ncta[k];
        runs[k]->smem = integrate_smem_bytes(hs[k]->n, hs[k]->ldk, ncta[k]);
        if (runs[k]->smem > 227 * 1024)
            return fail(MT_ERR_UNSUPPORTED, "integrator shared memory %zu exceeds 227 KB", runs[k]->smem);
        // about 0.25 s per launch for this group: 24 n^2 bytes per evaluation over ncta SMs
        const double t_eval = 24.0 * (double)hs[k]->n * (double)hs[k]->ldk / (ncta[k] * 30.0e9) + 15e-6;
        runs[k]->Q.evals_per_launch = std::min(100000LL, std::max(64LL, (long long)(0.25 / t_eval)));
    }
    // the L2 evict_last share of the loads, for the tensors of all instances together
    double tensor_bytes = 0.0;
    for (int k = 0; k < ninst; ++k) tensor_bytes += 24.0 * (double)hs[k]->n * (double)hs[k]->ldk;
    const float keep = l2_keep_fraction(hs[0]->device, tensor_bytes);
    for (int k = 0; k < ninst; ++k) runs[k]->P.l2_keep = keep;
    struct L2Reset { bool on; ~L2Reset() { if (on) cudaCtxResetPersistingL2Cache(); } } l2r{keep > 0.f};
    std::vector<GroupBack> back;
    long long launches = 0;
    double kernel_ms = 0.0;
    GroupPlan plan;
    plan.cap = cap;
    if (const char* e = getenv("MT_RAGGED_LAUNCH_S")) {   // device time per launch (tests: many relaunches)
        const double v = atof(e);
        if (v > 0.0 && v <= 10.0) {
            plan.launch_s = v;
            for (int k = 0; k < ninst; ++k) {
                const double t_eval = 24.0 * (double)hs[k]->n * (double)hs[k]->ldk / (ncta[k] * 30.0e9) + 15e-6;
                runs[k]->Q.evals_per_launch = std::min(100000LL, std::max(1LL, (long long)(v / t_eval)));
            }
        }
    }
    plan.work.resize(ninst);
    for (int k = 0; k < ninst; ++k) plan.work[k] = (double)hs[k]->n * (double)hs[k]->ldk;
    if ((rc = run_groups(rp, (options & MT_RAGGED_GRAPH) != 0, cs, back, launches, kernel_ms, &plan))) return rc;
    int worst = MT_OK;
    for (int k = 0; k < ninst; ++k) {
        const int r = integ_finish(*runs[k], back[k].st, t, nt, t_out + (size_t)k * nt, flags ? flags + (size_t)k * nt : nullptr,
                                   &stats[k]);
        if (r && worst == MT_OK) worst = r;
    }
    stats[0].launches = launches;
    stats[0].kernel_ms = kernel_ms;
    return worst;
}

int mt_set_row_shard(mt_handle* h, int rank, int world)
{
    if (!h) return fail(MT_ERR_ARG, "null handle");
    if (world < 2 || world > kMaxShards) return fail(MT_ERR_ARG, "world %d outside [2, %d]", world, kMaxShards);
    if (rank < 0 || rank >= world) return fail(MT_ERR_ARG, "rank %d outside [0, %d)", rank, world);
    if (h->n < world) return fail(MT_ERR_ARG, "%d cells cannot be split over %d ranks", h->n, world);
    if (h->K || h->shard_region) return fail(MT_ERR_STATE, "mt_set_row_shard must come before the tensor and the region");
    h->shard_rank = rank;
    h->shard_world = world;
    h->shard_cell0 = (int)(((long long)h->n * rank) / world);
    h->shard_ncell = (int)(((long long)h->n * (rank + 1)) / world) - h->shard_cell0;
    return MT_OK;
}

int mt_shard_region(mt_handle* h, void** region_dev, size_t* bytes)
{
    if (!h || !region_dev || !bytes) return fail(MT_ERR_ARG, "null argument");
    if (!sharded(h)) return fail(MT_ERR_STATE, "not a row shard: call mt_set_row_shard first");
    const ShardLayout lay = shard_layout(h->n, h->ldk, h->shard_world);
    if (!h->shard_region) {
        CUDA_TRY(dalloc(&h->shard_region, lay.bytes));
        CUDA_TRY(cudaMemset(h->shard_region, 0, lay.bytes));
        CUDA_TRY(cudaDeviceSynchronize());
        h->shard_peer[h->shard_rank] = h->shard_region;
    }
    *region_dev = h->shard_region;
    *bytes = lay.bytes;
    return MT_OK;
}

int mt_shard_ipc_handle(mt_handle* h, void* handle_out)
{
    if (!h || !handle_out) return fail(MT_ERR_ARG, "null argument");
    if (!h->shard_region) return fail(MT_ERR_STATE, "call mt_shard_region first");
    static_assert(sizeof(cudaIpcMemHandle_t) == 64, "IPC handle size");
    cudaIpcMemHandle_t ih;
    CUDA_TRY(cudaIpcGetMemHandle(&ih, h->shard_region));
    memcpy(handle_out, &ih, sizeof(ih));
    return MT_OK;
}

int mt_shard_open_peers(mt_handle* h, const void* handles)
{
    if (!h || !handles) return fail(MT_ERR_ARG, "null argument");
    if (!h->shard_region) return fail(MT_ERR_STATE, "call mt_shard_region first");
    if (h->shard_peers_set) return fail(MT_ERR_STATE, "the peers' regions are already set");
    const unsigned char* hb = static_cast<const unsigned char*>(handles);
    for (int p = 0; p < h->shard_world; ++p) {
        if (p == h->shard_rank) continue;
        cudaIpcMemHandle_t ih;
        memcpy(&ih, hb + (size_t)p * sizeof(ih), sizeof(ih));
        void* ptr = nullptr;
        CUDA_TRY(cudaIpcOpenMemHandle(&ptr, ih, cudaIpcMemLazyEnablePeerAccess));
        h->shard_peer[p] = ptr;
        h->shard_ipc[p] = true;
    }
    h->shard_peers_set = true;
    return MT_OK;
}

int mt_shard_set_peers(mt_handle* h, void* const* regions_dev)
{
    if (!h || !regions_dev) return fail(MT_ERR_ARG, "null argument");
    if (!h->shard_region) return fail(MT_ERR_STATE, "call mt_shard_region first");
    if (h->shard_peers_set) return fail(MT_ERR_STATE, "the peers' regions are already set");
    if (regions_dev[h->shard_rank] != h->shard_region)
        return fail(MT_ERR_ARG, "entry %d must be this rank's own region", h->shard_rank);
    for (int p = 0; p < h->shard_world; ++p)
        if (!regions_dev[p]) return fail(MT_ERR_ARG, "null region of rank %d", p);
    for (int p = 0; p < h->shard_world; ++p) h->shard_peer[p] = regions_dev[p];
    h->shard_peers_set = true;
    return MT_OK;
}

int mt_integrate_shards_local(mt_handle* const* hs, int world, const double* t, int nt, const double* m0_dev,
                              double tol, double thres, const double* t_conv, int nt_conv, double conv_tol,
                              double* t_out, double* y_out_dev, int* flags, mt_stats* stats, void* stream)
{
    if (!hs || world < 2 || world > kMaxShards || !t || nt < 2 || !m0_dev || !t_out || !y_out_dev || !stats)
        return fail(MT_ERR_ARG, "bad argument (2 <= world <= %d, nt >= 2 required)", kMaxShards);
    if (nt_conv < 0 || (nt_conv > 0 && !t_conv)) return fail(MT_ERR_ARG, "bad convergence-time list");
    int rc;
    for (int r = 0; r < world; ++r) {
        if (!hs[r]) return fail(MT_ERR_ARG, "null handle of rank %d", r);
        if ((rc = check_ready(hs[r], true, true))) return rc;
        if (!sharded(hs[r]) || hs[r]->shard_rank != r || hs[r]->shard_world != world)
            return fail(MT_ERR_ARG, "handle %d is not rank %d of %d row shards", r, r, world);
        if (hs[r]->n != hs[0]->n || hs[r]->device != hs[0]->device)
            return fail(MT_ERR_ARG, "the shards must share one grid and one device");
        if ((rc = shard_ready(hs[r]))) return rc;
    }
    const int grid = shard_grid(hs[0], hs[0]->num_sms / world);
    if (grid < 1) return fail(MT_ERR_UNSUPPORTED, "%d ranks exceed the %d SMs of one launch", world, hs[0]->num_sms);
    cudaStream_t cs = (cudaStream_t)stream;
    std::vector<std::unique_ptr<IntegRun>> runs(world);
    std::vector<IntegRun*> rp(world);
    std::vector<mt_stats> st(world);
    for (int r = 0; r < world; ++r) {
        if ((rc = build_link(hs[r], grid))) return rc;
        runs[r].reset(new IntegRun());
        rp[r] = runs[r].get();
        if ((rc = integ_prepare(hs[r], t, nt, m0_dev, tol, thres, t_conv, nt_conv, conv_tol, y_out_dev, grid, *runs[r],
                                &st[r], cs)))
            return rc;
    }
    std::vector<GroupBack> back;
    long long launches = 0;
    double kernel_ms = 0.0;
    rc = run_groups(rp, false, cs, back, launches, kernel_ms, nullptr);
    if (rc) {
        for (int r = 0; r < world; ++r) mark_broken(hs[r]);
        return rc;
    }
    for (int r = 0; r < world; ++r) {
        const RKS& a = back[r].st;
        const RKS& b = back[0].st;
        if (a.full_f_count + a.f_count != b.full_f_count + b.f_count || a.step_count != b.step_count ||
            a.ko != b.ko || a.t != b.t || a.xseq != b.xseq) {
            for (int q = 0; q < world; ++q) mark_broken(hs[q]);
            return fail(MT_ERR_SOLVER, "row shard %d took different steps from rank 0", r);
        }
        hs[r]->shard_xseq = a.xseq;
        hs[r]->shard_rseq = a.rseq;
    }
    rc = integ_finish(*runs[0], back[0].st, t, nt, t_out, flags, stats);
    stats->launches = launches;
    stats->kernel_ms = kernel_ms;
    return rc;
}

// ---------------------------------------------------------------------------
// batched instances
// ---------------------------------------------------------------------------
}  // extern "C"

namespace { struct BatchRun; }
static void batch_ws_free(mt_batch* bt);

struct mt_batch {
    mt_handle* h = nullptr;
    int B = 0, prec = 0;
    int CB = 0, IB = 0, S = 0, np = 0, Kd = 0, grid = 0;
    uint16_t* khi = nullptr;
    uint16_t* klo = nullptr;
    float* row_inv = nullptr;
    int8_t* klimb = nullptr;      // int8 backend: [4][3np][Kd]
    double* row_scale = nullptr;  // [3np]
    double* hext = nullptr;
    double* alpha0 = nullptr;
    int nt_hext = 0;
    bool have_dynamics = false;
    // the damping table shared by the instances whose alpha0 is 0 (alpha(), :281-294), and the
    // shared dynamics last set, so that either call may come first
    std::vector<double> alpha_tab;
    int solver = 2, renorm = 0;
    double gamma = 0.0;
    // device workspace of the integrator (state vectors, operands, partial sums), kept
    // between calls while the output count nt is unchanged
    BatchRun* ws = nullptr;
    int ws_nt = -1;
    // int8 GEMM schedule word per active tile count (autotuned by mt_batch_tune)
    std::vector<int> sched;
    bool tuned = false;
};

namespace {

PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;

int get_encoder()
{
    if (g_encode) return MT_OK;
    cudaDriverEntryPointQueryResult q;
    void* fn = nullptr;
    cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q);
    if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !fn)
        return fail(MT_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
    g_encode = (PFN_cuTensorMapEncodeTiled_v12000)fn;
    return MT_OK;
}

// 2-D BF16 tensor [outer][inner] (inner contiguous), box {32, box_outer}, 64-byte swizzle
int make_tmap(CUtensorMap* m, const void* base, uint64_t inner, uint64_t outer, uint32_t box_outer)
{
    int rc = get_encoder();
    if (rc) return rc;
    cuuint64_t dims[2] = {inner, outer};
    cuuint64_t strides[1] = {inner * 2};
    cuuint32_t box[2] = {(cuuint32_t)kTcKB, box_outer};
    cuuint32_t es[2] = {1, 1};
    CUresult r = g_encode(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides, box, es,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(MT_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return MT_OK;
}

// 3-D int8 tensor [limbs][outer][inner] (inner contiguous), box {128, box_outer, 1}, 128-byte swizzle
int make_tmap_i8(CUtensorMap* m, const void* base, uint64_t inner, uint64_t outer, uint64_t limbs, uint32_t box_outer)
{
    int rc = get_encoder();
    if (rc) return rc;
    cuuint64_t dims[3] = {inner, outer, limbs};
    cuuint64_t strides[2] = {inner, inner * outer};
    cuuint32_t box[3] = {(cuuint32_t)kI8KB, box_outer, 1};
    cuuint32_t es[3] = {1, 1, 1};
    CUresult r = g_encode(m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, const_cast<void*>(base), dims, strides, box, es,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(MT_ERR_CUDA, "cuTensorMapEncodeTiled (int8) failed (%d)", (int)r);
    return MT_OK;
}

DevProb batch_prob(const mt_batch* bt)
{
    DevProb P = make_prob(bt->h);
    return P;
}

}  // namespace

extern "C" {

int mt_batch_create(const mt_grid* g, int B, int precision, mt_batch** out)
{
    if (!out) return fail(MT_ERR_ARG, "null argument");
    *out = nullptr;
    if (B < 1) return fail(MT_ERR_ARG, "B must be >= 1");
    if (precision < 0 || precision > 4) return fail(MT_ERR_ARG, "unknown precision %d", precision);
    mt_handle* h = nullptr;
    int rc = mt_create(g, &h);
    if (rc) return rc;
    cudaError_t e = batch_upload_tables();
    if (e != cudaSuccess) { mt_destroy(h); return fail(MT_ERR_CUDA, "batch tables: %s", cudaGetErrorString(e)); }
    mt_batch* bt = new mt_batch();
    bt->h = h;
    bt->B = B;
    bt->prec = precision;
    bt->grid = batch_grid(h->n, B, h->num_sms, precision, &bt->CB, &bt->IB, &bt->S);
    bt->np = bt->CB * kCellBlock;
    bt->Kd = 3 * bt->np;
    bt->sched.assign(2 * kMaxIB + 1, bt->grid);   // all CTAs, tile-major
    if (precision == MT_PREC_INT8 && bt->Kd > 32000) {
        // D_s sums up to four limb products of magnitude <= 2^14 over the k range in int32
        mt_batch_destroy(bt);
        return fail(MT_ERR_UNSUPPORTED, "int8 precision supports up to 10624 cells");
    }
    *out = bt;
    return MT_OK;
}

int mt_batch_destroy(mt_batch* bt)
{
    if (!bt) return MT_OK;
    batch_ws_free(bt);
    free_ptr(bt->khi); free_ptr(bt->row_inv); free_ptr(bt->hext); free_ptr(bt->alpha0);
    free_ptr(bt->klimb); free_ptr(bt->row_scale);
    mt_destroy(bt->h);
    delete bt;
    return MT_OK;
}

int mt_batch_set_material(mt_batch* bt, double A0, const double* Ms, const double* K0, const double* u_ea)
{
    if (!bt) return fail(MT_ERR_ARG, "null handle");
    return mt_set_material(bt->h, A0, Ms, K0, u_ea);
}

// The shared part of the batch's dynamics lives in the inner handle: solver, gamma, the
// renormalisation switch and the damping table; per-instance fields and alpha0 are the
// batch's own.  Its field table is unused.
static int batch_shared_dynamics(mt_batch* bt)
{
    double dummy_tab[8] = {0, 0, 0, 0, 1, 0, 0, 0};
    const bool tab = !bt->alpha_tab.empty();
    return mt_set_dynamics(bt->h, bt->solver, bt->gamma, 1.0, tab ? bt->alpha_tab.data() : dummy_tab,
                           tab ? (int)(bt->alpha_tab.size() / 2) : 1, dummy_tab, 2, 0, bt->renorm);
}

int mt_batch_set_dynamics(mt_batch* bt, int solver, double gamma, const double* alpha0, const double* hext, int nt_hext,
                          int renormalize)
{
    if (!bt || !alpha0 || !hext || nt_hext < 1) return fail(MT_ERR_ARG, "bad argument");
    if (solver != 1 && solver != 2) return fail(MT_ERR_UNSUPPORTED, "solver %d", solver);
    const int Bp = bt->IB * kInstBlock;
    std::vector<double> he((size_t)Bp * nt_hext * 4, 0.0), al(Bp, 1.0);
    memcpy(he.data(), hext, sizeof(double) * (size_t)bt->B * nt_hext * 4);
    memcpy(al.data(), alpha0, sizeof(double) * bt->B);
    free_ptr(bt->hext); bt->hext = nullptr;
    free_ptr(bt->alpha0); bt->alpha0 = nullptr;
    CUDA_TRY(dalloc(&bt->hext, he.size()));
    CUDA_TRY(dalloc(&bt->alpha0, al.size()));
    CUDA_TRY(cudaMemcpy(bt->hext, he.data(), sizeof(double) * he.size(), cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(bt->alpha0, al.data(), sizeof(double) * al.size(), cudaMemcpyHostToDevice));
    bt->nt_hext = nt_hext;
    bt->solver = solver; bt->gamma = gamma; bt->renorm = renormalize ? 1 : 0;
    int rc = batch_shared_dynamics(bt);
    if (rc) return rc;
    bt->have_dynamics = true;
    return MT_OK;
}

int mt_batch_set_alpha_table(mt_batch* bt, const double* alpha_tab, int nt_alpha)
{
    if (!bt || nt_alpha < 0 || (nt_alpha > 0 && !alpha_tab)) return fail(MT_ERR_ARG, "bad argument");
    bt->alpha_tab.assign(alpha_tab, alpha_tab + 2 * (size_t)nt_alpha);
    return bt->have_dynamics ? batch_shared_dynamics(bt) : MT_OK;
}

int mt_batch_assemble_demag(mt_batch* bt, void* stream)
{
    if (!bt) return fail(MT_ERR_ARG, "null handle");
    int rc = mt_assemble_demag(bt->h, stream);
    if (rc) return rc;
    if (bt->prec == MT_PREC_INT8) {
        const size_t cnt = (size_t)bt->Kd * bt->Kd;
        if (!bt->klimb) {
            CUDA_TRY(dalloc(&bt->klimb, 4 * cnt));
            CUDA_TRY(dalloc(&bt->row_scale, (size_t)bt->Kd));
        }
        CUDA_TRY(launch_limb_tensor(bt->h->K, bt->h->n, bt->h->ldk, bt->np, bt->klimb, bt->row_scale,
                                    (cudaStream_t)stream));
    } else if (bt->prec != MT_PREC_FP32) {
        const size_t cnt = (size_t)bt->Kd * bt->Kd;
        if (!bt->khi) {
            CUDA_TRY(dalloc(&bt->khi, 2 * cnt));   // hi and lo contiguous: one L2 persistence window
            bt->klo = bt->khi + cnt;
            CUDA_TRY(dalloc(&bt->row_inv, (size_t)bt->Kd));
        }
        CUDA_TRY(launch_split_tensor(bt->h->K, bt->h->n, bt->h->ldk, bt->np, bt->prec, bt->khi, bt->klo, bt->row_inv,
                                     (cudaStream_t)stream));
    }
    return MT_OK;
}

}  // extern "C"

namespace {

struct BatchRun {
    IntegAlloc A;
    BatchBufs F;
    BatchParams Q;
    TcMaps maps;
    double* comb = nullptr;   // merged output and convergence times, capacity comb_cap
    int* cflags = nullptr;
    size_t comb_cap = 0;
};

}  // namespace

static void batch_ws_free(mt_batch* bt)
{
    delete bt->ws;   // frees the device buffers (cudaFree synchronises with the device)
    bt->ws = nullptr;
    bt->ws_nt = -1;
}

namespace {

// smallest Stream-K CTA count the autotuner tries (the slot storage is sized for it)
int sk_min_ctas(int grid) { return std::max(1, (2 * grid) / 3); }

// The workspace of one integration (or demag) call: allocated on the first call and
// kept in the handle while nt is unchanged; every call re-initialises it.
int batch_alloc(mt_batch* bt, BatchRun*& Rp, int nt, cudaStream_t s)
{
    mt_handle* h = bt->h;
    const int n = h->n;
    const int Bp = bt->IB * kInstBlock;
    const size_t n3 = 3 * (size_t)n;
    const int RB0 = bt->Kd / 128, nks0 = bt->Kd / kI8KB;
    const int maxseg0 = bt->prec == MT_PREC_INT8 ? batch_i8_maxseg(RB0, nks0, Bp / kI8N, sk_min_ctas(bt->grid)) : 0;
    if (!bt->ws || bt->ws_nt != nt) {
        batch_ws_free(bt);
        std::unique_ptr<BatchRun> W(new BatchRun());
        BatchRun& R = *W;
        BatchBufs& F = R.F;
        memset(&F, 0, sizeof(F));
        CUDA_TRY(R.A.get(&F.pool, 4 * (size_t)Bp * n3));
        CUDA_TRY(R.A.get(&F.deriv, 3 * (size_t)Bp * n3));
        CUDA_TRY(R.A.get(&F.stg, 12 * (size_t)Bp * n3));
        CUDA_TRY(R.A.get(&F.p, 6 * (size_t)Bp * n3));
        CUDA_TRY(R.A.get(&F.errest, (size_t)Bp * n3));
        CUDA_TRY(R.A.get(&F.weights, (size_t)Bp * n3));
        CUDA_TRY(R.A.get(&F.ylast, (size_t)Bp * n3));
        CUDA_TRY(R.A.get(&F.ystep, (size_t)Bp * n3));
        if (nt > 0) {
            CUDA_TRY(R.A.get(&F.t_out, (size_t)Bp * nt));
            CUDA_TRY(R.A.get(&F.flags_out, (size_t)Bp * nt));
        }
        if (bt->prec == MT_PREC_FP32) {
            CUDA_TRY(R.A.get(&F.m32, (size_t)Bp * 3 * h->ldk));
        } else if (bt->prec == MT_PREC_INT8) {
            CUDA_TRY(R.A.get(&F.mlimb, 4 * (size_t)Bp * bt->Kd));
            CUDA_TRY(R.A.get(&F.mcomp, 4 * (size_t)Bp * bt->Kd));
            CUDA_TRY(R.A.get(&F.reqbits, 3 * (size_t)(Bp / 32)));
        } else {
            CUDA_TRY(R.A.get(&F.mhi, (size_t)Bp * bt->Kd));
            CUDA_TRY(R.A.get(&F.mlo, (size_t)Bp * bt->Kd));
        }
        if (bt->prec == MT_PREC_INT8)
            CUDA_TRY(R.A.get(&F.part, (size_t)bt->grid * maxseg0 * kI8SlotElems));
        else
            CUDA_TRY(R.A.get(&F.hpart, (size_t)bt->S * Bp * 3 * bt->np));
        CUDA_TRY(R.A.get(&F.partials, 2 * (size_t)Bp * kRedSlots * bt->CB));
        CUDA_TRY(R.A.get(&F.redcnt, (size_t)Bp));
        CUDA_TRY(R.A.get(&F.inst, (size_t)bt->CB * Bp));
        CUDA_TRY(R.A.get(&F.gs, 1));
        CUDA_TRY(R.A.get(&F.counters, 6));
        CUDA_TRY(R.A.get(&F.ibreq, 6 * (size_t)bt->IB));
        if (getenv("MT_BATCH_PROFILE")) CUDA_TRY(R.A.get(&F.prof, 48));
        bt->ws = W.release();
        bt->ws_nt = nt;
    }
    Rp = bt->ws;
    BatchRun& R = *Rp;
    BatchBufs& F = R.F;
    F.y_out = nullptr;
    CUDA_TRY(cudaMemsetAsync(F.pool, 0, sizeof(double) * 4 * (size_t)Bp * n3, s));
    if (nt > 0) {
        CUDA_TRY(cudaMemsetAsync(F.t_out, 0, sizeof(double) * Bp * nt, s));
        CUDA_TRY(cudaMemsetAsync(F.flags_out, 0, sizeof(int) * Bp * nt, s));
    }
    if (F.m32) CUDA_TRY(cudaMemsetAsync(F.m32, 0, sizeof(float) * Bp * 3 * (size_t)h->ldk, s));
    if (F.mlimb) {
        CUDA_TRY(cudaMemsetAsync(F.mlimb, 0, 4 * (size_t)Bp * bt->Kd, s));
        CUDA_TRY(cudaMemsetAsync(F.mcomp, 0, 4 * (size_t)Bp * bt->Kd, s));
        CUDA_TRY(cudaMemsetAsync(F.reqbits, 0, sizeof(unsigned) * 3 * (Bp / 32), s));
    }
    if (F.mhi) {
        CUDA_TRY(cudaMemsetAsync(F.mhi, 0, 2 * (size_t)Bp * bt->Kd, s));
        CUDA_TRY(cudaMemsetAsync(F.mlo, 0, 2 * (size_t)Bp * bt->Kd, s));
    }
    CUDA_TRY(cudaMemsetAsync(F.counters, 0, sizeof(unsigned) * 6, s));
    CUDA_TRY(cudaMemsetAsync(F.ibreq, 0, sizeof(unsigned) * 6 * bt->IB, s));
    if (F.prof) CUDA_TRY(cudaMemsetAsync(F.prof, 0, sizeof(unsigned long long) * 48, s));
    const int RB = RB0, nks = nks0, maxseg = maxseg0;
    F.hext = bt->hext;
    F.alpha0 = bt->alpha0;
    BatchParams& Q = R.Q;
    memset(&Q, 0, sizeof(Q));
    Q.Bp = Bp; Q.B = bt->B; Q.CB = bt->CB; Q.IB = bt->IB; Q.S = bt->S; Q.np = bt->np; Q.Kd = bt->Kd;
    Q.nt = nt; Q.nt_hext = bt->nt_hext; Q.prec = bt->prec;
    Q.khi = bt->khi; Q.klo = bt->klo; Q.row_inv = bt->row_inv;
    Q.RB = RB; Q.nks = nks; Q.maxseg = maxseg; Q.row_scale = bt->row_scale;
    for (int k = 0; k <= 2 * kMaxIB; ++k) Q.sk_sched[k] = bt->sched[k];
    Q.renorm = h->renorm;
    if (!getenv("MT_BATCH_LOCAL_INST"))
        Q.inst_smem_bytes = batch_inst_smem(n, h->ldk, bt->prec, kInstBlock / bt->S, &Q.inst_smem_off, &Q.inst_per_warp);
    memset(&R.maps, 0, sizeof(R.maps));
    if (bt->prec == MT_PREC_INT8) {
        int rc;
        if ((rc = make_tmap_i8(&R.maps.ahi, bt->klimb, bt->Kd, bt->Kd, 4, 128))) return rc;
        if ((rc = make_tmap_i8(&R.maps.bhi, F.mlimb, bt->Kd, Bp, 4, kI8N))) return rc;
        if ((rc = make_tmap_i8(&R.maps.blo, F.mcomp, bt->Kd, Bp, 4, kI8N))) return rc;
    } else if (bt->prec != MT_PREC_FP32) {
        int rc;
        if ((rc = make_tmap(&R.maps.ahi, bt->khi, bt->Kd, bt->Kd, 128))) return rc;
        if ((rc = make_tmap(&R.maps.alo, bt->klo, bt->Kd, bt->Kd, 128))) return rc;
        if ((rc = make_tmap(&R.maps.bhi, F.mhi, bt->Kd, Bp, kTcN))) return rc;
        if ((rc = make_tmap(&R.maps.blo, F.mlo, bt->Kd, Bp, kTcN))) return rc;
    }
    return MT_OK;
}

}  // namespace

extern "C" {

// Autotuner of the int8 Stream-K GEMM.  For every count of active 64-instance tiles,
// times the product alone (one launch of the batch kernel in schedule-timing mode,
// CUDA events, best of three after a warm-up) for each candidate schedule: Stream-K CTA
// counts from all SMs down to two thirds of them in steps of 8, in tile-major and
// row-major unit order; keeps the fastest.  The exact product gives the same bits
// under every schedule.  Results are kept per device, grid and batch size for the
// life of the process.
namespace {
std::mutex g_tune_mu;
std::map<std::string, std::vector<int>> g_tune_cache;
}

int mt_batch_tune(mt_batch* bt, void* stream)
{
    if (!bt) return fail(MT_ERR_ARG, "null handle");
    if (bt->prec != MT_PREC_INT8) return MT_OK;   // the other precisions run fixed tiles
    if (!bt->klimb) return fail(MT_ERR_STATE, "call mt_batch_assemble_demag first");
    cudaStream_t s = (cudaStream_t)stream;
    const int JB = (bt->IB * kInstBlock) / kI8N;
    char key[128];
    snprintf(key, sizeof(key), "dev%d sms%d n%d Kd%d Bp%d grid%d", bt->h->device, bt->h->num_sms, bt->h->n, bt->Kd,
             bt->IB * kInstBlock, bt->grid);
    {
        std::lock_guard<std::mutex> lock(g_tune_mu);
        auto it = g_tune_cache.find(key);
        if (it != g_tune_cache.end()) { bt->sched = it->second; bt->tuned = true; return MT_OK; }
    }
    BatchRun* Rp = nullptr;
    int rc = batch_alloc(bt, Rp, 0, s);
    if (rc) return rc;
    BatchRun& R = *Rp;
    DevProb P = batch_prob(bt);
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    CUDA_TRY(cudaEventCreate(&ev0));
    CUDA_TRY(cudaEventCreate(&ev1));
    struct EvGuard { cudaEvent_t a, b; ~EvGuard() { cudaEventDestroy(a); cudaEventDestroy(b); } } evg{ev0, ev1};
    std::vector<int> cands;
    for (int G = bt->grid; G >= sk_min_ctas(bt->grid); G -= 8) cands.push_back(G);
    std::vector<int> sched(2 * kMaxIB + 1, bt->grid);
    R.Q.demag_only = 1;
    for (int nact = 1; nact <= JB; ++nact) {
        float best = 1e30f;
        int best_w = bt->grid;
        for (int order = 0; order < 2; ++order)
            for (int G : cands) {
                const int w = G | (order << 16);
                R.Q.tune_nact = nact;
                R.Q.tune_sched = w;
                float t_min = 1e30f;
                for (int rep = 0; rep < 4; ++rep) {
                    CUDA_TRY(cudaMemsetAsync(R.F.gs, 0, sizeof(GridSync), s));
                    CUDA_TRY(cudaEventRecord(ev0, s));
                    CUDA_TRY(launch_batch(P, R.F, R.Q, bt->grid, &R.maps, s));
                    CUDA_TRY(cudaEventRecord(ev1, s));
                    CUDA_TRY(cudaEventSynchronize(ev1));
                    float ms = 0.f;
                    CUDA_TRY(cudaEventElapsedTime(&ms, ev0, ev1));
                    if (rep > 0) t_min = std::min(t_min, ms);
                }
                GridSync gs_h;
                CUDA_TRY(cudaMemcpy(&gs_h, R.F.gs, sizeof(gs_h), cudaMemcpyDeviceToHost));
                if (gs_h.err || gs_h.abort)
                    return fail(MT_ERR_TIMEOUT, "schedule timing: bounded wait gave up (at %d)", gs_h.err_where);
                if (t_min < best) { best = t_min; best_w = w; }
            }
        sched[nact] = best_w;
    }
    bt->sched = sched;
    bt->tuned = true;
    std::lock_guard<std::mutex> lock(g_tune_mu);
    g_tune_cache[key] = sched;
    return MT_OK;
}

int mt_batch_set_schedule(mt_batch* bt, const int* ctas, const int* order, int n_tiles)
{
    if (!bt || !ctas || !order) return fail(MT_ERR_ARG, "bad argument");
    const int JB = (bt->IB * kInstBlock) / kI8N;
    if (n_tiles != JB) return fail(MT_ERR_ARG, "need one entry per tile count (%d)", JB);
    std::vector<int> sched(2 * kMaxIB + 1, bt->grid);
    for (int k = 1; k <= JB; ++k) {
        const int G = ctas[k - 1], o = order[k - 1];
        if (G < sk_min_ctas(bt->grid) || G > bt->grid || (o != 0 && o != 1))
            return fail(MT_ERR_ARG, "schedule %d: %d CTAs (allowed %d..%d), order %d", k, G, sk_min_ctas(bt->grid),
                        bt->grid, o);
        sched[k] = G | (o << 16);
    }
    bt->sched = sched;
    return MT_OK;
}

int mt_batch_get_schedule(mt_batch* bt, int* ctas, int* order, int max_tiles, int* n_tiles)
{
    if (!bt || !n_tiles) return fail(MT_ERR_ARG, "bad argument");
    const int JB = (bt->IB * kInstBlock) / kI8N;
    *n_tiles = JB;
    for (int k = 1; k <= JB && k <= max_tiles; ++k) {
        if (ctas) ctas[k - 1] = bt->sched[k] & 0xffff;
        if (order) order[k - 1] = (bt->sched[k] >> 16) & 1;
    }
    return MT_OK;
}

static int batch_integrate(mt_batch* bt, const double* t, int nt, const double* m0_dev, double tol, double thres,
                           const double* t_conv, int nt_conv, double conv_tol, double* t_out, double* y_out_dev,
                           double* y_out_host, int* flags, mt_stats* stats, void* stream);

int mt_batch_integrate(mt_batch* bt, const double* t, int nt, const double* m0_dev, double tol, double thres,
                       const double* t_conv, int nt_conv, double conv_tol, double* t_out, double* y_out_dev,
                       int* flags, mt_stats* stats, void* stream)
{
    return batch_integrate(bt, t, nt, m0_dev, tol, thres, t_conv, nt_conv, conv_tol, t_out, y_out_dev, nullptr, flags,
                           stats, stream);
}

int mt_batch_integrate_host(mt_batch* bt, const double* t, int nt, const double* m0_dev, double tol, double thres,
                            const double* t_conv, int nt_conv, double conv_tol, double* t_out, double* y_out_dev,
                            double* y_out_host, int* flags, mt_stats* stats, void* stream)
{
    if (!y_out_dev || !y_out_host) return fail(MT_ERR_ARG, "y_out_dev and y_out_host are required");
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, y_out_host) != cudaSuccess || a.type != cudaMemoryTypeHost) {
        cudaGetLastError();
        return fail(MT_ERR_ARG, "y_out_host must be page-locked host memory (cudaHostAlloc / pinned)");
    }
    return batch_integrate(bt, t, nt, m0_dev, tol, thres, t_conv, nt_conv, conv_tol, t_out, y_out_dev, y_out_host,
                           flags, stats, stream);
}

int mt_batch_demag_field(mt_batch* bt, const double* m_dev, double* H_dev, void* stream)
{
    if (!bt || !m_dev || !H_dev) return fail(MT_ERR_ARG, "bad argument");
    int rc = check_ready(bt->h, true, false);
    if (rc) return rc;
    if (bt->prec != MT_PREC_FP32 && !bt->khi && !bt->klimb) return fail(MT_ERR_STATE, "call mt_batch_assemble_demag first");
    cudaStream_t s = (cudaStream_t)stream;
    BatchRun* Rp = nullptr;
    if ((rc = batch_alloc(bt, Rp, 0, s))) return rc;
    BatchRun& R = *Rp;
    R.Q.demag_only = 1;
    R.Q.out_h = H_dev;
    CUDA_TRY(cudaMemsetAsync(R.F.gs, 0, sizeof(GridSync), s));
    CUDA_TRY(launch_batch_operand(m_dev, bt->B, bt->h->n, bt->h->ldk, bt->np, bt->prec, R.F.m32, R.F.mhi, R.F.mlo,
                                  R.F.mlimb, R.Q.Bp, R.F.gs, s));
    DevProb P = batch_prob(bt);
    CUDA_TRY(launch_batch(P, R.F, R.Q, bt->grid, bt->prec != MT_PREC_FP32 ? &R.maps : nullptr, s));
    GridSync gs_h;
    CUDA_TRY(cudaMemcpyAsync(&gs_h, R.F.gs, sizeof(gs_h), cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    if (gs_h.err == KERR_RANGE) return fail(MT_ERR_ARG, "int8 precision: a component of m is outside (-1.96, 1.96)");
    if (gs_h.err || gs_h.abort) return fail(MT_ERR_TIMEOUT, "batch demag: bounded wait gave up (at %d)", gs_h.err_where);
    return MT_OK;
}

// y_out_host (page-locked, [B][nt][3n], or nullptr): the samples every instance has
// finished are copied there after each launch, on a stream of their own, while the next
// launch runs; the rest after the last launch.
static int batch_integrate(mt_batch* bt, const double* t, int nt, const double* m0_dev, double tol, double thres,
                           const double* t_conv, int nt_conv, double conv_tol, double* t_out, double* y_out_dev,
                           double* y_out_host, int* flags, mt_stats* stats, void* stream)
{
    if (!bt) return fail(MT_ERR_ARG, "null handle");
    int rc = check_ready(bt->h, true, false);
    if (rc) return rc;
    if (!bt->have_dynamics) return fail(MT_ERR_STATE, "call mt_batch_set_dynamics first");
    if (bt->prec != MT_PREC_FP32 && !bt->khi && !bt->klimb) return fail(MT_ERR_STATE, "call mt_batch_assemble_demag first");
    if (!t || nt < 2 || !m0_dev || !t_out || !flags || !stats) return fail(MT_ERR_ARG, "bad argument (nt >= 2 required)");
    if (nt_conv < 0 || (nt_conv > 0 && !t_conv)) return fail(MT_ERR_ARG, "bad convergence-time list");
    cudaStream_t s = (cudaStream_t)stream;
    mt_handle* h = bt->h;
    const int n = h->n, B = bt->B;
    const size_t n3 = 3 * (size_t)n;
    for (int b = 0; b < B; ++b) { memset(&stats[b], 0, sizeof(mt_stats)); stats[b].converged_at = -1; }
    cudaCtxResetPersistingL2Cache();   // no tensor lines of an earlier single-instance field call stay kept in L2
    const double eps = 2.220446049250313e-16;
    const double round_off = 10.0 * eps, sqrrmc = sqrt(eps), cubrmc = pow(eps, 1.0 / 3.0);
    const double sqtiny = sqrt(2.2250738585072014e-308);
    const double toosml = round_off / (1.0 / 18.0);
    const double t_start = t[0], t_end = t[nt - 1];
    if (t_start == t_end) return fail(MT_ERR_ARG, "T_START = T_END");
    if (tol > 0.01 || tol < round_off) return fail(MT_ERR_ARG, "tol %g outside (%g, 0.01)", tol, round_off);
    if (thres < sqtiny) return fail(MT_ERR_ARG, "threshold %g below %g", thres, sqtiny);
    const double hmin0 = std::max(sqtiny, toosml * std::max(fabs(t_start), fabs(t_end)));
    if (fabs(t_end - t_start) < hmin0) return fail(MT_ERR_ARG, "T_END and T_START not distinguishable");
    std::vector<double> comb;
    for (int i = 0; i < nt + nt_conv; ++i) {
        const double v = (i < nt) ? t[i] : t_conv[i - nt];
        bool dup = (i > 0 && v == 0.0);
        for (double c : comb) if (c == v) { dup = true; break; }
        if (i == 0 || !dup) comb.push_back(v);
    }
    std::sort(comb.begin(), comb.end());
    std::vector<int> cflags(comb.size(), 0);
    for (size_t k = 0; k < comb.size(); ++k) {
        for (int q = 0; q < nt; ++q) if (t[q] == comb[k]) { cflags[k] |= 1; break; }
        for (int q = 0; q < nt_conv; ++q) if (t_conv[q] == comb[k]) { cflags[k] |= 2; break; }
    }
    BatchRun* Rp = nullptr;
    if ((rc = batch_alloc(bt, Rp, nt, s))) return rc;
    BatchRun& R = *Rp;
    BatchBufs& F = R.F;
    BatchParams& Q = R.Q;
    const int Bp = Q.Bp;
    if (comb.size() > R.comb_cap) {
        CUDA_TRY(R.A.get(&R.comb, comb.size()));
        CUDA_TRY(R.A.get(&R.cflags, comb.size()));
        R.comb_cap = comb.size();
    }
    double* d_comb = R.comb;
    int* d_cflags = R.cflags;
    CUDA_TRY(cudaMemcpyAsync(d_comb, comb.data(), sizeof(double) * comb.size(), cudaMemcpyHostToDevice, s));
    CUDA_TRY(cudaMemcpyAsync(d_cflags, cflags.data(), sizeof(int) * comb.size(), cudaMemcpyHostToDevice, s));
    F.y_out = y_out_dev;
    // y <- m0 (pool slot 0 of every instance), first sample, convergence reference
    CUDA_TRY(cudaMemcpyAsync(F.pool, m0_dev, sizeof(double) * (size_t)B * n3, cudaMemcpyDeviceToDevice, s));
    CUDA_TRY(cudaMemcpyAsync(F.ylast, m0_dev, sizeof(double) * (size_t)B * n3, cudaMemcpyDeviceToDevice, s));
    if (y_out_dev)   // first sample of every instance: rows nt * 3n apart
        CUDA_TRY(cudaMemcpy2DAsync(y_out_dev, sizeof(double) * nt * n3, m0_dev, sizeof(double) * n3,
                                   sizeof(double) * n3, B, cudaMemcpyDeviceToDevice, s));
    std::vector<BInst> init((size_t)bt->CB * Bp);
    for (int cb = 0; cb < bt->CB; ++cb)
        for (int b = 0; b < Bp; ++b) {
            BInst& I = init[(size_t)cb * Bp + b];
            memset(&I, 0, sizeof(I));
            RKS& st = I.s;
            st.t = t_start; st.t_old = t_start; st.t_start = t_start; st.t_end = t_end;
            st.dir = (t_end - t_start) >= 0 ? 1.0 : -1.0;
            st.tol = tol;
            st.h = std::max(fabs(t_end - t_start) / 8.0, hmin0);
            st.at_t_start = 1; st.phase2 = 1;
            st.iy = 0; st.iyold = 1; st.ia0 = 2; st.ia1 = 3;
            st.dyp = 0; st.dypold = 1; st.d8 = 2;
            st.ci = 1; st.ko = 1;
            st.converged_at = -1;
            I.pc = 0;
            I.req = (b < B) ? 0 : 3;
        }
    CUDA_TRY(cudaMemcpyAsync(F.inst, init.data(), sizeof(BInst) * init.size(), cudaMemcpyHostToDevice, s));
    Q.thres = thres; Q.round_off = round_off; Q.sqrrmc = sqrrmc; Q.cubrmc = cubrmc; Q.sqtiny = sqtiny;
    Q.toosml = toosml; Q.conv_tol = conv_tol;
    Q.comb_t = d_comb; Q.comb_flags = d_cflags; Q.ncomb = (int)comb.size();
    // ticks per launch: 4000 (about a second at the 256-instance film); MT_BATCH_TICKS sets
    // it, for example to profile one short launch
    Q.ticks_per_launch = 4000;
    if (const char* e = getenv("MT_BATCH_TICKS")) {
        const long long v = atoll(e);
        if (v >= 1 && v <= 1000000) Q.ticks_per_launch = v;
    }
    Q.evals_budget = 1LL << 60;
    DevProb P = batch_prob(bt);
    const size_t smem = batch_smem_bytes(n, h->ldk, bt->prec) + Q.inst_smem_bytes;
    if (smem > 227 * 1024) return fail(MT_ERR_UNSUPPORTED, "batch shared memory %zu exceeds 227 KB", smem);
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    CUDA_TRY(cudaEventCreate(&ev0));
    CUDA_TRY(cudaEventCreate(&ev1));
    struct EvGuard { cudaEvent_t a, b; ~EvGuard() { cudaEventDestroy(a); cudaEventDestroy(b); } } evg{ev0, ev1};
    double kernel_ms = 0.0;
    long long launches = 0;
    std::vector<BInst> hs(Bp);
    // L2 residency of the split tensor (process-local limit, restored on return)
    size_t l2_bytes = 0;
    float l2_hit = 0.f;
    size_t prev_limit = 0;
    bool limit_set = false;
    // Opt-in L2 residency of the split tensor (MT_L2_PERSIST=1).  Off by default: for the
    // int8 tensor the per-instance FP64 state gains more from L2 than the tensor does
    // (measured 57.9 against 55.6 simulated ns/s on the 256-instance film batch).
    if (bt->prec != MT_PREC_FP32 && getenv("MT_L2_PERSIST")) {
        int max_persist = 0, max_win = 0;
        cudaDeviceGetAttribute(&max_persist, cudaDevAttrMaxPersistingL2CacheSize, h->device);
        cudaDeviceGetAttribute(&max_win, cudaDevAttrMaxAccessPolicyWindowSize, h->device);
        const size_t want = 4 * (size_t)bt->Kd * bt->Kd;
        if (max_persist > 0 && max_win > 0 && cudaDeviceGetLimit(&prev_limit, cudaLimitPersistingL2CacheSize) == cudaSuccess) {
            const size_t lim = std::min(want, (size_t)max_persist);
            if (cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, lim) == cudaSuccess) {
                limit_set = true;
                l2_bytes = std::min(want, (size_t)max_win);
                l2_hit = (float)std::min(1.0, (double)lim / (double)l2_bytes);
            }
        }
        cudaGetLastError();
    }
    struct L2Guard {
        bool on; size_t prev;
        ~L2Guard() { if (on) { cudaCtxResetPersistingL2Cache(); cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, prev); } }
    } l2g{limit_set, prev_limit};
    long long last_sig = -1;
    // streamed read-back of finished samples (y_out_host)
    cudaStream_t cs2 = nullptr;
    if (y_out_host) CUDA_TRY(cudaStreamCreateWithFlags(&cs2, cudaStreamNonBlocking));
    struct CopyStream {
        cudaStream_t s;
        ~CopyStream() { if (s) { cudaStreamSynchronize(s); cudaStreamDestroy(s); } }
    } csg{cs2};
    int k_sent = 0;   // samples 0 .. k_sent - 1 of every instance are on their way to the host
    const size_t row = n3 * sizeof(double), pitch = (size_t)nt * row;
    auto send = [&](int k_to) -> cudaError_t {
        if (!y_out_host || k_to <= k_sent) return cudaSuccess;
        cudaError_t e = cudaMemcpy2DAsync(y_out_host + (size_t)k_sent * n3, pitch, y_out_dev + (size_t)k_sent * n3, pitch,
                                          (size_t)(k_to - k_sent) * row, (size_t)B, cudaMemcpyDeviceToHost, cs2);
        if (e == cudaSuccess) k_sent = k_to;
        return e;
    };
    for (;;) {
        CUDA_TRY(cudaMemsetAsync(F.gs, 0, sizeof(GridSync), s));
        CUDA_TRY(cudaMemsetAsync(F.counters, 0, sizeof(unsigned) * 6, s));
        CUDA_TRY(cudaMemsetAsync(F.ibreq, 0, sizeof(unsigned) * 6 * bt->IB, s));
        CUDA_TRY(cudaMemsetAsync(F.redcnt, 0, sizeof(unsigned) * Q.Bp, s));
        if (F.reqbits) CUDA_TRY(cudaMemsetAsync(F.reqbits, 0, sizeof(unsigned) * 3 * (Q.Bp / 32), s));
        CUDA_TRY(cudaEventRecord(ev0, s));
        CUDA_TRY(launch_batch(P, F, Q, bt->grid, bt->prec != MT_PREC_FP32 ? &R.maps : nullptr, s,
                              l2_bytes ? (bt->prec == MT_PREC_INT8 ? (const void*)bt->klimb : (const void*)bt->khi)
                                       : nullptr,
                              l2_bytes, l2_hit));
        CUDA_TRY(cudaEventRecord(ev1, s));
        GridSync gs_h;
        CUDA_TRY(cudaMemcpyAsync(&gs_h, F.gs, sizeof(gs_h), cudaMemcpyDeviceToHost, s));
        CUDA_TRY(cudaMemcpyAsync(hs.data(), F.inst, sizeof(BInst) * Bp, cudaMemcpyDeviceToHost, s));
        CUDA_TRY(cudaStreamSynchronize(s));
        float ms = 0.f;
        CUDA_TRY(cudaEventElapsedTime(&ms, ev0, ev1));
        kernel_ms += ms;
        launches++;
        if (gs_h.err == KERR_RANGE)
            return fail(MT_ERR_ARG, "int8 precision: a component of m left (-1.96, 1.96)");
        if (gs_h.err != 0 || gs_h.abort)
            return fail(MT_ERR_TIMEOUT, "batch integrator: bounded wait gave up (code %d at %d)", gs_h.err, gs_h.err_where);
        bool all_done = true;
        long long sig = 0;
        for (int b = 0; b < B; ++b) {
            if (hs[b].req != 3) all_done = false;
            sig += hs[b].s.full_f_count + hs[b].s.f_count + hs[b].s.ci;
        }
        if (all_done) break;
        if (sig == last_sig) return fail(MT_ERR_SOLVER, "batch integrator made no progress");
        last_sig = sig;
        if (y_out_host) {   // samples below every unfinished instance's output index are final
            int k_done = nt;
            for (int b = 0; b < B; ++b)
                if (hs[b].req != 3) k_done = std::min(k_done, hs[b].s.ko);
            CUDA_TRY(send(k_done));
        }
    }
    if (y_out_host) {
        CUDA_TRY(send(nt));
        CUDA_TRY(cudaStreamSynchronize(cs2));
    }
    std::vector<int> fl((size_t)Bp * nt);
    std::vector<double> to((size_t)Bp * nt);
    CUDA_TRY(cudaMemcpy(to.data(), F.t_out, sizeof(double) * to.size(), cudaMemcpyDeviceToHost));
    CUDA_TRY(cudaMemcpy(fl.data(), F.flags_out, sizeof(int) * fl.size(), cudaMemcpyDeviceToHost));
    int worst = 0;
    for (int b = 0; b < B; ++b) {
        memcpy(t_out + (size_t)b * nt, to.data() + (size_t)b * nt, sizeof(double) * nt);
        memcpy(flags + (size_t)b * nt, fl.data() + (size_t)b * nt, sizeof(int) * nt);
        t_out[(size_t)b * nt] = t[0];
        flags[(size_t)b * nt] = 0;
        const RKS& st = hs[b].s;
        stats[b].f_evals = st.full_f_count + st.f_count;
        stats[b].steps = st.step_count;
        stats[b].bad_steps = st.bad_step_count;
        stats[b].n_flag3 = st.n_flag3;
        stats[b].n_flag4 = st.n_flag4;
        stats[b].n_out = st.ko;
        stats[b].status = st.status;
        stats[b].converged_at = st.converged_at;
        if (st.status) worst = st.status;
    }
    stats[0].launches = launches;
    stats[0].kernel_ms = kernel_ms;
    if (F.prof) {
        unsigned long long pr[48];
        CUDA_TRY(cudaMemcpy(pr, F.prof, sizeof(pr), cudaMemcpyDeviceToHost));
        if (bt->prec == MT_PREC_INT8) {
            fprintf(stderr, "[batch profile] ticks by active 64-instance tiles (count, mean us):");
            for (int k = 0; k < 5; ++k)
                fprintf(stderr, " %d%s: %llu, %.1f;", k, k == 4 ? "+" : "", pr[37 + k],
                        pr[37 + k] ? pr[32 + k] / 1e3 / pr[37 + k] : 0.0);
            fprintf(stderr, "\n");
        }
        const double tk = pr[7] ? (double)pr[7] : 1.0;
        fprintf(stderr, "[batch profile] ticks %llu  per tick (us) at CTA 0: start %.2f B1 %.2f GEMM %.2f Bh %.2f "
                "P1 epilogue %.2f advance+publish %.2f  busiest CTA: GEMM %.2f (cta %llu) P1 advance %.2f (cta %llu)\n",
                pr[7], pr[0] / tk / 1e3, pr[1] / tk / 1e3, pr[2] / tk / 1e3, pr[3] / tk / 1e3, pr[6] / tk / 1e3,
                pr[4] / tk / 1e3, pr[9] / tk / 1e3, pr[13], pr[10] / tk / 1e3, pr[14]);
        if (bt->prec == MT_PREC_INT8)
            fprintf(stderr, "[batch profile] int8 GEMM at CTA 0 per tick (us): roles done %.2f, total %.2f; MMA waits "
                    "full %.2f tfree %.2f; epilogue waits %.2f drains %.2f; producer waits %.2f; units %.1f segments %.2f\n",
                    pr[23] / tk / 1e3, pr[24] / tk / 1e3, pr[16] / tk / 1e3, pr[17] / tk / 1e3, pr[18] / tk / 1e3,
                    pr[19] / tk / 1e3, pr[20] / tk / 1e3, pr[21] / tk, pr[22] / tk);
        fprintf(stderr, "[batch profile] CTA 0 warp 0: advance %.2f us per call (%llu calls), stage-argument loop "
                "%.2f us per call (%llu calls)\n", pr[28] ? pr[27] / 1e3 / pr[28] : 0.0, pr[28],
                pr[26] ? pr[25] / 1e3 / pr[26] : 0.0, pr[26]);
    }
    if (worst) return fail(MT_ERR_SOLVER, "an instance stopped with RKSUITE flag %d", worst);
    return MT_OK;
}

// ---------------------------------------------------------------------------
// reference compatibility shims (one process-wide problem)
// ---------------------------------------------------------------------------
static mt_handle* g_icl = nullptr;

int icl_initDemagMatrices(const float* Kxx, const float* Kxy, const float* Kxz, const float* Kyy, const float* Kyz,
                          const float* Kzz, int* n)
{
    if (!n || *n < 1) return fail(MT_ERR_ARG, "n must be >= 1");
    if (g_icl) { mt_destroy(g_icl); g_icl = nullptr; }
    mt_grid g = {*n, 1, 1, 1.0, 1.0, 1.0};
    int rc = mt_create(&g, &g_icl);
    if (rc) return rc;
    rc = mt_load_demag_colmajor(g_icl, Kxx, Kxy, Kxz, Kyy, Kyz, Kzz);
    if (rc) { mt_destroy(g_icl); g_icl = nullptr; }
    return rc;
}

int icl_MVMult_GetH(const float* Mx, const float* My, const float* Mz, float* Hx, float* Hy, float* Hz, int* n,
                    float* pref)
{
    if (!g_icl) return fail(MT_ERR_STATE, "icl_initDemagMatrices has not been called");
    if (!n || *n != g_icl->n || !pref || !Mx || !My || !Mz || !Hx || !Hy || !Hz) return fail(MT_ERR_ARG, "bad argument");
    mt_handle* h = g_icl;
    const int nn = h->n;
    int rc = ensure_m32(h);
    if (rc) return rc;
    IntegAlloc A;
    float *dm = nullptr, *dh = nullptr;
    CUDA_TRY(A.get(&dm, 3 * (size_t)nn));
    CUDA_TRY(A.get(&dh, 3 * (size_t)nn));
    CUDA_TRY(cudaMemcpy(dm, Mx, sizeof(float) * nn, cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(dm + nn, My, sizeof(float) * nn, cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(dm + 2 * nn, Mz, sizeof(float) * nn, cudaMemcpyHostToDevice));
    CUDA_TRY(launch_pack3_f32(dm, dm + nn, dm + 2 * nn, nn, h->ldk, h->m32, 0));
    DevProb P = make_prob(h);
    CUDA_TRY(launch_field(3, P, nullptr, h->m32, 0.0, nullptr, nullptr, nullptr, nullptr, dh, *pref, h->num_sms, 0));
    CUDA_TRY(cudaMemcpy(Hx, dh, sizeof(float) * nn, cudaMemcpyDeviceToHost));
    CUDA_TRY(cudaMemcpy(Hy, dh + nn, sizeof(float) * nn, cudaMemcpyDeviceToHost));
    CUDA_TRY(cudaMemcpy(Hz, dh + 2 * nn, sizeof(float) * nn, cudaMemcpyDeviceToHost));
    return MT_OK;
}

int icl_destroy(void)
{
    if (g_icl) { mt_destroy(g_icl); g_icl = nullptr; }
    return MT_OK;
}

// The six block matrices of the sparse shims (1-based CSR, rowInds[n] = nnz + rowInds[0]),
// kept on the host until all six have arrived, then merged into the receiver-row CSR.
namespace {
struct IclSparse {
    int n = 0;
    bool have[6] = {false, false, false, false, false, false};
    std::vector<int> rows[6], cols[6];
    std::vector<float> vals[6];
};
IclSparse g_icl_sp;
}

int icl_initDemagMatrices_sparse(int* n, int* nnz, int* mat_no, float* values, int* colInds, int* rowInds)
{
    if (!n || !nnz || !mat_no || *n < 1 || *nnz < 0 || *mat_no < 1 || *mat_no > 6 || !rowInds ||
        (*nnz > 0 && (!values || !colInds)))
        return fail(MT_ERR_ARG, "bad argument");
    IclSparse& S = g_icl_sp;
    if (S.n != *n) { S = IclSparse(); S.n = *n; }
    const int k = *mat_no - 1, nn = *n, base = rowInds[0];
    if (rowInds[nn] - base != *nnz) return fail(MT_ERR_ARG, "rowInds[n] - rowInds[0] must equal nnz");
    S.rows[k].assign(rowInds, rowInds + nn + 1);
    for (int& r : S.rows[k]) r -= base;
    S.cols[k].resize(*nnz);
    for (int e = 0; e < *nnz; ++e) {
        S.cols[k][e] = colInds[e] - 1;
        if (S.cols[k][e] < 0 || S.cols[k][e] >= nn) return fail(MT_ERR_ARG, "column index %d outside 1..n", colInds[e]);
    }
    S.vals[k].assign(values, values + *nnz);
    S.have[k] = true;
    for (int c = 0; c < 6; ++c) if (!S.have[c]) return MT_OK;
    // all six blocks present: one problem with the merged receiver-row CSR
    if (g_icl) { mt_destroy(g_icl); g_icl = nullptr; }
    mt_grid g = {nn, 1, 1, 1.0, 1.0, 1.0};
    int rc = mt_create(&g, &g_icl);
    if (rc) return rc;
    mt_handle* h = g_icl;
    static const int blk[3][3] = {{0, 1, 2}, {1, 3, 4}, {2, 4, 5}};
    std::vector<int> rowptr(3 * (size_t)nn + 1), col;
    std::vector<float> val;
    for (int i = 0; i < nn; ++i)
        for (int a = 0; a < 3; ++a) {
            rowptr[3 * i + a] = (int)col.size();
            for (int b = 0; b < 3; ++b) {
                const int c = blk[a][b];
                for (int e = S.rows[c][i]; e < S.rows[c][i + 1]; ++e) {
                    col.push_back(b * h->ldk + S.cols[c][e]);
                    val.push_back(S.vals[c][e]);
                }
            }
        }
    rowptr[3 * (size_t)nn] = (int)col.size();
    const size_t nz = std::max<size_t>(col.size(), 1);
    CUDA_TRY(dalloc(&h->sp_rowptr, rowptr.size()));
    CUDA_TRY(dalloc(&h->sp_col, nz));
    CUDA_TRY(dalloc(&h->sp_val, nz));
    CUDA_TRY(cudaMemcpy(h->sp_rowptr, rowptr.data(), sizeof(int) * rowptr.size(), cudaMemcpyHostToDevice));
    if (!col.empty()) {
        CUDA_TRY(cudaMemcpy(h->sp_col, col.data(), sizeof(int) * col.size(), cudaMemcpyHostToDevice));
        CUDA_TRY(cudaMemcpy(h->sp_val, val.data(), sizeof(float) * val.size(), cudaMemcpyHostToDevice));
    }
    h->sp_nnz = (long long)col.size();
    h->have_K = true;   // the product runs on the sparse rows; no dense tensor is kept
    return MT_OK;
}

int icl_MVMult_GetH_sparse(const float* Mx, const float* My, const float* Mz, float* Hx, float* Hy, float* Hz,
                           const int* n, const float* pref)
{
    if (!g_icl || !g_icl->sp_rowptr) return fail(MT_ERR_STATE, "icl_initDemagMatrices_sparse has not received all six blocks");
    return icl_MVMult_GetH(Mx, My, Mz, Hx, Hy, Hz, const_cast<int*>(n), const_cast<float*>(pref));
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free right-hand side
// ---------------------------------------------------------------------------
// mt_rhs keeps an FP32 copy of m for the demag product in memory it allocates
// on first use.  Some callers may not allocate device memory at all: host
// frameworks that hand out all device memory from their own pool, or host
// programs and control loops whose device-memory budget is fixed once they have
// started and must never touch the allocator again.  For them the same copy lives in this fixed array instead,
// reserved once when the library loads and held by every GPU that loads it
// until the process exits.  Its size fixes the largest grid this entry point
// accepts.
static __device__ __align__(256) float g_noalloc_m32[3 * MT_NOALLOC_MAX_CELLS];

namespace {

std::mutex g_noalloc_mu;
float* g_noalloc_ptr[256] = {nullptr};   // device address of g_noalloc_m32, per device ordinal

// Looked up once per device, with that device current.  In host code the
// array's name is only a host-side stand-in; kernels must get this address.
int noalloc_scratch(int dev, float** out)
{
    if (dev < 0 || dev >= 256) return fail(MT_ERR_ARG, "device ordinal %d out of range", dev);
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        float* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress((void**)&p, g_noalloc_m32);
        if (e != cudaSuccess || !p)
            return fail(MT_ERR_CUDA, "cudaGetSymbolAddress(g_noalloc_m32) on device %d: %s", dev, cudaGetErrorString(e));
        g_noalloc_ptr[dev] = p;
    }
    *out = g_noalloc_ptr[dev];
    return MT_OK;
}

}  // namespace

extern "C" int mt_rhs_noalloc(mt_handle* h, double t, const double* m_dev, double* dmdt_dev, void* stream)
{
    if (!h) return fail(MT_ERR_ARG, "null handle");
    if (int rc = refuse_sharded(h, "mt_rhs_noalloc")) return rc;
    if (h->n > MT_NOALLOC_MAX_CELLS)
        return fail(MT_ERR_ARG, "n = %d cells exceeds the %d-cell limit of mt_rhs_noalloc (use mt_rhs)", h->n,
                    MT_NOALLOC_MAX_CELLS);
    int rc = check_ready(h, true, true);
    if (rc) return rc;
    if (!m_dev || !dmdt_dev) return fail(MT_ERR_ARG, "null device pointer");
    int dev = -1;
    CUDA_TRY(cudaGetDevice(&dev));
    if (dev != h->device) return fail(MT_ERR_ARG, "current device %d is not the handle's device %d", dev, h->device);
    float* scratch = nullptr;
    if ((rc = noalloc_scratch(dev, &scratch))) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    DevProb P = make_prob(h);
    // the conversion rewrites all 3*ldk entries (zero padding included), so no
    // state left by an earlier call is read
    CUDA_TRY(launch_m_to_f32(m_dev, h->n, h->ldk, scratch, s));
    CUDA_TRY(launch_field(2, P, m_dev, scratch, t, dmdt_dev, nullptr, nullptr, nullptr, nullptr, 0.f, h->num_sms, s));
    return MT_OK;
}
