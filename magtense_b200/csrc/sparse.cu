// Thresholded-sparse demag tensor (dem_appr "threshold" / "threshold_fraction"):
// the entries of the dense FP32 tensor with |K| above a threshold, as one CSR
// matrix of 3n receiver rows (row 3 i + a: blocks K_ax, K_ay, K_az of cell i in
// that order, column b*ldk + j).  It replaces ApplyThresholdDense /
// ConvertDenseToSparse_s (DemagAuxFunctions.f90:20-122, util_micromag.f90:81-138),
// whose six block matrices keep |K| > threshold; the product then runs on the
// kept entries only (demag_cta_sparse in llg.cuh).  The threshold of the fraction
// mode comes from the bisection of FindThresholdFraction
// (DemagAuxFunctions.f90:353-428), run on the host over counts made here.
#include "common.cuh"
#include "sparse.cuh"

namespace {

__constant__ int cBlk[3][3] = {{0, 1, 2}, {1, 3, 4}, {2, 4, 5}};

// kept entries of every receiver row: one warp per row
__global__ void sp_count_kernel(const float* __restrict__ K, int n, int ldk, float thr, int* __restrict__ counts)
{
    const int lane = threadIdx.x & 31;
    const int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (row >= 3 * n) return;
    const int i = row / 3, a = row - 3 * i;
    int c = 0;
    for (int b = 0; b < 3; ++b) {
        const float* r = K + ((size_t)i * 6 + cBlk[a][b]) * ldk;
        for (int j = lane; j < n; j += 32) c += fabsf(r[j]) > thr ? 1 : 0;
    }
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if (lane == 0) counts[row] = c;
}

// the kept entries, block by block and in increasing source order within a row
__global__ void sp_fill_kernel(const float* __restrict__ K, int n, int ldk, float thr, const int* __restrict__ rowptr,
                               int* __restrict__ col, float* __restrict__ val)
{
    const int lane = threadIdx.x & 31;
    const int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (row >= 3 * n) return;
    const int i = row / 3, a = row - 3 * i;
    int pos = rowptr[row];
    const unsigned below = (1u << lane) - 1u;
    for (int b = 0; b < 3; ++b) {
        const float* r = K + ((size_t)i * 6 + cBlk[a][b]) * ldk;
        for (int j0 = 0; j0 < n; j0 += 32) {
            const int j = j0 + lane;
            const float v = j < n ? r[j] : 0.f;
            const bool keep = j < n && fabsf(v) > thr;
            const unsigned mask = __ballot_sync(0xffffffffu, keep);
            if (keep) {
                const int p = pos + __popc(mask & below);
                col[p] = b * ldk + j;
                val[p] = v;
            }
            pos += __popc(mask);
        }
    }
}

// positive entries of the six blocks (the set FindThresholdFraction works on): count,
// and the count of those <= f
__global__ void sp_count_pos_kernel(const float* __restrict__ K, int n, int ldk, float f,
                                    unsigned long long* __restrict__ out /* [2]: positive, positive <= f */)
{
    unsigned long long pos = 0, le = 0;
    const size_t tot = (size_t)n * 6 * n;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < tot; e += (size_t)gridDim.x * blockDim.x) {
        const size_t rc = e / n;
        const int j = (int)(e - rc * n);
        const float v = K[rc * ldk + j];
        if (v > 0.f) { pos++; if (v <= f) le++; }
    }
    for (int o = 16; o > 0; o >>= 1) {
        pos += __shfl_xor_sync(0xffffffffu, pos, o);
        le += __shfl_xor_sync(0xffffffffu, le, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&out[0], pos);
        atomicAdd(&out[1], le);
    }
}

// smallest and largest positive entry (as bit patterns: positive floats order like their bits)
__global__ void sp_pos_minmax_kernel(const float* __restrict__ K, int n, int ldk, unsigned* __restrict__ out /* min, max */)
{
    unsigned mn = 0xffffffffu, mx = 0u;
    const size_t tot = (size_t)n * 6 * n;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < tot; e += (size_t)gridDim.x * blockDim.x) {
        const size_t rc = e / n;
        const int j = (int)(e - rc * n);
        const float v = K[rc * ldk + j];
        if (v > 0.f) {
            const unsigned u = __float_as_uint(v);
            mn = min(mn, u);
            mx = max(mx, u);
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        mn = min(mn, __shfl_xor_sync(0xffffffffu, mn, o));
        mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMin(&out[0], mn);
        atomicMax(&out[1], mx);
    }
}

}  // namespace

cudaError_t sparse_count_rows(const float* K, int n, int ldk, float thr, int* counts, cudaStream_t s)
{
    const int threads = 256, rows = 3 * n;
    const int blocks = (rows * 32 + threads - 1) / threads;
    sp_count_kernel<<<blocks, threads, 0, s>>>(K, n, ldk, thr, counts);
    return cudaGetLastError();
}

cudaError_t sparse_fill_rows(const float* K, int n, int ldk, float thr, const int* rowptr, int* col, float* val,
                             cudaStream_t s)
{
    const int threads = 256, rows = 3 * n;
    const int blocks = (rows * 32 + threads - 1) / threads;
    sp_fill_kernel<<<blocks, threads, 0, s>>>(K, n, ldk, thr, rowptr, col, val);
    return cudaGetLastError();
}

cudaError_t sparse_count_positive(const float* K, int n, int ldk, float f, unsigned long long* out, cudaStream_t s)
{
    cudaError_t e = cudaMemsetAsync(out, 0, 2 * sizeof(unsigned long long), s);
    if (e != cudaSuccess) return e;
    sp_count_pos_kernel<<<592, 256, 0, s>>>(K, n, ldk, f, out);
    return cudaGetLastError();
}

cudaError_t sparse_positive_minmax(const float* K, int n, int ldk, unsigned* out, cudaStream_t s)
{
    const unsigned init[2] = {0xffffffffu, 0u};
    cudaError_t e = cudaMemcpyAsync(out, init, sizeof(init), cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return e;
    sp_pos_minmax_kernel<<<592, 256, 0, s>>>(K, n, ldk, out);
    return cudaGetLastError();
}
