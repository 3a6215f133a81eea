// Stand-alone (non-persistent) field kernels behind mt_demag_field, mt_fields,
// mt_rhs and icl_MVMult_GetH.  One CTA owns a few receiver cells and streams
// their tensor records (demag_cta in llg.cuh), then applies the per-cell
// epilogue.
#include <mutex>

#include "common.cuh"
#include "llg.cuh"
#include "fields.cuh"

namespace {

// m (3n FP64) -> FP32 [3][ldk] with zero padding (updateDemagfield :576-578)
__global__ void m_to_f32_kernel(const double* __restrict__ m, int n, int ldk, float* __restrict__ m32)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= 3 * ldk) return;
    const int a = e / ldk, i = e - a * ldk;
    m32[e] = (i < n) ? (float)m[(size_t)a * n + i] : 0.0f;
}

// three FP32 host-layout vectors -> [3][ldk]
__global__ void pack3_f32_kernel(const float* __restrict__ x, const float* __restrict__ y,
                                 const float* __restrict__ z, int n, int ldk, float* __restrict__ m32)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= 3 * ldk) return;
    const int a = e / ldk, i = e - a * ldk;
    const float* src = a == 0 ? x : (a == 1 ? y : z);
    m32[e] = (i < n) ? src[i] : 0.0f;
}

// Vector-Jacobian product of dm/dt = -gamma c - alpha (m x c), c = he x m
// (he = hh + hj + hm + hk, the internal field of cell_rhs) for a cotangent lam:
// with u = he x m and w = -gamma lam - alpha (lam x m),
//   d/dhe = m x w,   d/dm (through the cross products) = w x he - alpha (u x lam).
// The field terms then add (all three operators are symmetric):
//   exchange  hj = -2 Jfact L m        ->  -2 L (Jfact g_he)       (mode 5)
//   demag     hm = -Ms K m (FP32 K)    ->  -K (Ms g_he)            (mode 5, same streaming product)
//   anisotropy hk = -2 Kfact A m       ->  -2 Kfact A g_he         (here)
//   Zeeman    hh = -hext(t)            ->  d/dhext = -sum_i g_he   (by the caller)
//   per-cell Ms: d hm/dMs = -K m, d hj/dMs = -hj/Ms, d hk/dMs = -hk/Ms.
MT_DEV void cell_vjp(const DevProb& P, const double* m, int i, const float S[3], const TimeScalars& ts,
                     const double* lam, double gm[3], double ghe[3], double* gms)
{
    const int n = P.n;
    CellFields F = cell_fields(P, m, i, S, ts);
    const double mv[3] = {ldcg(&m[i]), ldcg(&m[n + i]), ldcg(&m[2 * n + i])};
    const double lv[3] = {lam[i], lam[n + i], lam[2 * n + i]};
    double he[3], u[3], w[3], lxm[3], wxh[3], uxl[3];
    for (int a = 0; a < 3; ++a) he[a] = F.hh[a] + F.hj[a] + F.hm[a] + F.hk[a];
    auto cross = [](const double* x, const double* y, double* z) {
        z[0] = x[1] * y[2] - x[2] * y[1];
        z[1] = x[2] * y[0] - x[0] * y[2];
        z[2] = x[0] * y[1] - x[1] * y[0];
    };
    cross(he, mv, u);
    cross(lv, mv, lxm);
    for (int a = 0; a < 3; ++a) w[a] = -P.gamma * lv[a] - ts.alpha * lxm[a];
    cross(mv, w, ghe);
    cross(w, he, wxh);
    cross(u, lv, uxl);
    const double k2 = -2.0 * __ldg(&P.Kfact[i]);
    const double A[6] = {__ldg(&P.A6[0 * (size_t)n + i]), __ldg(&P.A6[1 * (size_t)n + i]),
                         __ldg(&P.A6[2 * (size_t)n + i]), __ldg(&P.A6[3 * (size_t)n + i]),
                         __ldg(&P.A6[4 * (size_t)n + i]), __ldg(&P.A6[5 * (size_t)n + i])};
    const double Ag[3] = {A[0] * ghe[0] + A[1] * ghe[1] + A[2] * ghe[2], A[1] * ghe[0] + A[3] * ghe[1] + A[4] * ghe[2],
                          A[2] * ghe[0] + A[4] * ghe[1] + A[5] * ghe[2]};
    for (int a = 0; a < 3; ++a) gm[a] = wxh[a] - ts.alpha * uxl[a] + k2 * Ag[a];
    const double ms = (double)__ldg(&P.Mfact[i]);
    double g = 0.0;
    for (int a = 0; a < 3; ++a) g += ghe[a] * (-(double)S[a] - F.hj[a] / ms - F.hk[a] / ms);
    *gms = g;
}

template <int MODE>
__global__ void __launch_bounds__(kFieldThreads)
field_kernel(DevProb P, const double* __restrict__ m, const float* __restrict__ m32, double t, int cells_per_cta,
             double* o0, double* o1, double* o2, double* o3, float* h32, float pref)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const int JC = P.ldk < kDemagJC ? P.ldk : kDemagJC;
    float* sm_m = reinterpret_cast<float*>(smem);
    float* sm_part = sm_m + 3 * JC;
    float* sm_S = sm_part + 3 * kDemagMaxUnits;
    const int c0 = blockIdx.x * cells_per_cta;
    const int nc = min(cells_per_cta, P.n - c0);
    if (nc <= 0) return;
    demag_cta(P, m32, c0, nc, sm_m, sm_part, sm_S, 2);
    const int n = P.n;
    if (MODE == 3) {   // raw product H = pref * K m (FP32), reference shim
        for (int e = threadIdx.x; e < 3 * nc; e += blockDim.x) {
            const int cell = e / 3, a = e - cell * 3;
            h32[(size_t)a * n + c0 + cell] = __fmul_rn(pref, sm_S[e]);
        }
        return;
    }
    if (MODE == 5) {   // VJP, second pass: m32 holds Ms g_he; o1 holds Jfact g_he; o0 += -K(Ms g_he) - 2 L(Jfact g_he)
        for (int cell = threadIdx.x; cell < nc; cell += blockDim.x) {
            const int i = c0 + cell;
            for (int a = 0; a < 3; ++a) {
                const double lz = lap_cell_dev(P, o1 + (size_t)a * n, i);
                o0[(size_t)a * n + i] += -(double)sm_S[cell * 3 + a] - 2.0 * lz;
            }
        }
        return;
    }
    const TimeScalars ts = time_scalars(P, t);
    for (int cell = threadIdx.x; cell < nc; cell += blockDim.x) {
        const int i = c0 + cell;
        if (MODE == 0) {
            const float ms = __ldg(&P.Mfact[i]);
            for (int a = 0; a < 3; ++a) o0[(size_t)a * n + i] = (double)__fmul_rn(-sm_S[cell * 3 + a], ms);
        } else if (MODE == 1) {
            CellFields F = cell_fields(P, m, i, &sm_S[cell * 3], ts);
            for (int a = 0; a < 3; ++a) {
                o0[(size_t)a * n + i] = F.hj[a];
                o1[(size_t)a * n + i] = F.hh[a];
                o2[(size_t)a * n + i] = F.hk[a];
                o3[(size_t)a * n + i] = F.hm[a];
            }
        } else if (MODE == 4) {   // VJP, first pass: o3 = [lam (3n) | g_Ms (n)]; o0 = g_m (local part),
                                  // o1 = Jfact g_he, o2 = g_he, h32 = Ms g_he (FP32, [3][ldk])
            double gm[3], ghe[3], gms;
            cell_vjp(P, m, i, &sm_S[cell * 3], ts, o3, gm, ghe, &gms);
            const double jf = __ldg(&P.Jfact[i]);
            const float ms = __ldg(&P.Mfact[i]);
            for (int a = 0; a < 3; ++a) {
                o0[(size_t)a * n + i] = gm[a];
                o1[(size_t)a * n + i] = jf * ghe[a];
                o2[(size_t)a * n + i] = ghe[a];
                h32[(size_t)a * P.ldk + i] = (float)((double)ms * ghe[a]);
            }
            o3[3 * (size_t)n + i] = gms;
        } else {
            double o[3];
            cell_rhs(P, m, i, &sm_S[cell * 3], ts, o);
            for (int a = 0; a < 3; ++a) o0[(size_t)a * n + i] = o[a];
        }
    }
}

}  // namespace

cudaError_t launch_m_to_f32(const double* m, int n, int ldk, float* m32, cudaStream_t s)
{
    const int tot = 3 * ldk;
    m_to_f32_kernel<<<(tot + 255) / 256, 256, 0, s>>>(m, n, ldk, m32);
    return cudaGetLastError();
}

cudaError_t launch_pack3_f32(const float* x, const float* y, const float* z, int n, int ldk, float* m32,
                             cudaStream_t s)
{
    const int tot = 3 * ldk;
    pack3_f32_kernel<<<(tot + 255) / 256, 256, 0, s>>>(x, y, z, n, ldk, m32);
    return cudaGetLastError();
}

int field_cells_per_cta(int n, int num_sms)
{
    int target = 2 * num_sms;
    int c = (n + target - 1) / target;
    if (c < 1) c = 1;
    if (c > 1024) c = 1024;
    return c;
}

cudaError_t launch_field(int mode, const DevProb& P, const double* m, const float* m32, double t, double* o0,
                         double* o1, double* o2, double* o3, float* h32, float pref, int num_sms, cudaStream_t s)
{
    const int cpc = field_cells_per_cta(P.n, num_sms);
    const int grid = (P.n + cpc - 1) / cpc;
    const size_t smem = demag_smem_bytes(P.ldk, cpc);
    cudaError_t e = cudaSuccess;
    // the shared-memory limit is raised only when it grows (once per mode and size in practice),
    // so repeated launches, for example inside a stream capture, make no attribute calls.  The
    // per-device record is shared by every host thread, hence the lock around check and update.
    constexpr int kMaxDev = 256;
    static size_t smem_set[kMaxDev][6] = {};
    static std::mutex smem_mu;
    int dev = 0;
    e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    size_t* set = (dev >= 0 && dev < kMaxDev) ? smem_set[dev] : nullptr;
#define MT_LAUNCH(M)                                                                                           \
    do {                                                                                                       \
        {                                                                                                      \
            std::lock_guard<std::mutex> lock(smem_mu);                                                         \
            if (!set || smem > set[M]) {                                                                       \
                e = cudaFuncSetAttribute(field_kernel<M>, cudaFuncAttributeMaxDynamicSharedMemorySize,         \
                                         (int)smem);                                                           \
                if (e != cudaSuccess) return e;                                                                \
                if (set) set[M] = smem;                                                                        \
            }                                                                                                  \
        }                                                                                                      \
        field_kernel<M><<<grid, kFieldThreads, smem, s>>>(P, m, m32, t, cpc, o0, o1, o2, o3, h32, pref);       \
    } while (0)
    switch (mode) {
        case 0: MT_LAUNCH(0); break;
        case 1: MT_LAUNCH(1); break;
        case 2: MT_LAUNCH(2); break;
        case 3: MT_LAUNCH(3); break;
        case 4: MT_LAUNCH(4); break;
        case 5: MT_LAUNCH(5); break;
        default: return cudaErrorInvalidValue;
    }
#undef MT_LAUNCH
    return cudaGetLastError();
}
