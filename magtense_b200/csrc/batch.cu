// Batched adaptive integration of B Landau-Lifshitz instances sharing one
// geometry, in ONE persistent cooperative kernel.
//
// Every instance runs its own RKSUITE-90 method 'M' (per-instance t, h, phases,
// counters, flags, dense output), exactly as the single-instance integrator
// (integrate.cu) and the reference (RKSuitef90.f90: step_integrate_r1
// :1185-1587, step_r1 :1726-1978, stiff_r1 :1981-2367, interpolate_r1
// :2655-2997, range_integrate_r1 :942-1183; driver ODE_Solvers.f90:124-237).
// The control flow is written once, synchronously, as a coroutine: it yields
// when it needs a right-hand side f(t, y); norms over all its cells resolve in
// place (post_reduce: the instance's cell-block CTAs meet on a per-instance
// arrival counter).  The kernel advances all instances in lock-step "ticks":
//
//   B1  grid barrier (stage arguments and requests of all cells visible)
//   G   demag product of the requesting instances -> partial H
//   Bh  grid barrier (partial H visible)
//   P1  for instances that asked for f: sum the partials, apply the LL
//       epilogue (exchange, anisotropy, Zeeman at the instance's own t,
//       cross products) on the owned cells, advance to the next request,
//       publish the requests of the next tick
//
// Tile (cb, ib, s): receiver cells [128 cb, 128 cb + 128) for all three field
// components, instances [64 ib, 64 ib + 64), source range split s of S.  The
// coroutines of instances [64 ib + s*64/S, ...) on cells of block cb run in
// the same CTA, one warp per instance, so the epilogue reads only H the CTA
// group produced for its own cells.  Stage arguments alternate between two
// buffers so no argument is rewritten while another CTA may still read it
// (every rewrite of the same buffer is separated by a grid barrier).
#include "batch.cuh"
#include "gemm_tc.cuh"

namespace {

struct BS45b { double a[12][12]; double b[9]; double c[12]; double e[8]; double r[12][7]; };
__constant__ BS45b cB;

// destination ids of right-hand-side results
enum { DST_STG = 0, DST_DERIV = 20 };

struct BCtx {
    DevProb P;
    BatchBufs F;
    BatchParams Q;
    int cb, ib, s;          // tile coordinates of this CTA
    int c0, nc;             // owned cells
    int i0, ni;             // owned instances (coroutines)
    size_t n3;              // 3n
    int lane, warp, nwarps;
    unsigned char* smem;
    BInst* sinst;           // shared-memory copies of the owned coroutines
    long long tick;
    // int8 backend, set every tick: active instance tiles, Stream-K units and the
    // CTAs covering this CTA's tiles (3 components x 2 instance tiles from jb0)
    int nact;
    long long U;
    const int* act_pos;     // [2 IB] position of a 64-instance tile in the active list, -1 if idle
    int jb0;                // first tile of this CTA's instances (compact positions when packed)
    const SkCover* cov;     // [3][3]
    bool packed;            // instances sit at their compact positions (integration) or at b (demag only)
    const unsigned* bits;   // [Bp / 32] request bits of this tick (packed)
    const int* pre;         // [Bp / 32] requests before each word (packed)
    int sched;              // Stream-K schedule word of this tick's GEMM
    bool prev_valid;        // bits/pre hold the previous tick's requests (int8): the coroutines also
                            // write their operand rows at those compact positions
};

// compact position of requesting instance b: requests with a smaller index
MT_DEV int compact_pos(const BCtx& X, int b)
{
    if (!X.packed) return b;
    const int w = b >> 5;
    return X.pre[w] + __popc(X.bits[w] & ((1u << (b & 31)) - 1u));
}

// per-instance vector addressing
MT_DEV double* VPOOL(const BCtx& X, int k, int b) { return X.F.pool + ((size_t)k * X.Q.Bp + b) * X.n3; }
MT_DEV double* VDER(const BCtx& X, int k, int b) { return X.F.deriv + ((size_t)k * X.Q.Bp + b) * X.n3; }
MT_DEV double* VSTG(const BCtx& X, int k, int b) { return X.F.stg + ((size_t)k * X.Q.Bp + b) * X.n3; }
MT_DEV double* VP(const BCtx& X, int k, int b) { return X.F.p + ((size_t)k * X.Q.Bp + b) * X.n3; }
MT_DEV double* VONE(const BCtx& X, double* base, int b) { return base + (size_t)b * X.n3; }

MT_DEV double* dst_ptr(const BCtx& X, int id, int b)
{
    if (id >= DST_DERIV) return VDER(X, id - DST_DERIV, b);
    return VSTG(X, id, b);
}

// hi/lo split of one FP32 value into the 16-bit operand format of the precision
MT_DEV void split_store(float f, int prec, uint16_t* hi_out, uint16_t* lo_out)
{
    if (prec == kPrecFP16x3S) {
        const __half hi = __float2half_rn(f);
        const __half lo = __float2half_rn(f - __half2float(hi));
        *hi_out = __half_as_ushort(hi);
        *lo_out = __half_as_ushort(lo);
    } else {
        const __nv_bfloat16 hi = __float2bfloat16_rn(f);
        const __nv_bfloat16 lo = __float2bfloat16_rn(f - __bfloat162float(hi));
        *hi_out = __bfloat16_as_ushort(hi);
        *lo_out = __bfloat16_as_ushort(lo);
    }
}

// own elements of one instance, lane-strided: component a, cell i, index q = a*n + i
#define FOR_OWN_W(X, q)                                                                       \
    for (int _e = (X).lane; _e < 3 * (X).nc; _e += 32)                                        \
        if ([[maybe_unused]] const int _a = (_e >= (X).nc) + (_e >= 2 * (X).nc),              \
                      _i = (X).c0 + (_e - _a * (X).nc), q = _a * (X).P.n + _i; true)

// int8 limbs of one source value: mq = rint(v 2^30) = m0 2^24 + m1 2^16 + m2 2^8 + m3
// (signed digits, m3 lowest).  |v| must stay below 1.96 so that m0 fits; a value
// outside records KERR_RANGE and stops the launch.
constexpr double kI8MScale = 1073741824.0;   // 2^30
constexpr double kI8MMax = 1.96;

MT_DEV void i8_store_m(double v, int8_t* dst, size_t limb_stride, GridSync* gs, int8_t* dst2 = nullptr)
{
    if (!(fabs(v) <= kI8MMax)) {
        if (atomicCAS(&gs->err, 0, KERR_RANGE) == 0) gs->err_where = 300;
        atomicExch(&gs->abort, 1);
        v = 0.0;
    }
    // |v| <= 1.96, so rint(v 2^30) fits in 32 bits; x - dl is a multiple of 256 and the
    // arithmetic shift divides it exactly
    int x = __double2int_rn(v * kI8MScale);
    int8_t d[4];
#pragma unroll
    for (int l = 3; l >= 1; --l) {
        const int dl = (int)(signed char)(x & 0xff);
        d[l] = (int8_t)dl;
        x = (x - dl) >> 8;
    }
    d[0] = (int8_t)x;
#pragma unroll
    for (int l = 0; l < 4; ++l) dst[(size_t)l * limb_stride] = d[l];
    if (dst2) {
#pragma unroll
        for (int l = 0; l < 4; ++l) dst2[(size_t)l * limb_stride] = d[l];
    }
}

// write the stage argument (FP64) and the GEMM operand copy for one element
MT_DEV void put_arg(const BCtx& X, int argi, int b, int q, double v)
{
    VPOOL(X, argi, b)[q] = v;
    const int n = X.P.n;
    const int a = (q >= n) + (q >= 2 * n), i = q - a * n;   // q < 3n
    const float f = (float)v;
    if (X.Q.prec == kPrecI8) {
        int8_t* comp = nullptr;
        if (X.prev_valid && ((X.bits[b >> 5] >> (b & 31)) & 1u))
            comp = X.F.mcomp + (size_t)compact_pos(X, b) * X.Q.Kd + (size_t)a * X.Q.np + i;
        i8_store_m(v, X.F.mlimb + (size_t)b * X.Q.Kd + (size_t)a * X.Q.np + i, (size_t)X.Q.Bp * X.Q.Kd, X.F.gs, comp);
    } else if (X.Q.prec == kPrecFP32) {
        X.F.m32[((size_t)b * 3 + a) * X.P.ldk + i] = f;
    } else {
        const size_t col = (size_t)b * X.Q.Kd + (size_t)a * X.Q.np + i;
        split_store(f, X.Q.prec, X.F.mhi + col, X.F.mlo + col);
    }
}

// Where the stage argument of instance b goes: its FP64 copy and the GEMM
// operand of the precision, as plain pointers and strides.
struct ArgDst {
    double* pool;          // FP64 argument (3n)
    int prec, n, np, ldk;
    float* m32;            // fp32: [3][ldk] of instance b
    uint16_t* mhi;         // 16-bit splits: column b*Kd
    uint16_t* mlo;
    int8_t* mlimb;         // int8: column b*Kd of limb 0
    int8_t* mcomp;         // int8: the instance's row at its previous compact position, or nullptr
    size_t limb_stride;
    GridSync* gs;
};

MT_DEV ArgDst arg_dst(const BCtx& X, int argi, int b)
{
    ArgDst d;
    d.pool = VPOOL(X, argi, b);
    d.prec = X.Q.prec; d.n = X.P.n; d.np = X.Q.np; d.ldk = X.P.ldk;
    d.m32 = X.F.m32 ? X.F.m32 + (size_t)b * 3 * X.P.ldk : nullptr;
    d.mhi = X.F.mhi ? X.F.mhi + (size_t)b * X.Q.Kd : nullptr;
    d.mlo = X.F.mlo ? X.F.mlo + (size_t)b * X.Q.Kd : nullptr;
    d.mlimb = X.F.mlimb ? X.F.mlimb + (size_t)b * X.Q.Kd : nullptr;
    d.mcomp = (X.F.mlimb && X.prev_valid && ((X.bits[b >> 5] >> (b & 31)) & 1u))
                  ? X.F.mcomp + (size_t)compact_pos(X, b) * X.Q.Kd : nullptr;
    d.limb_stride = (size_t)X.Q.Bp * X.Q.Kd;
    d.gs = X.F.gs;
    return d;
}

MT_DEV void put_arg_d(const ArgDst& d, int q, double v)
{
    d.pool[q] = v;
    const int a = (q >= d.n) + (q >= 2 * d.n), i = q - a * d.n;   // q < 3n
    if (d.prec == kPrecI8) {
        i8_store_m(v, d.mlimb + (size_t)a * d.np + i, d.limb_stride, d.gs,
                   d.mcomp ? d.mcomp + (size_t)a * d.np + i : nullptr);
    } else if (d.prec == kPrecFP32) {
        d.m32[(size_t)a * d.ldk + i] = (float)v;
    } else {
        const size_t col = (size_t)a * d.np + i;
        split_store((float)v, d.prec, d.mhi + col, d.mlo + col);
    }
}

struct StgPtrs { const double* s[8]; };

// The stage argument y + h sum_j a_ij k_j of stage i on the lane's owned elements,
// with the stepb error estimate at stage 7 (returned: the lane's max) and the
// combination kept for the error estimate at stage 8.  Non-inlined and fed plain
// pointers, so its loop runs from registers.
__device__ __noinline__ double stage_args(int i, const double* __restrict__ y, const double* __restrict__ yp,
                                          StgPtrs st, double* __restrict__ es, ArgDst d, double htry, double thr,
                                          int lane, int c0, int nc)
{
    constexpr int U = 2;   // elements per lane in flight
    double lm = 0.0;
    const int n = d.n, tot = 3 * nc;
    for (int e0 = lane; e0 < tot; e0 += 32 * U) {
        int q[U];
        bool on[U];
        double kv[U][8], ypq[U], yq[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int e = e0 + 32 * u;
            on[u] = e < tot;
            const int ee = on[u] ? e : e0;
            const int a = (ee >= nc) + (ee >= 2 * nc);   // ee < 3 nc
            q[u] = a * n + c0 + (ee - a * nc);
#pragma unroll
            for (int j = 2; j <= 7; ++j) kv[u][j] = (j <= i - 1) ? ldcg(&st.s[j][q[u]]) : 0.0;
            ypq[u] = ldcg(&yp[q[u]]);
            yq[u] = ldcg(&y[q[u]]);
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            if (!on[u]) continue;
            double e = xmul(cB.a[i][1], ypq[u]);
#pragma unroll
            for (int j = 2; j <= 7; ++j) {
                if (j > i - 1) break;
                const double aij = cB.a[i][j];
                if (aij == 0.0) continue;
                e = xadd(e, xmul(aij, kv[u][j]));
            }
            const double yn = xadd(yq[u], xmul(htry, e));
            put_arg_d(d, q[u], yn);
            if (i == 8) es[q[u]] = e;
            if (i == 7) {
                double v = xmul(cB.e[1], ypq[u]);
                v = xadd(v, xmul(cB.e[3], kv[u][3]));
                v = xadd(v, xmul(cB.e[4], kv[u][4]));
                v = xadd(v, xmul(cB.e[5], kv[u][5]));
                v = xadd(v, xmul(cB.e[6], kv[u][6]));
                const double wq = fmax(xmul(0.5, xadd(fabs(yq[u]), fabs(yn))), thr);
                lm = fmax(lm, fabs(v) / wq);
            }
        }
    }
    __syncwarp();
    return lm;
}

// The other per-element loops of a step, written like stage_args: non-inlined, plain
// pointers, kInFlight elements per lane in flight, each element's arithmetic in the same
// order as the synchronous formulation (and the oracle).  Two measured faster than one,
// three or six (the stage-argument loop too): more loads in flight per lane slowed
// every warp's loop down.
constexpr int kInFlight = 2;

MT_DEV int own_q(int e, int n, int c0, int nc)
{
    const int a = (e >= nc) + (e >= 2 * nc);   // e < 3 nc
    return a * n + c0 + (e - a * nc);
}

// stage i = 9..11 of the interpolant: y_old + h_old (a_i1 k1 + sum_{j=2}^{i-1} a_ij k_j), k8 = y'
struct IntPtrs { const double* k[11]; };

__device__ __noinline__ void interp_stage_args(int i, const double* __restrict__ yold, const double* __restrict__ k1,
                                               IntPtrs st, ArgDst d, double h_old, int lane, int c0, int nc)
{
    const int n = d.n, tot = 3 * nc;
    for (int e0 = lane; e0 < tot; e0 += 32 * kInFlight) {
        int q[kInFlight];
        bool on[kInFlight];
        double kv[kInFlight][11], k1q[kInFlight], yoq[kInFlight];
#pragma unroll
        for (int u = 0; u < kInFlight; ++u) {
            const int e = e0 + 32 * u;
            on[u] = e < tot;
            q[u] = own_q(on[u] ? e : e0, n, c0, nc);
#pragma unroll
            for (int j = 2; j <= 10; ++j) kv[u][j] = (j <= i - 1) ? ldcg(&st.k[j][q[u]]) : 0.0;
            k1q[u] = ldcg(&k1[q[u]]);
            yoq[u] = ldcg(&yold[q[u]]);
        }
#pragma unroll
        for (int u = 0; u < kInFlight; ++u) {
            if (!on[u]) continue;
            double e = xmul(cB.a[i][1], k1q[u]);
#pragma unroll
            for (int j = 2; j <= 10; ++j) {
                if (j > i - 1) break;
                e = xadd(e, xmul(cB.a[i][j], kv[u][j]));
            }
            put_arg_d(d, q[u], xadd(yoq[u], xmul(h_old, e)));
        }
    }
    __syncwarp();
}

// the interpolant's coefficients p1..p5 (the vendored grouping of terms), times h_old
struct PolyPtrs { const double* k[12]; double* p[6]; };

__device__ __noinline__ void interp_coeffs(PolyPtrs pp, double ho, int lane, int n, int c0, int nc)
{
    const int tot = 3 * nc;
    for (int e0 = lane; e0 < tot; e0 += 32 * kInFlight) {
        int q[kInFlight];
        bool on[kInFlight];
        double K[kInFlight][12];
#pragma unroll
        for (int u = 0; u < kInFlight; ++u) {
            const int e = e0 + 32 * u;
            on[u] = e < tot;
            q[u] = own_q(on[u] ? e : e0, n, c0, nc);
            K[u][1] = ldcg(&pp.k[1][q[u]]);
#pragma unroll
            for (int j = 3; j <= 11; ++j) K[u][j] = ldcg(&pp.k[j][q[u]]);
        }
#pragma unroll
        for (int u = 0; u < kInFlight; ++u) {
            if (!on[u]) continue;
            const double K1 = K[u][1], K3 = K[u][3], K4 = K[u][4], K5 = K[u][5], K6 = K[u][6], K7 = K[u][7];
            const double K8 = K[u][8], K9 = K[u][9], K10 = K[u][10], K11 = K[u][11];
#define R(i, j) cB.r[i][j]
#define M(a, b2) xmul(a, b2)
#define A(a, b2) xadd(a, b2)
            const double p5 = A(A(M(R(5, 6), K5), A(A(M(R(10, 6), K10), M(R(8, 6), K8)), A(M(R(7, 6), K7), M(R(6, 6), K6)))),
                                A(A(A(M(R(4, 6), K4), M(R(9, 6), K9)), A(M(R(3, 6), K3), M(R(11, 6), K11))), M(R(1, 6), K1)));
            const double p4 = A(A(A(M(R(10, 5), K10), M(R(9, 5), K9)), A(A(M(R(7, 5), K7), M(R(6, 5), K6)), M(R(5, 5), K5))),
                                A(A(A(M(R(4, 5), K4), M(R(8, 5), K8)), A(M(R(3, 5), K3), M(R(11, 5), K11))), M(R(1, 5), K1)));
            const double p3 = A(A(A(A(M(R(4, 4), K4), M(R(8, 4), K8)), A(M(R(7, 4), K7), M(R(6, 4), K6))), M(R(5, 4), K5)),
                                A(A(A(M(R(10, 4), K10), M(R(9, 4), K9)), A(M(R(3, 4), K3), M(R(11, 4), K11))), M(R(1, 4), K1)));
            const double p2 = A(A(A(M(R(5, 3), K5), M(R(6, 3), K6)),
                                  A(A(A(M(R(3, 3), K3), M(R(9, 3), K9)), A(M(R(10, 3), K10), M(R(8, 3), K8))), M(R(1, 3), K1))),
                                A(A(M(R(4, 3), K4), M(R(11, 3), K11)), M(R(7, 3), K7)));
            const double p1 = A(A(A(M(R(5, 2), K5), A(A(M(R(6, 2), K6), M(R(8, 2), K8)), M(R(1, 2), K1))),
                                  A(A(M(R(3, 2), K3), M(R(9, 2), K9)), M(R(10, 2), K10))),
                                A(A(M(R(4, 2), K4), M(R(11, 2), K11)), M(R(7, 2), K7)));
#undef R
#undef M
#undef A
            pp.p[5][q[u]] = xmul(ho, p5); pp.p[4][q[u]] = xmul(ho, p4); pp.p[3][q[u]] = xmul(ho, p3);
            pp.p[2][q[u]] = xmul(ho, p2); pp.p[1][q[u]] = xmul(ho, p1);
        }
    }
    __syncwarp();
}

// the interpolated solution at sigma: ((((p5 s + p4) s + p3) s + p2) s + p1) s + h y') s + y
__device__ __noinline__ void interp_eval(PolyPtrs pp, const double* __restrict__ y, const double* __restrict__ yp,
                                         double* __restrict__ dst, double sigma, double h_old, int lane, int n, int c0,
                                         int nc)
{
    const int tot = 3 * nc;
    for (int e0 = lane; e0 < tot; e0 += 32 * kInFlight) {
        int q[kInFlight];
        bool on[kInFlight];
        double P[kInFlight][6], ypq[kInFlight], yq[kInFlight];
#pragma unroll
        for (int u = 0; u < kInFlight; ++u) {
            const int e = e0 + 32 * u;
            on[u] = e < tot;
            q[u] = own_q(on[u] ? e : e0, n, c0, nc);
#pragma unroll
            for (int j = 1; j <= 5; ++j) P[u][j] = ldcg(&pp.p[j][q[u]]);
            ypq[u] = ldcg(&yp[q[u]]);
            yq[u] = ldcg(&y[q[u]]);
        }
#pragma unroll
        for (int u = 0; u < kInFlight; ++u) {
            if (!on[u]) continue;
            double v = xmul(P[u][5], sigma);
            v = xmul(xadd(v, P[u][4]), sigma);
            v = xmul(xadd(v, P[u][3]), sigma);
            v = xmul(xadd(v, P[u][2]), sigma);
            v = xmul(xadd(v, P[u][1]), sigma);
            dst[q[u]] = xadd(xmul(xadd(v, xmul(h_old, ypq[u])), sigma), yq[u]);
        }
    }
    __syncwarp();
}

// the error estimate of a completed step and the new weights; returns the lane's max of |es| / w
struct ErrPtrs { const double* k[8]; };

__device__ __noinline__ double step_error(ErrPtrs st, const double* __restrict__ y, const double* __restrict__ yp,
                                          const double* __restrict__ yn, const double* __restrict__ k8,
                                          double* __restrict__ es, double* __restrict__ w, double htry, double thr,
                                          int lane, int n, int c0, int nc)
{
    const int tot = 3 * nc;
    double lm = 0.0;
    for (int e0 = lane; e0 < tot; e0 += 32 * kInFlight) {
        int q[kInFlight];
        bool on[kInFlight];
        double kv[kInFlight][8], esq[kInFlight], ypq[kInFlight], k8q[kInFlight], yq[kInFlight], ynq[kInFlight];
#pragma unroll
        for (int u = 0; u < kInFlight; ++u) {
            const int e = e0 + 32 * u;
            on[u] = e < tot;
            q[u] = own_q(on[u] ? e : e0, n, c0, nc);
#pragma unroll
            for (int i = 2; i <= 7; ++i) kv[u][i] = ldcg(&st.k[i][q[u]]);
            esq[u] = ldcg(&es[q[u]]);
            ypq[u] = ldcg(&yp[q[u]]);
            k8q[u] = ldcg(&k8[q[u]]);
            yq[u] = ldcg(&y[q[u]]);
            ynq[u] = ldcg(&yn[q[u]]);
        }
#pragma unroll
        for (int u = 0; u < kInFlight; ++u) {
            if (!on[u]) continue;
            double v = esq[u];
            v = xsub(v, xmul(cB.b[1], ypq[u]));
#pragma unroll
            for (int i = 2; i <= 7; ++i) {
                if (cB.b[i] == 0.0) continue;
                v = xsub(v, xmul(cB.b[i], kv[u][i]));
            }
            v = xsub(v, xmul(cB.b[8], k8q[u]));
            v = xmul(htry, v);
            es[q[u]] = v;
            const double wq = fmax(xmul(0.5, xadd(fabs(yq[u]), fabs(ynq[u]))), thr);
            w[q[u]] = wq;
            lm = fmax(lm, fabs(v) / wq);
        }
    }
    __syncwarp();
    return lm;
}

MT_DEV double warp_red(double v, bool is_max)
{
    return is_max ? warp_max(v) : warp_sum(v);
}

// Reductions of K values over all cells of instance b.  Every cell-block CTA of the
// instance runs the same coroutine and reaches the same reduction: post_reduce
// writes the warp's partials to the slots of its cell block, counts the CTA in the
// instance's arrival counter and yields (req 2); resolve_reduce, run by the caller
// before it resumes the coroutine, waits (bounded) until all CB cell blocks have
// arrived and combines the CB partials in cell-block order, so every copy of the
// coroutine gets the same bits.  Slots alternate between two halves by the
// reduction's parity: a CTA can post reduction r + 1 only after all have arrived at
// r, and reduction r + 2 (same half) only after all have read r.  On a timeout the
// launch aborts and the coroutine is left with req 5.
MT_DEV double* red_slot(const BCtx& X, const BInst& I, int b)
{
    return X.F.partials + (size_t)(I.red_seq & 1) * X.Q.Bp * kRedSlots * X.Q.CB + (size_t)b * kRedSlots * X.Q.CB;
}

MT_DEV void post_reduce(const BCtx& X, BInst& I, int b, const double* v, int K, bool is_max)
{
    double* slot = red_slot(X, I, b);
    for (int k = 0; k < K; ++k) {
        const double r = warp_red(v[k], is_max);
        if (X.lane == 0) slot[(size_t)k * X.Q.CB + X.cb] = r;
    }
    if (X.lane == 0) {
        __threadfence();
        atomicAdd(&X.F.redcnt[b], 1u);
    }
    I.req = 2;
    I.red_k = K;
    I.red_max = is_max ? 1 : 0;
}

__device__ __noinline__ int wait_arrivals(unsigned* cnt, unsigned target, GridSync* gs, int lane)
{
    int ok = 1;
    if (lane == 0) {
        long long it = 0;
        const uint64_t t0 = globaltimer_ns();
        while ((int)(ld_acquire_u32(cnt) - target) < 0) {
            if (ld_volatile_i32(&gs->abort)) { ok = 0; break; }
            if (++it > kSpinLimit || ((it & 1023) == 0 && globaltimer_ns() - t0 > kTimeoutNs)) {
                if (atomicCAS(&gs->err, 0, KERR_BARRIER_TIMEOUT) == 0) gs->err_where = 400;
                atomicExch(&gs->abort, 1);
                ok = 0;
                break;
            }
            __nanosleep(20);
        }
    }
    __syncwarp();
    return __shfl_sync(0xffffffffu, ok, 0);
}

MT_DEV void resolve_reduce(const BCtx& X, BInst& I, int b)
{
    const unsigned target = (unsigned)X.Q.CB * (unsigned)(I.red_seq + 1);
    const double* slot = red_slot(X, I, b);
    I.red_seq++;
    if (!wait_arrivals(&X.F.redcnt[b], target, X.F.gs, X.lane)) { I.req = 5; return; }
    for (int k = 0; k < I.red_k; ++k) {
        double r = 0.0;
        for (int c = 0; c < X.Q.CB; ++c) {
            const double x = ldcg(&slot[(size_t)k * X.Q.CB + c]);
            r = (c == 0) ? x : (I.red_max ? fmax(r, x) : r + x);
        }
        I.red[k] = r;
    }
    I.req = 0;
}

// advance instance b to its next right-hand-side request, resolving its reductions
// on the way (returns with req 1, 3 done, 4 parked or 5 aborting)
#define ADVANCE_TO_REQUEST(X, I, b)                             \
    do {                                                        \
        advance(X, I, b);                                       \
        if ((I).req == 2) resolve_reduce(X, I, b);              \
    } while ((I).req == 0)

// time-dependent scalars of instance b
MT_DEV TimeScalars inst_scalars(const BCtx& X, int b, double t)
{
    DevProb P = X.P;
    P.hext = X.F.hext + (size_t)b * X.Q.nt_hext * 4;
    P.nt_hext = X.Q.nt_hext;
    P.alpha0 = X.F.alpha0[b];
    return time_scalars(P, t);
}

// ---------------------------------------------------------------------------
// The coroutine.  Yield points: Y_RHS (after writing the argument), Y_RED
// (after posting partials).  Control flow mirrors rk_range_integrate /
// rk_step_integrate / rk_step / rk_stiff / rk_interpolate in integrate.cu.
// ---------------------------------------------------------------------------
#define CO_YIELD(I, lbl) do { (I).pc = (lbl); return; case (lbl):; } while (0)
#define Y_RHS(I, lbl, t_, argi_, dst_) do { (I).req = 1; (I).t_rhs = (t_); (I).rhs_arg = (argi_); \
                                           (I).rhs_dst = (dst_); CO_YIELD(I, lbl); } while (0)

enum {
    L_START = 0, L_DRIVER, L_FIRSTF, L_FIRSTF_RED, L_STIFF1, L_STIFF2, L_STIFF_AJ, L_STIFF_AJ_RED, L_STEPB,
    L_STAGE, L_STEPA, L_FINAL, L_INTERP, L_CONV, L_DONE, L_STIFF_NORM,
    L_STIFF_LOOP = 100,   // + 10 * which vector (1,2,3) + sub
};

MT_DEV void copy_own(const BCtx& X, const double* src, double* dst)
{
    FOR_OWN_W(X, q) dst[q] = ldcg(&src[q]);
    __syncwarp();
}

MT_DEV void advance(BCtx& X, BInst& I, int b)
{
    RKS& s = I.s;
    const double thr = X.Q.thres;
    const size_t n3 = X.n3;
    (void)n3;
    switch (I.pc) {
    case L_START:
    // ================================ driver loop over output times
    for (;;) {
        if (s.ci >= X.Q.ncomb) { s.finished = 1; break; }
        I.t_want = X.Q.comb_t[s.ci];
        I.cf = X.Q.comb_flags[s.ci];
        I.dst_slot = ((I.cf & 1) && s.ko < X.Q.nt) ? 1 : 0;
        // ---- range_integrate prologue
        if (s.at_t_start) {
            s.range_t_end = s.t_end;
            s.tlast = s.t_start;
            I.t_got = s.t_start;
            s.h = fmin(fabs(s.h), fabs(xsub(I.t_want, s.t_start)));
            s.h = fmax(s.h, fmax(X.Q.sqtiny, xmul(X.Q.toosml, fmax(fabs(s.t_start), fabs(s.t_end)))));
        } else if (s.tlast == s.range_t_end) {
            s.status = 911; s.finished = 1; break;
        }
        if (xmul(s.dir, xsub(I.t_want, s.tlast)) <= 0.0 || xmul(s.dir, xsub(I.t_want, s.range_t_end)) > 0.0) {
            s.status = 911; s.finished = 1; break;
        }
        I.flag = 1;
        // ---- range_integrate loop
        for (;;) {
            if (xmul(s.dir, xsub(s.t, I.t_want)) >= 0.0) {
                // ---------------- interpolate
                if (!s.intrp_ready) {
                    for (I.i_stage = 9; I.i_stage <= 11; ++I.i_stage) {
                        {
                            const int i = I.i_stage;
                            const int argi = (i == 10) ? s.ia0 : s.ia1;
                            const double* yold = VPOOL(X, s.iyold, b);
                            const double* k1 = VDER(X, s.dypold, b);
                            const double* k8 = VDER(X, s.dyp, b);
                            IntPtrs ip;
                            for (int j = 0; j < 11; ++j) ip.k[j] = (j == 8) ? k8 : (j >= 2) ? VSTG(X, j, b) : nullptr;
                            interp_stage_args(i, yold, k1, ip, arg_dst(X, argi, b), s.h_old, X.lane, X.c0, X.nc);
                            I.tstg = xadd(s.t_old, xmul(cB.c[i], s.h_old));
                            I.argi = argi;
                        }
                        Y_RHS(I, L_INTERP + 1000 + 0, I.tstg, I.argi, DST_STG + I.i_stage);
                        s.f_count++;
                    }
                    {
                        const double ho = s.h_old;
                        const double* k1 = VDER(X, s.dypold, b);
                        const double* k8 = VDER(X, s.dyp, b);
                        PolyPtrs pp;
                        for (int j = 0; j < 12; ++j) pp.k[j] = (j == 1) ? k1 : (j == 8) ? k8 : (j >= 3) ? VSTG(X, j, b) : nullptr;
                        for (int j = 0; j < 6; ++j) pp.p[j] = (j >= 1) ? VP(X, j, b) : nullptr;
                        interp_coeffs(pp, ho, X.lane, X.P.n, X.c0, X.nc);
                        s.intrp_ready = 1;
                    }
                }
                {
                    const double sigma = xsub(I.t_want, s.t) / s.h_old;
                    const double* y = VPOOL(X, s.iy, b);
                    const double* yp = VDER(X, s.dyp, b);
                    double* dst = I.dst_slot ? X.F.y_out ? X.F.y_out + ((size_t)b * X.Q.nt + s.ko) * X.n3 : VONE(X, X.F.ystep, b)
                                             : VONE(X, X.F.ystep, b);
                    PolyPtrs pp;
                    for (int j = 0; j < 12; ++j) pp.k[j] = nullptr;
                    for (int j = 0; j < 6; ++j) pp.p[j] = (j >= 1) ? VP(X, j, b) : nullptr;
                    interp_eval(pp, y, yp, dst, sigma, s.h_old, X.lane, X.P.n, X.c0, X.nc);
                    I.t_got = I.t_want;
                }
                break;
            }
            // ---------------- step_integrate
            if (s.full_f_count + s.f_count >= I.budget_mark) {
                // per-launch budget exhausted: park here; the next launch resumes
                I.req = 4;
                CO_YIELD(I, L_DRIVER);
            }
            I.ier = 1;
            if (s.at_t_start) {
                {   // the GEMM operand holds the argument of the next request
                    const double* y = VPOOL(X, s.iy, b);
                    FOR_OWN_W(X, q) put_arg(X, s.iy, b, q, ldcg(&y[q]));
                    __syncwarp();
                }
                Y_RHS(I, L_FIRSTF, s.t, s.iy, DST_DERIV + s.dyp);
                s.f_count++;
                {
                    const double* y = VPOOL(X, s.iy, b);
                    const double* yp = VDER(X, s.dyp, b);
                    double* w = X.F.weights + (size_t)b * X.n3;
                    double mx = -1.0;
                    FOR_OWN_W(X, q) {
                        const double yq = ldcg(&y[q]);
                        const double wq = fmax(fabs(yq), thr);
                        w[q] = wq;
                        if (yq != 0.0) mx = fmax(mx, fabs(ldcg(&yp[q])) / wq);
                    }
                    __syncwarp();
                    post_reduce(X, I, b, &mx, 1, true);
                }
                CO_YIELD(I, L_FIRSTF_RED);
                {
                    s.phase2 = 1;
                    s.h = fabs(s.h);
                    const double ypnorm = fmax(0.0, I.red[0] < 0.0 ? -1.0 : I.red[0]);
                    const double tau = root5(s.tol);
                    if (xmul(s.h, ypnorm) > tau) s.h = tau / ypnorm;
                    I.hmin = fmax(X.Q.sqtiny, xmul(X.Q.toosml, fmax(fabs(s.t_start), fabs(s.t_end))));
                    s.h = xmul(s.dir, fmax(s.h, I.hmin));
                }
            } else if (s.at_t_end) {
                I.ier = 911;
            }
            if (I.ier == 1) {
                I.phase3 = 1;
                I.failed = 0;
                for (;;) {   // take_step
                    s.h = copysign(fabs(s.h), s.dir);
                    s.at_t_end = xmul(s.dir, xsub(xadd(s.t, s.h), s.t_end)) >= 0.0;
                    if (s.at_t_end) s.h = xsub(s.t_end, s.t);
                    else if (xmul(s.dir, xsub(xadd(s.t, xmul(2.0, s.h)), s.t_end)) >= 0.0) s.h = xsub(s.t_end, s.t) / 2.0;
                    I.hmin = fmax(X.Q.sqtiny, xmul(X.Q.toosml, fmax(fabs(s.t), fabs(xadd(s.t, s.h)))));
                    if (fabs(s.h) < I.hmin) { I.ier = 5; break; }
                    if (s.chkeff) {
                        s.hit_t_end_count++;
                        if (s.hit_t_end_count >= 100 && s.hit_t_end_count >= s.step_count / 3) {
                            I.ier = 2; s.hit_t_end_count = 0; break;
                        }
                    }
                    if (!I.failed) {
                        // ---------------- stiffness diagnosis (stiff_r1)
                        {
                            const int toomch = s.f_count > 5000;
                            if (toomch) { I.ier = 3; s.full_f_count += s.f_count; s.f_count = 0; }
                            I.sure = 0;
                            I.lots = 0;
                            if ((s.step_count - 10) % 40 == 0) {
                                I.lots = s.stiff_bad_step_count >= 10;
                                s.stiff_bad_step_count = 0;
                            }
                            I.maybe = toomch || I.lots;
                        }
                        if (I.maybe) {
                            {
                                double* w = X.F.weights + (size_t)b * X.n3;
                                const double* y = VPOOL(X, s.iy, b);
                                const double* yo = VPOOL(X, s.iyold, b);
                                FOR_OWN_W(X, q) w[q] = fmax(xmul(0.5, xadd(fabs(ldcg(&y[q])), fabs(ldcg(&yo[q])))), thr);
                                __syncwarp();
                                const double rat = fabs(s.h / s.h_average);
                                I.maybe = 0.2 < rat && rat < 5.0;
                                if (I.maybe) I.maybe = xmul(7.0, fabs(xsub(s.t_end, s.t) / s.h_average)) > 5000.0;
                            }
                            if (I.maybe) {
                                {
                                    const double* w = X.F.weights + (size_t)b * X.n3;
                                    const double* v0 = X.F.errest + (size_t)b * X.n3;
                                    const double* y = VPOOL(X, s.iy, b);
                                    double v[2] = {0.0, 0.0};
                                    FOR_OWN_W(X, q) {
                                        const double wq = ldcg(&w[q]);
                                        v[0] += (ldcg(&v0[q]) / wq) * (ldcg(&v0[q]) / wq);
                                        v[1] += (ldcg(&y[q]) / wq) * (ldcg(&y[q]) / wq);
                                    }
                                    post_reduce(X, I, b, v, 2, false);
                                }
                                CO_YIELD(I, L_STIFF1);
                                I.v0v0 = I.red[0];
                                I.scale = xmul(sqrt(I.red[1]), X.Q.sqrrmc);
                                if (I.scale == 0.0) { I.scale = xmul(I.v0v0, X.Q.sqrrmc); I.maybe = I.scale > 0.0; }
                            }
                        }
                        if (I.maybe) {
                            if (I.v0v0 == 0.0) {
                                {
                                    double* v0 = X.F.errest + (size_t)b * X.n3;
                                    const double* w = X.F.weights + (size_t)b * X.n3;
                                    double v = 0.0;
                                    FOR_OWN_W(X, q) { v0[q] = 1.0; const double wq = ldcg(&w[q]); v += (1.0 / wq) * (1.0 / wq); }
                                    post_reduce(X, I, b, &v, 1, false);
                                }
                                CO_YIELD(I, L_STIFF2);
                                I.v0v0 = I.red[0];
                            }
                            {
                                double* v0 = X.F.errest + (size_t)b * X.n3;
                                const double v0nrm = sqrt(I.v0v0);
                                FOR_OWN_W(X, q) v0[q] = ldcg(&v0[q]) / v0nrm;
                                __syncwarp();
                                I.v0v0 = 1.0;
                                I.rold = 0.0; I.rho = 0.0;
                                I.root_re[0] = I.root_re[1] = I.root_im[0] = I.root_im[1] = 0.0;
                                I.ntry = 1;
                            }
                            for (;;) {
                                // v1 = J v0 (approx_jacobian), wip(v1,v1), wip(v1,v0)
                                {
                                    const double temp1 = I.scale / sqrt(I.v0v0);
                                    const double* y = VPOOL(X, s.iy, b);
                                    const double* v0 = X.F.errest + (size_t)b * X.n3;
                                    FOR_OWN_W(X, q) put_arg(X, s.ia1, b, q, xadd(ldcg(&y[q]), xmul(temp1, ldcg(&v0[q]))));
                                    __syncwarp();
                                    I.tstg = temp1;
                                }
                                Y_RHS(I, L_STIFF_LOOP + 11, s.t, s.ia1, DST_STG + 2);
                                s.f_count++;
                                {
                                    const double fac = s.h_average / I.tstg;
                                    double* v1 = VSTG(X, 2, b);
                                    const double* yp = VDER(X, s.dyp, b);
                                    const double* v0 = X.F.errest + (size_t)b * X.n3;
                                    const double* w = X.F.weights + (size_t)b * X.n3;
                                    double v[2] = {0.0, 0.0};
                                    FOR_OWN_W(X, q) {
                                        const double x = xmul(fac, xsub(ldcg(&v1[q]), ldcg(&yp[q])));
                                        v1[q] = x;
                                        const double wq = ldcg(&w[q]);
                                        v[0] += (x / wq) * (x / wq);
                                        v[1] += (x / wq) * (ldcg(&v0[q]) / wq);
                                    }
                                    post_reduce(X, I, b, v, 2, false);
                                }
                                CO_YIELD(I, L_STIFF_LOOP + 12);
                                I.v1v1 = I.red[0]; I.v1v0 = I.red[1];
                                if (sqrt(I.v1v1) > 1.0e10 * sqrt(I.v0v0)) { I.maybe = 0; break; }
                                if (I.ntry == 1) {
                                    I.rold = I.v1v0 / I.v0v0;
                                    if (fabs(I.rold) < X.Q.cubrmc) { I.maybe = 0; break; }
                                } else {
                                    const double ratio = I.v1v0 / I.v0v0;
                                    I.rho = fabs(ratio);
                                    const double det = I.v0v0 * I.v1v1 - I.v1v0 * I.v1v0;
                                    const bool big = det == 0.0 || (fabs(det / I.v0v0) <= fabs(I.v1v1) * 1e-6 &&
                                                                    fabs(ratio - I.rold) <= 0.001 * I.rho);
                                    if (big) { I.root_re[0] = ratio; I.root_im[0] = 0; I.root_re[1] = 0; I.root_im[1] = 0; }
                                    I.rold = ratio;
                                    if (big) break;
                                }
                                // v2 = J v1
                                {
                                    const double temp1 = I.scale / sqrt(I.v1v1);
                                    const double* y = VPOOL(X, s.iy, b);
                                    const double* v1 = VSTG(X, 2, b);
                                    FOR_OWN_W(X, q) put_arg(X, s.ia1, b, q, xadd(ldcg(&y[q]), xmul(temp1, ldcg(&v1[q]))));
                                    __syncwarp();
                                    I.tstg = temp1;
                                }
                                Y_RHS(I, L_STIFF_LOOP + 21, s.t, s.ia1, DST_STG + 3);
                                s.f_count++;
                                {
                                    const double fac = s.h_average / I.tstg;
                                    double* v2 = VSTG(X, 3, b);
                                    const double* yp = VDER(X, s.dyp, b);
                                    const double* v0 = X.F.errest + (size_t)b * X.n3;
                                    const double* v1 = VSTG(X, 2, b);
                                    const double* w = X.F.weights + (size_t)b * X.n3;
                                    double v[3] = {0.0, 0.0, 0.0};
                                    FOR_OWN_W(X, q) {
                                        const double x = xmul(fac, xsub(ldcg(&v2[q]), ldcg(&yp[q])));
                                        v2[q] = x;
                                        const double wq = ldcg(&w[q]);
                                        v[0] += (x / wq) * (x / wq);
                                        v[1] += (x / wq) * (ldcg(&v0[q]) / wq);
                                        v[2] += (x / wq) * (ldcg(&v1[q]) / wq);
                                    }
                                    post_reduce(X, I, b, v, 3, false);
                                }
                                CO_YIELD(I, L_STIFF_LOOP + 22);
                                I.v2v2 = I.red[0]; I.v2v0 = I.red[1]; I.v2v1 = I.red[2];
                                {
                                    const double ratio = I.v2v1 / I.v1v1;
                                    I.rho = fabs(ratio);
                                    const double det = I.v1v1 * I.v2v2 - I.v2v1 * I.v2v1;
                                    const bool big = det == 0.0 || (fabs(det / I.v1v1) <= fabs(I.v2v2) * 1e-6 &&
                                                                    fabs(ratio - I.rold) <= 0.001 * I.rho);
                                    if (big) { I.root_re[0] = ratio; I.root_im[0] = 0; I.root_re[1] = 0; I.root_im[1] = 0; }
                                    I.rold = ratio;
                                    if (big) break;
                                    const double det1 = I.v0v0 * I.v1v1 - I.v1v0 * I.v1v0;
                                    I.alpha1 = (-I.v0v0 * I.v2v1 + I.v1v0 * I.v2v0) / det1;
                                    I.beta1 = (I.v1v0 * I.v2v1 - I.v1v1 * I.v2v0) / det1;
                                }
                                // v3 = J v2
                                {
                                    const double temp1 = I.scale / sqrt(I.v2v2);
                                    const double* y = VPOOL(X, s.iy, b);
                                    const double* v2 = VSTG(X, 3, b);
                                    FOR_OWN_W(X, q) put_arg(X, s.ia1, b, q, xadd(ldcg(&y[q]), xmul(temp1, ldcg(&v2[q]))));
                                    __syncwarp();
                                    I.tstg = temp1;
                                }
                                Y_RHS(I, L_STIFF_LOOP + 31, s.t, s.ia1, DST_STG + 4);
                                s.f_count++;
                                {
                                    const double fac = s.h_average / I.tstg;
                                    double* v3 = VSTG(X, 4, b);
                                    const double* yp = VDER(X, s.dyp, b);
                                    const double* v1 = VSTG(X, 2, b);
                                    const double* v2 = VSTG(X, 3, b);
                                    const double* w = X.F.weights + (size_t)b * X.n3;
                                    double v[3] = {0.0, 0.0, 0.0};
                                    FOR_OWN_W(X, q) {
                                        const double x = xmul(fac, xsub(ldcg(&v3[q]), ldcg(&yp[q])));
                                        v3[q] = x;
                                        const double wq = ldcg(&w[q]);
                                        v[0] += (x / wq) * (x / wq);
                                        v[1] += (x / wq) * (ldcg(&v1[q]) / wq);
                                        v[2] += (x / wq) * (ldcg(&v2[q]) / wq);
                                    }
                                    post_reduce(X, I, b, v, 3, false);
                                }
                                CO_YIELD(I, L_STIFF_LOOP + 32);
                                I.v3v3 = I.red[0]; I.v3v1 = I.red[1]; I.v3v2 = I.red[2];
                                {
                                    const double ratio = I.v3v2 / I.v2v2;
                                    I.rho = fabs(ratio);
                                    const double det = I.v2v2 * I.v3v3 - I.v3v2 * I.v3v2;
                                    const bool big = det == 0.0 || (fabs(det / I.v2v2) <= fabs(I.v3v3) * 1e-6 &&
                                                                    fabs(ratio - I.rold) <= 0.001 * I.rho);
                                    if (big) { I.root_re[0] = ratio; I.root_im[0] = 0; I.root_re[1] = 0; I.root_im[1] = 0; }
                                    I.rold = ratio;
                                    if (big) break;
                                    const double det2 = I.v1v1 * I.v2v2 - I.v2v1 * I.v2v1;
                                    const double alpha2 = (-I.v1v1 * I.v3v2 + I.v2v1 * I.v3v1) / det2;
                                    const double beta2 = (I.v2v1 * I.v3v2 - I.v2v2 * I.v3v1) / det2;
                                    const double res2 = fabs(I.v3v3 + alpha2 * I.v3v2 + beta2 * I.v3v1 + alpha2 * I.v3v2 +
                                                             alpha2 * alpha2 * I.v2v2 + alpha2 * beta2 * I.v2v1 + beta2 * I.v3v1 +
                                                             beta2 * alpha2 * I.v2v1 + beta2 * beta2 * I.v1v1);
                                    if (res2 <= fabs(I.v3v3) * 1e-6) {
                                        // quadratic roots (both roots as tabulated in the vendored code)
                                        double pr_re, pr_im, r_re, r_im;
                                        {
                                            const double tmp = I.alpha1 / 2.0;
                                            const double x = tmp * tmp - I.beta1;
                                            const double sgn = signbit(tmp * 0.0 + 0.0 * tmp) ? -1.0 : 1.0;
                                            const double sre = x >= 0 ? sqrt(x) : 0.0, sim = x >= 0 ? 0.0 : sgn * sqrt(-x);
                                            if (sre == 0.0 && sim == 0.0) { pr_re = -tmp; pr_im = 0.0; }
                                            else { pr_re = -tmp + sre; pr_im = sim; }
                                        }
                                        {
                                            const double tmp = alpha2 / 2.0;
                                            const double x = tmp * tmp - beta2;
                                            const double sgn = signbit(tmp * 0.0 + 0.0 * tmp) ? -1.0 : 1.0;
                                            const double sre = x >= 0 ? sqrt(x) : 0.0, sim = x >= 0 ? 0.0 : sgn * sqrt(-x);
                                            if (sre == 0.0 && sim == 0.0) { r_re = -tmp; r_im = 0.0; }
                                            else { r_re = -tmp + sre; r_im = sim; }
                                        }
                                        I.root_re[0] = I.root_re[1] = r_re;
                                        I.root_im[0] = I.root_im[1] = r_im;
                                        I.rho = hypot(pr_re, pr_im);
                                        const double dist = hypot(r_re - pr_re, r_im - pr_im);
                                        if (dist <= 0.001 * I.rho) break;
                                    }
                                }
                                I.ntry++;
                                if (I.ntry > 8) { I.maybe = 0; break; }
                                {
                                    const double v3nrm = sqrt(I.v3v3);
                                    double* v0 = X.F.errest + (size_t)b * X.n3;
                                    const double* v3 = VSTG(X, 4, b);
                                    FOR_OWN_W(X, q) v0[q] = ldcg(&v3[q]) / v3nrm;
                                    __syncwarp();
                                    I.v0v0 = 1.0;
                                }
                            }
                            if (I.maybe) {
                                if (I.root_re[0] < 0.0) {
                                    if (!(hypot(I.root_re[1], I.root_im[1]) >= 0.9 * I.rho && I.root_re[1] > 0.0)) {
                                        if (fabs(I.root_im[0]) <= fabs(I.root_re[0]) * 5.2) I.sure = I.rho >= 0.9 * 3.9;
                                    }
                                }
                            }
                        }
                        if (I.sure) I.ier = 4;
                        if (I.ier != 1) break;
                    }
                    // ---------------- step_r1 (one attempt with phase-2 restarts)
                    I.htry = s.h;
                    for (;;) {
                        if (s.phase2) {
                            double* w = X.F.weights + (size_t)b * X.n3;
                            const double* y = VPOOL(X, s.iy, b);
                            FOR_OWN_W(X, q) w[q] = fmax(thr, fabs(ldcg(&y[q])));
                            __syncwarp();
                        }
                        I.flag = 0;   // restart marker
                        for (I.i_stage = 2; I.i_stage <= 8; ++I.i_stage) {
                            {
                                const int i = I.i_stage;
                                const int argi = (i & 1) ? s.ia1 : s.ia0;
                                const double* y = VPOOL(X, s.iy, b);
                                const double* yp = VDER(X, s.dyp, b);
                                double* es = X.F.errest + (size_t)b * X.n3;
                                double lm = 0.0;
                                const uint64_t tv0 = (X.F.prof && blockIdx.x == 0 && threadIdx.x == 0) ? globaltimer_ns() : 0;
                                StgPtrs sp;
                                for (int j = 0; j < 8; ++j) sp.s[j] = (j >= 2) ? VSTG(X, j, b) : nullptr;
                                lm = stage_args(i, y, yp, sp, es, arg_dst(X, argi, b), I.htry, thr, X.lane, X.c0, X.nc);
                                if (tv0) { atomicAdd(&X.F.prof[25], globaltimer_ns() - tv0); atomicAdd(&X.F.prof[26], 1ull); }
                                if (i == 7) post_reduce(X, I, b, &lm, 1, true);
                                I.tstg = xadd(s.t, xmul(cB.c[i], I.htry));
                                if (s.at_t_end && cB.c[i] == 1.0) I.tstg = s.t_end;
                            }
                            if (I.i_stage == 7) {
                                CO_YIELD(I, L_STEPB);
                                I.err = xmul(fabs(s.h), I.red[0]);
                                if (I.err > s.tol) break;
                            }
                            Y_RHS(I, L_STAGE, I.tstg, (I.i_stage & 1) ? s.ia1 : s.ia0,
                                  I.i_stage == 8 ? DST_DERIV + s.d8 : DST_STG + I.i_stage);
                            s.f_count++;
                            if (s.phase2 && I.i_stage <= 3 && fabs(I.htry) > I.hmin) {
                                {
                                    const int argi = (I.i_stage & 1) ? s.ia1 : s.ia0;
                                    const double* yn = VPOOL(X, argi, b);
                                    const double* y = VPOOL(X, s.iy, b);
                                    const double* yp = VDER(X, s.dyp, b);
                                    const double* out = VSTG(X, I.i_stage, b);
                                    double* w = X.F.weights + (size_t)b * X.n3;
                                    double m4[4] = {0.0, 0.0, 0.0, 0.0};
                                    FOR_OWN_W(X, q) {
                                        const double ynq = ldcg(&yn[q]), yq = ldcg(&y[q]);
                                        const double wq = fmax(ldcg(&w[q]), fabs(ynq));
                                        w[q] = wq;
                                        m4[0] = fmax(m4[0], fabs(yq) / wq);
                                        m4[1] = fmax(m4[1], fabs(ynq) / wq);
                                        m4[2] = fmax(m4[2], fabs(xsub(ynq, yq)) / wq);
                                        m4[3] = fmax(m4[3], fabs(xsub(ldcg(&out[q]), ldcg(&yp[q]))) / wq);
                                    }
                                    post_reduce(X, I, b, m4, 4, true);
                                }
                                CO_YIELD(I, L_STEPA);
                                {
                                    double ynrm = I.red[0], ystgnm = I.red[1], argdif = I.red[2];
                                    const double fdiff = I.red[3];
                                    const double tdiff = xsub(I.tstg, s.t);
                                    const double twt = fabs(xsub(s.t_end, s.t));
                                    ynrm = fmax(ynrm, fabs(s.t) / twt);
                                    ystgnm = fmax(ystgnm, fabs(I.tstg) / twt);
                                    argdif = fmax(argdif, fabs(tdiff) / twt);
                                    bool cutbak = false;
                                    if (argdif > xmul(X.Q.round_off, fmax(ynrm, ystgnm))) {
                                        if (xmul(fabs(I.htry), fdiff) > xmul(3.9, argdif)) {
                                            const double scl = fmax(0.125, fmin(0.5, xmul(3.9, argdif) / xmul(fabs(I.htry), fdiff)));
                                            I.htry = xmul(scl, I.htry);
                                            cutbak = true;
                                        }
                                    }
                                    if (cutbak) {
                                        s.at_t_end = 0;
                                        if (fabs(I.htry) <= I.hmin) { I.htry = copysign(I.hmin, I.htry); s.phase2 = 0; }
                                        I.flag = 1;
                                    }
                                }
                                if (I.flag) break;
                            }
                        }
                        if (I.flag) continue;        // phase-2 restart
                        if (I.i_stage == 7) break;   // early rejection by stepb (err set)
                        {
                            const double* y = VPOOL(X, s.iy, b);
                            const double* yp = VDER(X, s.dyp, b);
                            const double* yn = VPOOL(X, s.ia0, b);
                            const double* k8 = VDER(X, s.d8, b);
                            double* es = X.F.errest + (size_t)b * X.n3;
                            double* w = X.F.weights + (size_t)b * X.n3;
                            ErrPtrs ep;
                            for (int j = 0; j < 8; ++j) ep.k[j] = (j >= 2) ? VSTG(X, j, b) : nullptr;
                            double lm = step_error(ep, y, yp, yn, k8, es, w, I.htry, thr, X.lane, X.P.n, X.c0, X.nc);
                            post_reduce(X, I, b, &lm, 1, true);
                        }
                        CO_YIELD(I, L_FINAL);
                        I.err = I.red[0];
                        break;
                    }
                    s.h = I.htry;
                    {
                        double alpha;
                        if (I.err > s.tol) {
                            if (s.at_t_start) { I.phase3 = 0; alpha = 0.5; }
                            else {
                                s.bad_step_count++;
                                s.stiff_bad_step_count++;
                                alpha = I.failed ? 0.5 : fmax(xmul(0.8, root5(s.tol / I.err)), 0.5);
                            }
                            s.h = xmul(alpha, s.h);
                            I.failed = 1;
                            continue;
                        }
                        double beta = root5(I.err / s.tol);
                        if (!s.at_t_start) {
                            const double t1 = root5(I.err) / s.h;
                            const double t2 = root5(s.errold) / s.h_old;
                            if (t1 < xmul(t2, 100.0) && t2 < xmul(t1, 100.0)) beta = xmul(beta, t1 / t2);
                        }
                        alpha = 8.0;
                        if (0.8 < xmul(beta, alpha)) alpha = 0.8 / beta;
                        if (s.at_t_start) {
                            s.phase2 = 0;
                            I.phase3 = I.phase3 && !s.at_t_end && (alpha > 4.0);
                            if (I.phase3) { s.h = xmul(alpha, s.h); continue; }
                        }
                        alpha = fmin(alpha, 2.0);
                        if (I.failed) alpha = fmin(alpha, 1.0);
                        alpha = fmax(alpha, 0.5);
                        s.h_old = s.h;
                        s.h = xmul(alpha, s.h);
                        if (s.at_t_start) s.h_average = s.h_old;
                        else s.h_average = xadd(xmul(0.9, s.h_average), xmul(0.1, s.h_old));
                        s.at_t_start = 0;
                        s.errold = I.err;
                        s.t_old = s.t;
                        if (s.at_t_end) s.t = s.t_end; else s.t = xadd(s.t, s.h_old);
                        s.step_count++;
                        const int oy = s.iy, oyo = s.iyold, oa0 = s.ia0;
                        s.iyold = oy; s.iy = oa0; s.ia0 = oyo;
                        const int dp = s.dyp, dpo = s.dypold, d8 = s.d8;
                        s.dypold = dp; s.dyp = d8; s.d8 = dpo;
                        if (X.Q.renorm) {
                            double* v = VPOOL(X, s.iy, b);
                            const int n = X.P.n;
                            for (int cell = X.lane; cell < X.nc; cell += 32) {
                                const int i = X.c0 + cell;
                                const double x = v[i], y = v[n + i], z = v[2 * n + i];
                                const double r = sqrt(xadd(xadd(xmul(x, x), xmul(y, y)), xmul(z, z)));
                                if (r > 0.0) { v[i] = x / r; v[n + i] = y / r; v[2 * n + i] = z / r; }
                            }
                            __syncwarp();
                        }
                    }
                    break;
                }
            }
            s.at_t_end = s.t == s.t_end;
            s.chkeff = s.at_t_end;
            if (I.ier == 1) { s.intrp_ready = 0; continue; }
            if (I.ier >= 911) { s.status = I.ier; s.finished = 1; break; }
            // flag 2..5: return y at the current internal time
            {
                const double* y = VPOOL(X, s.iy, b);
                double* dst = I.dst_slot ? X.F.y_out ? X.F.y_out + ((size_t)b * X.Q.nt + s.ko) * X.n3 : VONE(X, X.F.ystep, b)
                                         : VONE(X, X.F.ystep, b);
                copy_own(X, y, dst);
                I.t_got = s.t;
                I.flag = I.ier;
            }
            break;
        }
        if (s.finished) break;
        s.tlast = I.t_got;
        if (I.flag == 3) s.n_flag3++;
        if (I.flag == 4) s.n_flag4++;
        if (I.flag == 5 || I.flag == 2) s.status = I.flag;
        if (I.cf & 2) {
            {
                const double* dst = I.dst_slot ? X.F.y_out ? X.F.y_out + ((size_t)b * X.Q.nt + s.ko) * X.n3 : VONE(X, X.F.ystep, b)
                                               : VONE(X, X.F.ystep, b);
                const double* yl = VONE(X, X.F.ylast, b);
                double ce = 0.0;
                FOR_OWN_W(X, q) ce = fmax(ce, fabs(xsub(ldcg(&dst[q]), ldcg(&yl[q]))));
                post_reduce(X, I, b, &ce, 1, true);
            }
            CO_YIELD(I, L_CONV);
            {
                const double* dst = I.dst_slot ? X.F.y_out ? X.F.y_out + ((size_t)b * X.Q.nt + s.ko) * X.n3 : VONE(X, X.F.ystep, b)
                                               : VONE(X, X.F.ystep, b);
                if (I.red[0] < X.Q.conv_tol) {
                    if (s.ko < X.Q.nt) {
                        if (!I.dst_slot && X.F.y_out) copy_own(X, dst, X.F.y_out + ((size_t)b * X.Q.nt + s.ko) * X.n3);
                        if (X.cb == 0 && X.lane == 0) {
                            X.F.t_out[(size_t)b * X.Q.nt + s.ko] = I.t_got;
                            X.F.flags_out[(size_t)b * X.Q.nt + s.ko] = I.flag;
                        }
                    }
                    s.converged_at = s.ko;
                    s.finished = 1;
                    s.ci++;
                    break;
                }
                copy_own(X, dst, VONE(X, X.F.ylast, b));
            }
        }
        if (I.dst_slot) {
            if (X.cb == 0 && X.lane == 0) {
                X.F.t_out[(size_t)b * X.Q.nt + s.ko] = I.t_got;
                X.F.flags_out[(size_t)b * X.Q.nt + s.ko] = I.flag;
            }
            s.ko++;
        }
        s.ci++;
        if (s.status) { s.finished = 1; break; }
    }
    I.req = 3;
    I.pc = L_DONE;
    return;
    case L_DONE:
        I.req = 3;
        return;
    default:
        break;
    }
}

// ---------------------------------------------------------------------------
// LL epilogue for one instance on the owned cells: sum the S partial demag
// products and write f to the requested destination.
// ---------------------------------------------------------------------------
// exact demag field of cell i, instance b (int8 backend): -Ms_i 2^(-30-e_r) RN(H_int)
MT_DEV void i8_cell_field(const BCtx& X, int b, int i, double hm[3])
{
    const double ms = (double)__ldg(&X.P.Mfact[i]);
    const int k = compact_pos(X, b);
    const int jl = k / kI8N - X.jb0;
    for (int a = 0; a < 3; ++a) {
        const int r = a * X.Q.np + i;
        const double h = i8_tile_sum(X.F.part, X.Q.maxseg, X.cov[a * 3 + jl], r & 127, k % kI8N);
        hm[a] = xmul(-ms, xmul(h, __ldg(&X.Q.row_scale[r])));
    }
}

// covers of this CTA's tiles (3 components x 3 tiles from jb0; threads 0..8).
// Packed: tile j of the compact list is active tile j; otherwise act_pos maps tiles.
MT_DEV void i8_fill_cover(BCtx& X, SkCover* cov)
{
    const int k = threadIdx.x;
    if (k < 9 && X.nc > 0) {
        const int a = k / 3, jb = X.jb0 + k % 3;
        SkCover cv = {0, -1, 0};
        const int pos = X.packed ? (jb < X.nact ? jb : -1) : (jb < 2 * X.Q.IB ? X.act_pos[jb] : -1);
        if (pos >= 0) {
            const long long t = sk_tile(sk_sched_order(X.sched), pos, (a * X.Q.np + X.c0) / 128, X.nact, X.Q.RB);
            cv = sk_cover(t, X.Q.nks, X.U, sk_sched_ctas(X.sched));
        }
        cov[k] = cv;
    }
}

// copy the limbs of this CTA's share of the requesting instances to their compact rows
MT_DEV void i8_pack(const BCtx& X, int nreq, const unsigned* bits, const int* pre, int W)
{
    const int G = gridDim.x, c = blockIdx.x;
    const int k0 = (int)((long long)nreq * c / G), k1 = (int)((long long)nreq * (c + 1) / G);
    const size_t plane = (size_t)X.Q.Bp * X.Q.Kd;
    const int v16 = X.Q.Kd / 16;   // Kd is a multiple of 384
    for (int k = k0; k < k1; ++k) {
        // instance of compact position k: the word that holds it, then the bit
        int w = 0;
        while (w + 1 < W && pre[w + 1] <= k) ++w;
        unsigned m = bits[w];
        for (int r = k - pre[w]; r > 0; --r) m &= m - 1u;
        const int b = (w << 5) + (__ffs(m) - 1);
        for (int e = threadIdx.x; e < 4 * v16; e += blockDim.x) {
            const int l = e / v16, v = e - l * v16;
            const uint4* src = reinterpret_cast<const uint4*>(X.F.mlimb + l * plane + (size_t)b * X.Q.Kd) + v;
            uint4* dst = reinterpret_cast<uint4*>(X.F.mcomp + l * plane + (size_t)k * X.Q.Kd) + v;
            *dst = __ldcg(src);
        }
    }
}

MT_DEV void epilogue_cell(const BCtx& X, int b, const TimeScalars& ts, int arg, int dst, int i)
{
    const int n = X.P.n;
    const double* m = VPOOL(X, arg, b);
    double* out = dst_ptr(X, dst, b);
    if (X.Q.prec == kPrecI8) {
        double hm[3], o[3];
        i8_cell_field(X, b, i, hm);
        cell_rhs_h(X.P, m, i, hm, ts, o);
        out[i] = o[0]; out[n + i] = o[1]; out[2 * n + i] = o[2];
        return;
    }
    float S[3];
    for (int a = 0; a < 3; ++a) {
        float acc = 0.f;
        for (int sp = 0; sp < X.Q.S; ++sp) acc += ldcg(&X.F.hpart[(((size_t)sp * X.Q.Bp + b) * 3 + a) * X.Q.np + i]);
        S[a] = acc;
    }
    double o[3];
    cell_rhs(X.P, m, i, S, ts, o);
    out[i] = o[0]; out[n + i] = o[1]; out[2 * n + i] = o[2];
}

// request of one instance in the LL epilogue: the field and damping at its time, the
// argument and the destination
struct ReqDesc { TimeScalars ts; int on, arg, dst, pad; };

// LL epilogue of the int8 backend over the CTA's requesting instances.  Thread t keeps
// cell t % 128 of the block, with the cell's constants loaded once, and takes every
// fourth requesting instance; all loads of one (instance, cell) are in flight together.
// The arithmetic is that of the per-cell form (cell_rhs_h with the exact demag field).
MT_DEV void epilogue_i8(const BCtx& X, const ReqDesc* req, int* eli, int* s_nel)
{
    static_assert(kBatchThreads % kCellBlock == 0, "whole cell blocks of threads");
    constexpr int kGroups = kBatchThreads / kCellBlock;
    const int tid = threadIdx.x, cell = tid % kCellBlock, g = tid / kCellBlock;
    const int n = X.P.n;
    if (tid == 0) {
        int k = 0;
        for (int li = 0; li < X.ni; ++li)
            if (req[li].on) eli[k++] = li;
        *s_nel = k;
    }
    __syncthreads();
    const int nel = *s_nel;
    if (cell >= X.nc) return;
    const int i = X.c0 + cell;
    double rs[3], ac[7];
    int lr[3];
    const double ms = (double)__ldg(&X.P.Mfact[i]), jf = __ldg(&X.P.Jfact[i]);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        rs[a] = __ldg(&X.Q.row_scale[a * X.Q.np + i]);
        lr[a] = (a * X.Q.np + i) & 127;
    }
    aniso_load(X.P, i, ac);
    for (int le = g; le < nel; le += kGroups) {
        const int li = eli[le], b = X.i0 + li;
        const int k = compact_pos(X, b), lj = k % kI8N, jl = k / kI8N - X.jb0;
        const double* m = VPOOL(X, req[li].arg, b);
        long long hv[3][6];
        double o[3][7];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            i8_tile_load(X.F.part, X.Q.maxseg, X.cov[a * 3 + jl], lr[a], lj, hv[a]);
            lap_load(X.P, m + (size_t)a * n, i, o[a]);
        }
        const TimeScalars& ts = req[li].ts;
        double he[3], hk[3], out[3];
        aniso_from(ac, o[0][3], o[1][3], o[2][3], hk);
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const double h = i8_tile_finish(X.F.part, X.Q.maxseg, X.cov[a * 3 + jl], lr[a], lj, hv[a]);
            const double hm = xmul(-ms, xmul(h, rs[a]));
            const double hj = xmul(xmul(-2.0, lap_from(X.P, o[a], i)), jf);
            const double hh = -(a == 0 ? ts.hx : a == 1 ? ts.hy : ts.hz);
            he[a] = xadd(xadd(xadd(hh, hj), hm), hk[a]);
        }
        ll_from_heff(X.P, o[0][3], o[1][3], o[2][3], he, ts.alpha, out);
        double* d = dst_ptr(X, req[li].dst, b);
        d[i] = out[0]; d[n + i] = out[1]; d[2 * n + i] = out[2];
    }
}

// ---------------------------------------------------------------------------
// FP32 SIMT demag tile: H[s][inst][a][cell] for cells of block cb, instances of
// block ib, sources of split s, from the cell-row FP32 tensor.
// ---------------------------------------------------------------------------
constexpr int kSimtJT = 16;

MT_DEV void gemm_tile_simt(const BCtx& X)
{
    const int ldk = X.P.ldk, n = X.P.n;
    float* Ks = reinterpret_cast<float*>(X.smem);        // [6][JT][128]
    float* Ms = Ks + 6 * kSimtJT * kCellBlock;             // [JT][3][64]
    const int tid = threadIdx.x;
    const int tc = tid & 31, ti = tid >> 5;                // 32 cell groups x 16 instance groups
    const int cbase = X.cb * kCellBlock;
    for (int half = 0; half < kInstBlock / 64; ++half) {
    const int ibase = X.ib * kInstBlock + half * 64;
    const int j4tot = ldk >> 2;
    const int js = (int)(((long long)j4tot * X.s) / X.Q.S) * 4;
    const int je = (int)(((long long)j4tot * (X.s + 1)) / X.Q.S) * 4;
    float acc[4][4][3];
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int r = 0; r < 4; ++r) acc[q][r][0] = acc[q][r][1] = acc[q][r][2] = 0.f;
    for (int j0 = js; j0 < je; j0 += kSimtJT) {
        const int len = min(kSimtJT, je - j0);   // multiple of 4
        __syncthreads();
        // K rows: 128 cells x 6 comps x len floats
        for (int e = tid; e < kCellBlock * 6 * (kSimtJT / 4); e += blockDim.x) {
            const int cell = e / (6 * (kSimtJT / 4));
            const int rem = e - cell * 6 * (kSimtJT / 4);
            const int c = rem / (kSimtJT / 4), j4 = rem - c * (kSimtJT / 4);
            float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
            if (cbase + cell < n && 4 * j4 < len)
                v = __ldg(reinterpret_cast<const float4*>(X.P.K + ((size_t)(cbase + cell) * 6 + c) * ldk + j0) + j4);
            float* d = Ks + (c * kSimtJT + 4 * j4) * kCellBlock + cell;
            d[0] = v.x; d[kCellBlock] = v.y; d[2 * kCellBlock] = v.z; d[3 * kCellBlock] = v.w;
        }
        for (int e = tid; e < 64 * 3 * (kSimtJT / 4); e += blockDim.x) {
            const int inst = e / (3 * (kSimtJT / 4));
            const int rem = e - inst * 3 * (kSimtJT / 4);
            const int bb = rem / (kSimtJT / 4), j4 = rem - bb * (kSimtJT / 4);
            float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
            if (4 * j4 < len)
                v = __ldcg(reinterpret_cast<const float4*>(X.F.m32 + ((size_t)(ibase + inst) * 3 + bb) * ldk + j0) + j4);
            float* d = Ms + ((4 * j4) * 3 + bb) * 64 + inst;
            d[0] = v.x; d[3 * 64] = v.y; d[6 * 64] = v.z; d[9 * 64] = v.w;
        }
        __syncthreads();
        for (int jj = 0; jj < len; ++jj) {
            float kv[4][6], mv[4][3];
#pragma unroll
            for (int q = 0; q < 4; ++q)
#pragma unroll
                for (int c = 0; c < 6; ++c) kv[q][c] = Ks[(c * kSimtJT + jj) * kCellBlock + tc + 32 * q];
#pragma unroll
            for (int r = 0; r < 4; ++r)
#pragma unroll
                for (int bb = 0; bb < 3; ++bb) mv[r][bb] = Ms[(jj * 3 + bb) * 64 + ti + 16 * r];
#pragma unroll
            for (int q = 0; q < 4; ++q)
#pragma unroll
                for (int r = 0; r < 4; ++r) {
                    // explicit FMAs: this file is compiled without contraction (the FP64
                    // coroutine arithmetic must round every operation like the oracle)
                    acc[q][r][0] = __fmaf_rn(kv[q][0], mv[r][0], acc[q][r][0]);
                    acc[q][r][0] = __fmaf_rn(kv[q][1], mv[r][1], acc[q][r][0]);
                    acc[q][r][0] = __fmaf_rn(kv[q][2], mv[r][2], acc[q][r][0]);
                    acc[q][r][1] = __fmaf_rn(kv[q][1], mv[r][0], acc[q][r][1]);
                    acc[q][r][1] = __fmaf_rn(kv[q][3], mv[r][1], acc[q][r][1]);
                    acc[q][r][1] = __fmaf_rn(kv[q][4], mv[r][2], acc[q][r][1]);
                    acc[q][r][2] = __fmaf_rn(kv[q][2], mv[r][0], acc[q][r][2]);
                    acc[q][r][2] = __fmaf_rn(kv[q][4], mv[r][1], acc[q][r][2]);
                    acc[q][r][2] = __fmaf_rn(kv[q][5], mv[r][2], acc[q][r][2]);
                }
        }
    }
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int r = 0; r < 4; ++r)
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                const int cell = cbase + tc + 32 * q, inst = ibase + ti + 16 * r;
                X.F.hpart[(((size_t)X.s * X.Q.Bp + inst) * 3 + a) * X.Q.np + cell] = acc[q][r][a];
            }
    __syncthreads();
    }
}

constexpr int kMaxInstPerWarp = 8;

// Estimated work of advancing a served coroutine to its next request, in FP64 vectors its
// loops stream: after stage i of a step the stage-(i+1) argument (i + 2 vectors); after
// the last stage the error estimate, the step's end and the next step's first argument;
// after an interpolation stage the next one, or the interpolant and its outputs.
MT_DEV int advance_weight(const BInst& I)
{
    if (I.pc == L_STAGE) return I.i_stage >= 8 ? 24 : I.i_stage + 3;
    if (I.pc >= L_INTERP + 1000) return 16;
    return 8;
}

// Publish the state of the warp's coroutines for tick tk: active instances and
// right-hand-side requests (per 64-instance tile, and as request bits for the int8
// packing), counted once per instance by its cell block 0.  Slot tk % 3 was cleared
// by CTA 0 after the first barrier of tick tk - 1 (or by the host before the
// launch), and is read after the first barrier of tick tk.
MT_DEV void publish_requests(const BInst* L, int mine, const BCtx& X, int W, bool i8, long long tk)
{
    const BatchParams& Q = X.Q;
    const BatchBufs& F = X.F;
    int my_active = 0, my_rhs = 0;
    int rhs_tile[2] = {0, 0};   // requests per 64-instance tile, tiles jb0 and jb0 + 1
    for (int k = 0; k < mine; ++k) {
        const int req = L[k].req;
        const int b = X.i0 + X.warp + k * X.nwarps;
        if (b >= Q.B) continue;
        if (req != 3 && req != 4) my_active++;
        if (req == 1) {
            my_rhs++;
            rhs_tile[(b / kI8N - X.i0 / kI8N) & 1]++;
            if (i8 && X.cb == 0 && X.lane == 0) atomicOr(&F.reqbits[(tk % 3) * W + (b >> 5)], 1u << (b & 31));
        }
    }
    if (X.lane == 0 && X.cb == 0 && (my_active | my_rhs)) {
        unsigned* c = F.counters + 2 * (tk % 3);
        atomicAdd(&c[0], (unsigned)my_active);
        atomicAdd(&c[1], (unsigned)my_rhs);
        for (int h = 0; h < 2; ++h)
            if (rhs_tile[h]) atomicAdd(&F.ibreq[(tk % 3) * 2 * Q.IB + X.i0 / kI8N + h], (unsigned)rhs_tile[h]);
    }
}


__global__ void __launch_bounds__(kBatchThreads, 1)
batch_kernel(DevProb P, BatchBufs F, BatchParams Q, const __grid_constant__ TcMaps maps)
{
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    BCtx X;
    X.P = P; X.F = F; X.Q = Q;
    const int t = blockIdx.x;
    X.s = t % Q.S;
    X.ib = (t / Q.S) % Q.IB;
    X.cb = t / (Q.S * Q.IB);
    const bool owner = X.cb < Q.CB;    // CTAs past CB x IB x S only take GEMM work (int8 backend)
    X.c0 = owner ? X.cb * kCellBlock : 0;
    X.nc = owner ? min(kCellBlock, P.n - X.c0) : 0;
    const int per = kInstBlock / Q.S;
    X.i0 = X.ib * kInstBlock + X.s * per;
    X.ni = owner ? per : 0;
    X.nact = 0;
    X.U = 0;
    __shared__ int s_act[2 * kMaxIB], s_actpos[2 * kMaxIB];
    __shared__ SkCover s_cov[9];
    __shared__ unsigned s_bits[4 * kMaxIB];
    __shared__ int s_pre[4 * kMaxIB + 1];
    X.act_pos = s_actpos;
    X.jb0 = X.i0 / kI8N;
    X.cov = s_cov;
    X.packed = false;
    X.sched = 0;
    X.prev_valid = false;
    X.bits = s_bits;
    X.pre = s_pre;
    const int W = Q.Bp / 32;
    X.n3 = 3 * (size_t)P.n;
    X.lane = threadIdx.x & 31;
    X.warp = threadIdx.x >> 5;
    X.nwarps = blockDim.x >> 5;
    X.smem = smem_raw;
    const bool i8 = Q.prec == kPrecI8;
    const bool tc = Q.prec != kPrecFP32 && !i8;
    __shared__ ReqDesc s_req[kInstBlock];
    __shared__ int s_eli[kInstBlock], s_nel;
    TcState tcs;
    tcs.kb_done = 0; tcs.tiles = 0; tcs.tmem = 0;
    if (tc) tc_init_impl(X.smem, tcs);
    if (i8) tc_i8_init(X.smem, tcs);
    // The coroutines of a warp: one copy per warp in shared memory when the CTA's copies
    // fit next to the GEMM's buffers (every lane reads and writes the same, identical
    // values), otherwise one copy per lane in local memory.
    BInst L_loc[kMaxInstPerWarp];
    BInst* Lsm = Q.inst_smem_off ? reinterpret_cast<BInst*>(smem_raw + Q.inst_smem_off) : nullptr;
    BInst* L = Lsm ? Lsm + (size_t)X.warp * Q.inst_per_warp : L_loc;
    __shared__ int s_adv[kInstBlock], s_adv_w[kInstBlock], s_wt[kInstBlock], s_nadv;
    int mine = 0;
    for (int li = X.warp; li < X.ni && mine < kMaxInstPerWarp; li += X.nwarps, ++mine) {
        const long long* src = reinterpret_cast<const long long*>(&F.inst[(size_t)X.cb * Q.Bp + X.i0 + li]);
        long long* dst = reinterpret_cast<long long*>(&L[mine]);
        if (Q.inst_smem_off) {
            for (int w = X.lane; w < (int)(sizeof(BInst) / 8); w += 32) dst[w] = __ldcg(src + w);
            __syncwarp();
        } else {
            for (int w = 0; w < (int)(sizeof(BInst) / 8); ++w) dst[w] = __ldcg(src + w);
        }
        if (L[mine].req == 4) L[mine].req = 0;                 // parked by the previous launch
        L[mine].red_seq = 0;                                   // the arrival counters start at zero
        L[mine].budget_mark = L[mine].s.full_f_count + L[mine].s.f_count + Q.evals_budget;
    }
    __syncwarp();
    bool ok = true;
    if (Q.demag_only) {
        // one product of the operands already in place, then H = -Ms * sum of partials
        if (i8) {
            const int JB = Q.Bp / kI8N;
            for (int k = threadIdx.x; k < JB; k += blockDim.x) { s_act[k] = k; s_actpos[k] = k; }
            __syncthreads();
            X.nact = Q.tune_nact > 0 ? Q.tune_nact : JB;
            X.U = (long long)X.nact * Q.RB * Q.nks;
            X.sched = Q.tune_sched ? Q.tune_sched : Q.sk_sched[X.nact];
            if (Q.tune_nact == 0) i8_fill_cover(X, s_cov);
            ok = tc_i8_streamk(X.smem, F, F.part, Q.maxseg, maps, &maps.bhi, X.nact, s_act, Q.RB, Q.nks, X.sched, tcs);
            if (Q.tune_nact > 0) {   // schedule timing: the product only
                tc_finish_impl(X.smem, tcs);
                return;
            }
        } else if (!tc) {
            gemm_tile_simt(X);
        } else {
            ok = tc_gemm_tile_impl(X.smem, Q, F, maps, X.cb, X.ib, X.s, Q.prec != kPrecBF16x2,
                                   Q.prec == kPrecFP16x3S, Q.prec == kPrecFP16x3S ? Q.row_inv : nullptr, tcs);
        }
        if (ok && grid_sync(F.gs, 5)) {
            const int n = P.n;
            for (int e = threadIdx.x; e < X.ni * 3 * X.nc; e += blockDim.x) {
                const int li = e / (3 * X.nc), rem = e - li * 3 * X.nc;
                const int a = rem / X.nc, i = X.c0 + (rem - a * X.nc);
                const int b = X.i0 + li;
                if (b >= Q.B) continue;
                double h;
                if (i8) {
                    const int r = a * Q.np + i;
                    const double v = i8_tile_sum(F.part, Q.maxseg, s_cov[a * 3 + b / kI8N - X.jb0], r & 127, b % kI8N);
                    h = xmul(-(double)__ldg(&P.Mfact[i]), xmul(v, __ldg(&Q.row_scale[r])));
                } else {
                    float acc = 0.f;
                    for (int sp = 0; sp < Q.S; ++sp)
                        acc += __ldcg(&F.hpart[(((size_t)sp * Q.Bp + b) * 3 + a) * Q.np + i]);
                    h = (double)__fmul_rn(-acc, __ldg(&P.Mfact[i]));
                }
                Q.out_h[(size_t)b * 3 * n + (size_t)a * n + i] = h;
            }
        }
        if (tc || i8) tc_finish_impl(X.smem, tcs);
        return;
    }
    const bool prof = F.prof != nullptr && threadIdx.x == 0;
    unsigned long long acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    uint64_t tp = prof ? globaltimer_ns() : 0;
#define PROF_MARK(k)                                       \
    do {                                                   \
        if (prof) {                                        \
            const uint64_t _n = globaltimer_ns();          \
            acc[k] += _n - tp;                             \
            tp = _n;                                       \
        }                                                  \
    } while (0)
    long long ticks_run = 0;
    unsigned long long hist_ns[5] = {0, 0, 0, 0, 0}, hist_n[5] = {0, 0, 0, 0, 0};   // ticks by active tiles
    // Each tick: A advance every coroutine whose request was served (and, in the first
    // tick of a launch, those starting or resumed after a budget stop) to its next
    // request, resolving reductions on the way, and publish the requests; B1; the
    // demag product of the requesting instances; Bh; the LL epilogue of those
    // instances.  Requests still pending when a launch ends are served by the next.
    for (long long tick = 0; ok; ++tick) {
        const uint64_t t_tick = prof ? globaltimer_ns() : 0;
        if (Lsm) {
            // Every coroutine of the CTA is in shared memory: the ones to advance are dealt to
            // the warps in index order, so a thinned-out set still keeps every warp busy.  The
            // order is the same in every cell-block copy of the instances (their states are
            // identical), so the in-place reductions wait on copies that run in the same order.
            __syncthreads();
            if (X.warp == 0) {
                int cnt = 0;
                for (int c = 0; c < X.ni; c += 32) {
                    const int li = c + X.lane;
                    const bool need = li < X.ni && X.i0 + li < Q.B &&
                                      Lsm[(li % X.nwarps) * Q.inst_per_warp + li / X.nwarps].req == 0;
                    const unsigned bal = __ballot_sync(0xffffffffu, need);
                    if (need) s_adv_w[cnt + __popc(bal & ((1u << X.lane) - 1u))] = li;
                    cnt += __popc(bal);
                }
                __syncwarp();
                // Heaviest first: each coroutine's work up to its next request, estimated from
                // where it resumes (the vectors its next loops stream), ranks the served ones;
                // ties keep index order.  The states, and so the order, are the same in every
                // cell-block copy of the instances.
                for (int k = X.lane; k < cnt; k += 32) s_wt[k] = advance_weight(Lsm[(s_adv_w[k] % X.nwarps) *
                                                                                    Q.inst_per_warp + s_adv_w[k] / X.nwarps]);
                __syncwarp();
                for (int k = X.lane; k < cnt; k += 32) {
                    int r = 0;
                    for (int o = 0; o < cnt; ++o)
                        r += (s_wt[o] > s_wt[k]) || (s_wt[o] == s_wt[k] && o < k);
                    s_adv[r] = s_adv_w[k];
                }
                if (X.lane == 0) s_nadv = cnt;
            }
            __syncthreads();
            // dealt in snake order (warp w takes ranks w, 2 nw - 1 - w, 2 nw + w, ...), so a
            // warp's heavy coroutine of one round pairs with a light one of the next
            for (int r = 0; r * X.nwarps < s_nadv; ++r) {
                const int j = r * X.nwarps + ((r & 1) ? X.nwarps - 1 - X.warp : X.warp);
                if (j >= s_nadv) continue;
                const int li = s_adv[j];
                BInst& I = Lsm[(li % X.nwarps) * Q.inst_per_warp + li / X.nwarps];
                const uint64_t ta = (F.prof && t == 0 && threadIdx.x == 0) ? globaltimer_ns() : 0;
                ADVANCE_TO_REQUEST(X, I, X.i0 + li);
                if (ta) { atomicAdd(&F.prof[27], globaltimer_ns() - ta); atomicAdd(&F.prof[28], 1ull); }
            }
            __syncthreads();
        } else {
            for (int k = 0; k < mine; ++k) {
                BInst& I = L[k];
                const int b = X.i0 + X.warp + k * X.nwarps;
                if (b >= Q.B || I.req != 0) continue;
                const uint64_t ta = (F.prof && t == 0 && threadIdx.x == 0) ? globaltimer_ns() : 0;
                ADVANCE_TO_REQUEST(X, I, b);
                if (ta) { atomicAdd(&F.prof[27], globaltimer_ns() - ta); atomicAdd(&F.prof[28], 1ull); }
            }
        }
        if (tick >= Q.ticks_per_launch) break;
        publish_requests(L, mine, X, W, i8, tick);
        asm volatile("fence.proxy.async.global;" ::: "memory");   // operand stores -> TMA reads
        __syncthreads();
        PROF_MARK(4);
        unsigned* ctr = F.counters + 2 * (tick % 3);
        ticks_run++;
        if (!grid_sync(F.gs, 1)) { ok = false; break; }
        PROF_MARK(1);
        const unsigned active = __ldcg(&ctr[0]);
        // requests in this CTA's 128-instance block (its two 64-instance tiles)
        const unsigned nreq = __ldcg(&F.ibreq[(tick % 3) * 2 * Q.IB + 2 * X.ib]) +
                              __ldcg(&F.ibreq[(tick % 3) * 2 * Q.IB + 2 * X.ib + 1]);
        if (t == 0 && threadIdx.x == 0) {
            unsigned* nxt = F.counters + 2 * ((tick + 1) % 3);
            nxt[0] = 0; nxt[1] = 0;
            for (int k = 0; k < 2 * Q.IB; ++k) F.ibreq[((tick + 1) % 3) * 2 * Q.IB + k] = 0;
            if (i8) for (int w = 0; w < W; ++w) F.reqbits[((tick + 1) % 3) * W + w] = 0u;
        }
        if (active == 0) break;
        if (i8) {
            // requesting instances, packed in index order: every CTA builds the same prefix table,
            // copies its share of their operand rows to the compact buffer, then the GEMM runs
            // over ceil(requests / 64) tiles of that buffer
            // Every active instance requests a right-hand side in every tick (norms resolve
            // in place), so the set of requests only shrinks within a launch: the same count
            // as in the previous tick means the same set, and the coroutines have already
            // written their rows at their compact positions (put_arg).  Otherwise pack.
            const int nr_prev = X.prev_valid ? s_pre[W] : -1;
            __syncthreads();
            for (int w = threadIdx.x; w < W; w += blockDim.x) s_bits[w] = __ldcg(&F.reqbits[(tick % 3) * W + w]);
            __syncthreads();
            if (threadIdx.x == 0) {
                int acc = 0;
                for (int w = 0; w < W; ++w) { s_pre[w] = acc; acc += __popc(s_bits[w]); }
                s_pre[W] = acc;
            }
            __syncthreads();
            const int nr = s_pre[W];
            const bool same = nr == nr_prev;
            X.packed = true;
            X.nact = (nr + kI8N - 1) / kI8N;
            X.U = (long long)X.nact * Q.RB * Q.nks;
            X.sched = Q.sk_sched[X.nact];
            // first compact position among this CTA's requesting instances
            {
                int first = 1 << 30;
                for (int li = 0; li < X.ni; ++li) {
                    const int b = X.i0 + li;
                    if (b < Q.B && ((s_bits[b >> 5] >> (b & 31)) & 1u)) { first = compact_pos(X, b); break; }
                }
                X.jb0 = first < (1 << 30) ? first / kI8N : 0;
            }
            i8_fill_cover(X, s_cov);   // read in the epilogue, after the barrier that follows the GEMM
            if (!same) {
                i8_pack(X, nr, s_bits, s_pre, W);
                asm volatile("fence.proxy.async.global;" ::: "memory");   // packed rows -> TMA reads
                __syncthreads();
                if (!grid_sync(F.gs, 6)) { ok = false; break; }
            }
            X.prev_valid = true;
            for (int k = threadIdx.x; k < X.nact; k += blockDim.x) s_act[k] = k;
            __syncthreads();
            if (X.nact > 0 && !tc_i8_streamk(X.smem, F, F.part, Q.maxseg, maps, &maps.blo, X.nact, s_act, Q.RB, Q.nks,
                                             X.sched, tcs))
                ok = false;
        } else if (nreq > 0) {
            if (!tc) gemm_tile_simt(X);
            else if (!tc_gemm_tile_impl(X.smem, Q, F, maps, X.cb, X.ib, X.s, Q.prec != kPrecBF16x2,
                                        Q.prec == kPrecFP16x3S, Q.prec == kPrecFP16x3S ? Q.row_inv : nullptr, tcs))
                ok = false;
        }
        __syncthreads();
        PROF_MARK(2);
        if (!grid_sync(F.gs, 2)) { ok = false; break; }
        PROF_MARK(3);
        if (!ok) break;
        // LL epilogue of every requesting instance on the owned cells, spread over all threads
        for (int k = 0; k < mine; ++k) {
            const BInst& I = L[k];
            if (X.lane == 0) {
                const int li = X.warp + k * X.nwarps;
                const bool on = X.i0 + li < Q.B && I.req == 1;
                s_req[li].on = on ? 1 : 0;
                s_req[li].arg = I.rhs_arg;
                s_req[li].dst = I.rhs_dst;
                // field and damping of the instance at the request time, once per instance
                if (on) s_req[li].ts = inst_scalars(X, X.i0 + li, I.t_rhs);
            }
        }
        __syncthreads();
        if (i8) {
            epilogue_i8(X, s_req, s_eli, &s_nel);
        } else {
            for (int e = threadIdx.x; e < X.ni * X.nc; e += blockDim.x) {
                const int li = e / X.nc, cell = e - li * X.nc;
                if (!s_req[li].on) continue;
                epilogue_cell(X, X.i0 + li, s_req[li].ts, s_req[li].arg, s_req[li].dst, X.c0 + cell);
            }
        }
        __syncthreads();
        for (int k = 0; k < mine; ++k)   // served: the next tick resumes these coroutines
            if (L[k].req == 1 && X.i0 + X.warp + k * X.nwarps < Q.B) L[k].req = 0;
        PROF_MARK(6);
        if (prof && i8) {
            const int k = X.nact < 4 ? X.nact : 4;
            hist_ns[k] += globaltimer_ns() - t_tick;
            hist_n[k]++;
        }
    }
    if (prof) {
        if (t == 0) {
            for (int k = 0; k < 7; ++k) atomicAdd(&F.prof[k], acc[k]);
            atomicAdd(&F.prof[7], (unsigned long long)ticks_run);
            for (int k = 0; k < 5; ++k) { atomicAdd(&F.prof[32 + k], hist_ns[k]); atomicAdd(&F.prof[37 + k], hist_n[k]); }
        }
        // busiest CTA per work phase (P2, GEMM, P1): value and CTA index
        const int work[3] = {0, 2, 4};
        for (int k = 0; k < 3; ++k) {
            const unsigned long long v = acc[work[k]];
            const unsigned long long old = atomicMax(&F.prof[8 + k], v);
            if (v > old) F.prof[12 + k] = (unsigned long long)t;
        }
    }
#undef PROF_MARK
    if (tc || i8) tc_finish_impl(X.smem, tcs);
    if (ok && X.lane == 0) {
        for (int k = 0; k < mine; ++k) {
            const int li = X.warp + k * X.nwarps;
            long long* dst = reinterpret_cast<long long*>(&F.inst[(size_t)X.cb * Q.Bp + X.i0 + li]);
            const long long* src = reinterpret_cast<const long long*>(&L[k]);
            for (int w = 0; w < (int)(sizeof(BInst) / 8); ++w) dst[w] = src[w];
        }
    }
}

// power-of-two row scale for the fp16s tensor: largest |K| of row r into [2^13, 2^14)
__global__ void row_scale_kernel(const float* __restrict__ K, int n, int ldk, int np, float* __restrict__ row_inv)
{
    const int row = blockIdx.x;          // (a, i) row of the 3np x 3np matrix
    const int a = row / np, i = row - a * np;
    static const int blk[3][3] = {{0, 1, 2}, {1, 3, 4}, {2, 4, 5}};
    float mx = 0.f;
    if (i < n)
        for (int bb = 0; bb < 3; ++bb)
            for (int j = threadIdx.x; j < n; j += blockDim.x)
                mx = fmaxf(mx, fabsf(K[((size_t)i * 6 + blk[a][bb]) * ldk + j]));
    __shared__ float red[32];
    for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = mx;
    __syncthreads();
    if (threadIdx.x == 0) {
        float m = 0.f;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) m = fmaxf(m, red[w]);
        int e = 0;
        if (m > 0.f) { frexpf(m, &e); }          // m = f * 2^e, f in [0.5, 1)
        const int shift = (m > 0.f) ? 14 - e : 0;  // m * 2^shift in [2^13, 2^14)
        row_inv[row] = ldexpf(1.0f, -shift);
    }
}

// FP32 cell-row tensor -> 16-bit hi/lo [3np][Kd] (rows (a,i), cols (b,j)), zero padded;
// fp16s rows are multiplied by 1/row_inv first
__global__ void split_tensor_kernel(const float* __restrict__ K, int n, int ldk, int np, int prec,
                                    const float* __restrict__ row_inv, uint16_t* __restrict__ khi,
                                    uint16_t* __restrict__ klo)
{
    const int Kd = 3 * np;
    const size_t tot = (size_t)Kd * Kd;
    static const int blk[3][3] = {{0, 1, 2}, {1, 3, 4}, {2, 4, 5}};
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < tot; e += (size_t)gridDim.x * blockDim.x) {
        const int row = (int)(e / Kd), col = (int)(e - (size_t)row * Kd);
        const int a = row / np, i = row - a * np, bb = col / np, j = col - bb * np;
        float v = 0.f;
        if (i < n && j < n) v = K[((size_t)i * 6 + blk[a][bb]) * ldk + j];
        if (prec == kPrecFP16x3S) v = v / row_inv[row];   // exact: power of two
        split_store(v, prec, khi + e, klo + e);
    }
}

// int8 tensor rows: 2^e_r puts the largest |K| of row r into [2^29, 2^30);
// row_scale[r] = 2^(-30 - e_r) converts the exact limb sum back (0 for empty rows)
__global__ void i8_row_kernel(const float* __restrict__ K, int n, int ldk, int np, int* __restrict__ row_exp,
                              double* __restrict__ row_scale)
{
    const int row = blockIdx.x;
    const int a = row / np, i = row - a * np;
    static const int blk[3][3] = {{0, 1, 2}, {1, 3, 4}, {2, 4, 5}};
    float mx = 0.f;
    if (i < n)
        for (int bb = 0; bb < 3; ++bb)
            for (int j = threadIdx.x; j < n; j += blockDim.x)
                mx = fmaxf(mx, fabsf(K[((size_t)i * 6 + blk[a][bb]) * ldk + j]));
    __shared__ float red[32];
    for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = mx;
    __syncthreads();
    if (threadIdx.x == 0) {
        float m = 0.f;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) m = fmaxf(m, red[w]);
        int e = 0;
        if (m > 0.f) frexpf(m, &e);                // m = f 2^e, f in [0.5, 1)
        const int ex = (m > 0.f) ? 30 - e : 0;     // m 2^ex in [2^29, 2^30)
        row_exp[row] = ex;
        row_scale[row] = (m > 0.f) ? ldexp(1.0, -30 - ex) : 0.0;
    }
}

// FP32 cell-row tensor -> four int8 limbs [4][3np][Kd] of Kq = rint(K 2^e_r),
// Kq = k0 2^24 + k1 2^16 + k2 2^8 + k3 (signed digits, k3 lowest), zero padded
__global__ void i8_limb_kernel(const float* __restrict__ K, int n, int ldk, int np, const int* __restrict__ row_exp,
                               int8_t* __restrict__ klimb)
{
    const int Kd = 3 * np;
    const size_t tot = (size_t)Kd * Kd;
    static const int blk[3][3] = {{0, 1, 2}, {1, 3, 4}, {2, 4, 5}};
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < tot; e += (size_t)gridDim.x * blockDim.x) {
        const int row = (int)(e / Kd), col = (int)(e - (size_t)row * Kd);
        const int a = row / np, i = row - a * np, bb = col / np, j = col - bb * np;
        float v = 0.f;
        if (i < n && j < n) v = K[((size_t)i * 6 + blk[a][bb]) * ldk + j];
        long long x = __double2ll_rn(ldexp((double)v, row_exp[row]));
#pragma unroll
        for (int l = 3; l >= 1; --l) {
            const int d = (int)(signed char)(x & 0xff);
            klimb[(size_t)l * tot + e] = (int8_t)d;
            x = (x - d) >> 8;
        }
        klimb[e] = (int8_t)x;
    }
}

// m (B x 3n FP64) -> GEMM operand of every instance
__global__ void batch_operand_kernel(const double* __restrict__ m, int B, int n, int ldk, int np, int prec,
                                     float* __restrict__ m32, uint16_t* __restrict__ mhi, uint16_t* __restrict__ mlo,
                                     int8_t* __restrict__ mlimb, int Bp, GridSync* gs)
{
    const size_t tot = (size_t)B * 3 * n;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < tot; e += (size_t)gridDim.x * blockDim.x) {
        const int b = (int)(e / (3 * (size_t)n));
        const int q = (int)(e - (size_t)b * 3 * n);
        const int a = q / n, i = q - a * n;
        const float f = (float)m[e];
        if (prec == kPrecI8) {
            i8_store_m(m[e], mlimb + (size_t)b * 3 * np + (size_t)a * np + i, (size_t)Bp * 3 * np, gs);
        } else if (prec == kPrecFP32) {
            m32[((size_t)b * 3 + a) * ldk + i] = f;
        } else {
            const size_t col = (size_t)b * 3 * np + (size_t)a * np + i;
            split_store(f, prec, mhi + col, mlo + col);
        }
    }
}

}  // namespace

static void bs45b_fill(BS45b& T);

cudaError_t launch_batch_operand(const double* m, int B, int n, int ldk, int np, int prec, float* m32, uint16_t* mhi,
                                 uint16_t* mlo, int8_t* mlimb, int Bp, GridSync* gs, cudaStream_t s)
{
    batch_operand_kernel<<<592, 256, 0, s>>>(m, B, n, ldk, np, prec, m32, mhi, mlo, mlimb, Bp, gs);
    return cudaGetLastError();
}

cudaError_t launch_limb_tensor(const float* K, int n, int ldk, int np, int8_t* klimb, double* row_scale,
                               cudaStream_t s)
{
    int* row_exp = nullptr;
    cudaError_t e = cudaMallocAsync(&row_exp, sizeof(int) * 3 * (size_t)np, s);
    if (e != cudaSuccess) return e;
    i8_row_kernel<<<3 * np, 256, 0, s>>>(K, n, ldk, np, row_exp, row_scale);
    e = cudaGetLastError();
    if (e == cudaSuccess) {
        i8_limb_kernel<<<1184, 256, 0, s>>>(K, n, ldk, np, row_exp, klimb);
        e = cudaGetLastError();
    }
    cudaError_t e2 = cudaFreeAsync(row_exp, s);
    return e != cudaSuccess ? e : e2;
}

// slots per CTA: the longest Stream-K range (all instance tiles active) spans
// at most ceil(len / nks) + 1 tiles
int batch_i8_maxseg(int RB, int nks, int JB, int G)
{
    const long long U = (long long)RB * nks * JB;
    const long long len = (U + G - 1) / G;
    return (int)((len + nks - 1) / nks) + 1;
}

cudaError_t batch_upload_tables()
{
    static BS45b T;
    bs45b_fill(T);
    return cudaMemcpyToSymbol(cB, &T, sizeof(T));
}

int batch_grid(int n, int B, int num_sms, int prec, int* CB, int* IB, int* S)
{
    *CB = (n + kCellBlock - 1) / kCellBlock;
    *IB = (B + kInstBlock - 1) / kInstBlock;
    const int tiles = (*CB) * (*IB);
    int s = num_sms / tiles;
    if (s > 4) s = 4;
    if (s < 1) s = 1;
    if (s == 3) s = 2;   // every split owns kInstBlock / s instances: s divides 128
    // the source range of every split is a whole number of 32-wide k-blocks
    const int Kd = 3 * (*CB) * kCellBlock;
    while (s > 1 && (Kd % (32 * s)) != 0) --s;
    *S = s;
    // int8: the coroutine owners as above, the Stream-K GEMM on every SM
    if (prec == kPrecI8 && tiles * s < num_sms) return num_sms;
    return tiles * s;
}

size_t batch_smem_bytes(int n, int ldk, int prec)
{
    (void)n; (void)ldk;
    if (prec == kPrecI8) return tc_i8_smem_bytes();
    return prec == kPrecFP32 ? (size_t)(6 * kSimtJT * kCellBlock + kSimtJT * 3 * 64) * sizeof(float)
                             : tc_smem_bytes();
}

// where the coroutine copies go in dynamic shared memory (0: local memory) and how much
// they add, for per_cta instances per CTA on kBatchThreads threads
size_t batch_inst_smem(int n, int ldk, int prec, int per_cta, int* off, int* per_warp)
{
    const int nw = kBatchThreads / 32;
    *per_warp = (per_cta + nw - 1) / nw;
    const size_t base = (batch_smem_bytes(n, ldk, prec) + 127) & ~(size_t)127;
    const size_t bytes = (size_t)nw * (*per_warp) * sizeof(BInst);
    constexpr size_t kStaticBudget = 12 * 1024;   // the kernel's static shared memory, rounded up
    if (*per_warp > kMaxInstPerWarp || base + bytes + kStaticBudget > 227 * 1024) { *off = 0; return 0; }
    *off = (int)base;
    return (base - batch_smem_bytes(n, ldk, prec)) + bytes;
}

cudaError_t launch_batch(const DevProb& P, const BatchBufs& Bf, const BatchParams& Q, int grid, const void* tmaps,
                         cudaStream_t s, const void* l2_base, size_t l2_bytes, float l2_hit)
{
    const size_t smem = batch_smem_bytes(P.n, P.ldk, Q.prec) + Q.inst_smem_bytes;
    cudaError_t e = cudaFuncSetAttribute(batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    TcMaps m;
    memset(&m, 0, sizeof(m));
    if (tmaps) memcpy(&m, tmaps, sizeof(m));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(kBatchThreads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[2];
    memset(attr, 0, sizeof(attr));
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    int na = 1;
    if (l2_base && l2_bytes) {
        // keep the split tensor resident in L2 across ticks (the per-instance state streams past it)
        attr[1].id = cudaLaunchAttributeAccessPolicyWindow;
        attr[1].val.accessPolicyWindow.base_ptr = const_cast<void*>(l2_base);
        attr[1].val.accessPolicyWindow.num_bytes = l2_bytes;
        attr[1].val.accessPolicyWindow.hitRatio = l2_hit;
        attr[1].val.accessPolicyWindow.hitProp = cudaAccessPropertyPersisting;
        attr[1].val.accessPolicyWindow.missProp = cudaAccessPropertyStreaming;
        na = 2;
    }
    cfg.attrs = attr;
    cfg.numAttrs = na;
    return cudaLaunchKernelEx(&cfg, batch_kernel, P, Bf, Q, m);
}

cudaError_t launch_split_tensor(const float* K, int n, int ldk, int np, int prec, uint16_t* khi, uint16_t* klo,
                                float* row_inv, cudaStream_t s)
{
    if (prec == kPrecFP16x3S) {
        row_scale_kernel<<<3 * np, 256, 0, s>>>(K, n, ldk, np, row_inv);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    split_tensor_kernel<<<1184, 256, 0, s>>>(K, n, ldk, np, prec, row_inv, khi, klo);
    return cudaGetLastError();
}

static void bs45b_fill(BS45b& T)
{
    memset(&T, 0, sizeof(T));
    auto& a = T.a;
    a[2][1] = 1.0 / 6.0;
    a[3][1] = 2.0 / 27.0; a[3][2] = 4.0 / 27.0;
    a[4][1] = 183.0 / 1372.0; a[4][2] = -162.0 / 343.0; a[4][3] = 1053.0 / 1372.0;
    a[5][1] = 68.0 / 297.0; a[5][2] = -4.0 / 11.0; a[5][3] = 42.0 / 143.0; a[5][4] = 1960.0 / 3861.0;
    a[6][1] = 597.0 / 22528.0; a[6][2] = 81.0 / 352.0; a[6][3] = 63099.0 / 585728.0;
    a[6][4] = 58653.0 / 366080.0; a[6][5] = 4617.0 / 20480.0;
    a[7][1] = 174197.0 / 959244.0; a[7][2] = -30942.0 / 79937.0; a[7][3] = 8152137.0 / 19744439.0;
    a[7][4] = 666106.0 / 1039181.0; a[7][5] = -29421.0 / 29068.0; a[7][6] = 482048.0 / 414219.0;
    a[8][1] = 587.0 / 8064.0; a[8][3] = 4440339.0 / 15491840.0;
    a[8][4] = 24353.0 / 124800.0; a[8][5] = 387.0 / 44800.0; a[8][6] = 2152.0 / 5985.0;
    a[8][7] = 7267.0 / 94080.0;
    T.b[1] = 2479.0 / 34992.0; T.b[3] = 123.0 / 416.0; T.b[4] = 612941.0 / 3411720.0;
    T.b[5] = 43.0 / 1440.0; T.b[6] = 2272.0 / 6561.0; T.b[7] = 79937.0 / 1113912.0; T.b[8] = 3293.0 / 556956.0;
    T.e[1] = -3.0 / 1280.0; T.e[3] = 6561.0 / 632320.0; T.e[4] = -343.0 / 20800.0;
    T.e[5] = 243.0 / 12800.0; T.e[6] = -1.0 / 95.0;
    T.c[2] = 1.0 / 6.0; T.c[3] = 2.0 / 9.0; T.c[4] = 3.0 / 7.0; T.c[5] = 2.0 / 3.0; T.c[6] = 3.0 / 4.0;
    T.c[7] = 1.0; T.c[8] = 1.0; T.c[9] = 1.0 / 2.0; T.c[10] = 5.0 / 6.0; T.c[11] = 1.0 / 9.0;
    a[9][1] = 455.0 / 6144.0; a[10][1] = -837888343715.0 / 13176988637184.0;
    a[11][1] = 98719073263.0 / 1551965184000.0;
    a[10][2] = 30409415.0 / 52955362.0; a[11][2] = 1307.0 / 123552.0;
    a[9][3] = 10256301.0 / 35409920.0; a[10][3] = -48321525963.0 / 759168069632.0;
    a[11][3] = 4632066559387.0 / 70181753241600.0;
    a[9][4] = 2307361.0 / 17971200.0; a[10][4] = 8530738453321.0 / 197654829557760.0;
    a[11][4] = 7828594302389.0 / 382182512025600.0;
    a[9][5] = -387.0 / 102400.0; a[10][5] = 1361640523001.0 / 1626788720640.0;
    a[11][5] = 40763687.0 / 11070259200.0;
    a[9][6] = 73.0 / 5130.0; a[10][6] = -13143060689.0 / 38604458898.0;
    a[11][6] = 34872732407.0 / 224610586200.0;
    a[9][7] = -7267.0 / 215040.0; a[10][7] = 18700221969.0 / 379584034816.0;
    a[11][7] = -2561897.0 / 30105600.0;
    a[9][8] = 1.0 / 32.0; a[10][8] = -5831595.0 / 847285792.0; a[11][8] = 1.0 / 10.0;
    a[10][9] = -5183640.0 / 26477681.0; a[11][9] = -1.0 / 10.0;
    a[11][10] = -1403317093.0 / 11371610250.0;
    auto& r = T.r;
    r[1][6] = -12134338393.0 / 1050809760.0; r[1][5] = -1620741229.0 / 50038560.0;
    r[1][4] = -2048058893.0 / 59875200.0; r[1][3] = -87098480009.0 / 5254048800.0;
    r[1][2] = -11513270273.0 / 3502699200.0;
    r[3][6] = -33197340367.0 / 1218433216.0; r[3][5] = -539868024987.0 / 6092166080.0;
    r[3][4] = -39991188681.0 / 374902528.0; r[3][3] = -69509738227.0 / 1218433216.0;
    r[3][2] = -29327744613.0 / 2436866432.0;
    r[4][6] = -284800997201.0 / 19905339168.0; r[4][5] = -7896875450471.0 / 165877826400.0;
    r[4][4] = -333945812879.0 / 5671036800.0; r[4][3] = -16209923456237.0 / 497633479200.0;
    r[4][2] = -2382590741699.0 / 331755652800.0;
    r[5][6] = -540919.0 / 741312.0; r[5][5] = -103626067.0 / 43243200.0; r[5][4] = -633779.0 / 211200.0;
    r[5][3] = -32406787.0 / 18532800.0; r[5][2] = -36591193.0 / 86486400.0;
    r[6][6] = 7157998304.0 / 374350977.0; r[6][5] = 30405842464.0 / 623918295.0;
    r[6][4] = 183022264.0 / 5332635.0; r[6][3] = -3357024032.0 / 1871754885.0;
    r[6][2] = -611586736.0 / 89131185.0;
    r[7][6] = -138073.0 / 9408.0; r[7][5] = -719433.0 / 15680.0; r[7][4] = -1620541.0 / 31360.0;
    r[7][3] = -385151.0 / 15680.0; r[7][2] = -65403.0 / 15680.0;
    r[8][6] = 1245.0 / 64.0; r[8][5] = 3991.0 / 64.0; r[8][4] = 4715.0 / 64.0; r[8][3] = 2501.0 / 64.0;
    r[8][2] = 149.0 / 16.0; r[8][1] = 1.0;
    r[9][6] = 55.0 / 3.0; r[9][5] = 71.0; r[9][4] = 103.0; r[9][3] = 199.0 / 3.0; r[9][2] = 16.0;
    r[10][6] = -1774004627.0 / 75810735.0; r[10][5] = -1774004627.0 / 25270245.0;
    r[10][4] = -26477681.0 / 359975.0; r[10][3] = -11411880511.0 / 379053675.0;
    r[10][2] = -423642896.0 / 126351225.0;
    r[11][6] = 35.0; r[11][5] = 105.0; r[11][4] = 117.0; r[11][3] = 59.0; r[11][2] = 12.0;
}
