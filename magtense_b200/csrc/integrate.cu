// Device-resident adaptive Runge-Kutta integration of the Landau-Lifshitz
// equation: RKSUITE-90 method 'M' (the Bogacki-Shampine 4(5) FSAL pair with a
// sixth-degree interpolant) driven by the output-time loop of
// MagTense_ODE_RKSuite, all inside ONE persistent cooperative kernel.
//
// Reference behaviour followed (paths relative to the MagTense project root,
// source/NumericalIntegration/NumericalIntegration/):
//   RKSuitef90.f90  setup_r1 :596-856, range_integrate_r1 :942-1183,
//                   step_integrate_r1 :1185-1587, step_r1 :1726-1978 (stepa,
//                   stepb), stiff_r1 :1981-2367, interpolate_r1 :2655-2997,
//                   method_const case 2 :223-412, :568-591
//   ODE_Solvers.f90 MagTense_ODE_RKSuite :124-237
//
// Execution model.  Every CTA owns a contiguous range of cells (all three
// components).  All scalar control state (t, h, phases, counters) is computed
// redundantly and identically by every thread of every CTA from the same
// inputs, so no broadcast is needed.  Vector operations touch only owned
// elements.  Global data dependencies are:
//   * a right-hand-side evaluation reads the stage argument of ALL cells
//     (demag product, exchange neighbours) -> grid barrier before it;
//   * norms and inner products -> per-CTA partials + grid barrier + a
//     fixed-order combine done identically by every CTA.
// Stage arguments alternate between two buffers so that a fast CTA never
// overwrites an argument a slow CTA is still reading.  All waits are bounded
// (grid_sync in common.cuh).  A row-sharded instance (ShardLink in
// integrate.cuh) runs the same code on every rank with each rank's CTAs owning
// that rank's cells; its argument stores and reduction partials go to every
// rank and its barriers span all ranks (sync_all).  The kernel returns after a budget of
// right-hand-side evaluations with its full state saved, and is relaunched by
// the host until the run ends.
#include "common.cuh"
#include "llg.cuh"
#include "integrate.cuh"

namespace {

// Bogacki-Shampine 4(5) coefficients as tabulated in RKSuitef90.f90:252-411
// (1-based indices, published method constants).
struct BS45 { double a[12][12]; double b[9]; double c[12]; double e[8]; double r[12][7]; };
__constant__ BS45 cT;

constexpr int kRed = 4;   // values per grid reduction slot

struct Ctx {
    DevProb P;
    IntegBufs B;
    IntegParams Q;
    int c0, nc;                 // owned cells
    float* sm_m; float* sm_part; float* sm_S;
    double* sm_scr;             // 32 doubles
    double* sm_red;             // kRed doubles
    int rcount;
    long long budget_end;       // stop when f_total reaches this
    bool abort;
    int grank, gsize;           // this CTA's rank in the instance's CTA group, and the group size
    const ShardLink* L;         // row shards, or nullptr
    int srank, sworld;          // shard rank and count (0, 1 without shards)
    int slot0, nslots;          // this group's first reduction slot, and the slots over all ranks
    long long xseq;             // cross-rank barriers passed
};

// ---- own-element iteration ---------------------------------------------
// element e in [0, 3*nc): component a = e / nc, cell i = c0 + e % nc,
// FP64 index q = a*n + i, FP32 shadow index a*ldk + i.
#define FOR_OWN(X, q, q32)                                                              \
    for (int _e = threadIdx.x; _e < 3 * (X).nc; _e += blockDim.x)                       \
        if ([[maybe_unused]] const int _a = _e / (X).nc, _i = (X).c0 + (_e - _a * (X).nc), \
                      q = _a * (X).P.n + _i, q32 = _a * (X).P.ldk + _i; true)

// Barrier of all CTAs of the instance.  Row shards: the rank's CTAs meet, the
// rank's first CTA raises its epoch flag in every rank's region (release at
// system scope), and every CTA of every rank waits until all ranks' flags carry
// the epoch (acquire at system scope; bounded by the link's timeout, after which
// KERR_PEER_TIMEOUT is recorded and the instance aborts).  Each thread fences its
// peer stores at system scope before it arrives.
//
// A rank that gives up raises the sticky abort word in every rank's region.  A
// rank checks its own abort word before it raises its flag and while it waits,
// so a peer that was between barriers when another rank gave up stops at its
// next barrier (KERR_PEER_ABORT) instead of waiting out its own timeout: its
// peer stores end one barrier interval after the abort.
MT_DEV bool sync_all(Ctx& X, int where)
{
    if (!X.L) {
        if (!group_sync(X.B.gs, X.gsize, where)) { X.abort = true; return false; }
        return true;
    }
    __threadfence_system();
    if (!group_sync(X.B.gs, X.gsize, where)) { X.abort = true; return false; }
    X.xseq++;
    const unsigned ep = (unsigned)X.xseq;
    const unsigned* own_abort = X.L->flags[X.srank] + kMaxShards;
    __shared__ int s_xok;
    if (threadIdx.x == 0) s_xok = 1;
    __syncthreads();
    if (threadIdx.x < X.sworld) {
        const int p = threadIdx.x;
        bool gave_up = false;
        if (ld_acquire_sys_u32(own_abort) != 0u) {
            if (atomicCAS(&X.B.gs->err, 0, KERR_PEER_ABORT) == 0) X.B.gs->err_where = where;
            atomicExch(&X.B.gs->abort, 1);
            s_xok = 0;
        } else {
            if (X.grank == 0) st_release_sys_u32(X.L->flags[p] + X.srank, ep);
            const unsigned* f = X.L->flags[X.srank] + p;
            const unsigned long long tmo = X.L->timeout_ns;
            long long it = 0;
            const uint64_t t0 = globaltimer_ns();
            while ((int)(ld_acquire_sys_u32(f) - ep) < 0) {
                if (ld_volatile_i32(&X.B.gs->abort)) { s_xok = 0; break; }
                if (ld_acquire_sys_u32(own_abort) != 0u) {
                    if (atomicCAS(&X.B.gs->err, 0, KERR_PEER_ABORT) == 0) X.B.gs->err_where = where;
                    atomicExch(&X.B.gs->abort, 1);
                    s_xok = 0;
                    break;
                }
                if ((unsigned long long)(++it) > tmo / 8 || ((it & 1023) == 0 && globaltimer_ns() - t0 > tmo)) {
                    if (atomicCAS(&X.B.gs->err, 0, KERR_PEER_TIMEOUT) == 0) X.B.gs->err_where = where;
                    atomicExch(&X.B.gs->abort, 1);
                    s_xok = 0;
                    gave_up = true;
                    break;
                }
                __nanosleep(64);
            }
        }
        if (gave_up)   // tell every rank (this one included) to stop at its next barrier
            for (int r = 0; r < X.sworld; ++r) st_release_sys_u32(X.L->flags[r] + kMaxShards, 1u);
    }
    __syncthreads();
    if (!s_xok) { X.abort = true; return false; }
    return true;
}

template <bool IsMax, int K>
MT_DEV bool grid_reduce(Ctx& X, double (&v)[K], int where)
{
    for (int k = 0; k < K; ++k) v[k] = block_reduce<IsMax>(v[k], X.sm_scr);
    const size_t half = (size_t)(X.rcount & 1) * X.nslots * kRed;
    double* buf = X.B.partials + half;
    X.rcount++;
    if (threadIdx.x == 0) {
        const int slot = (X.slot0 + X.grank) * kRed;
        if (X.L) {
            for (int p = 0; p < X.sworld; ++p)
                for (int k = 0; k < K; ++k) X.L->partials[p][half + slot + k] = v[k];
        } else {
            for (int k = 0; k < K; ++k) buf[slot + k] = v[k];
        }
    }
    if (!sync_all(X, where)) return false;
    if (threadIdx.x < 32) {
        for (int k = 0; k < K; ++k) {
            double r = IsMax ? 0.0 : 0.0;
            bool have = false;
            for (int b = threadIdx.x; b < X.nslots; b += 32) {
                double x = ldcg(&buf[b * kRed + k]);
                if (IsMax) r = have ? fmax(r, x) : x; else r += x;
                have = true;
            }
            if (IsMax) { if (!have) r = ldcg(&buf[k]); r = warp_max(r); }
            else r = warp_sum(r);
            if (threadIdx.x == 0) X.sm_red[k] = r;
        }
    }
    __syncthreads();
    for (int k = 0; k < K; ++k) v[k] = X.sm_red[k];
    __syncthreads();
    return true;
}

MT_DEV bool barrier(Ctx& X, int where) { return sync_all(X, where); }

// right-hand side of the LL equation at (t, arg) for the owned cells
MT_DEV void feval(Ctx& X, RKS& s, double t, int argi, double* out)
{
    const double* arg = X.B.pool[argi];
    const float* arg32 = X.B.pool32[argi];
    demag_cta(X.P, arg32, X.c0, X.nc, X.sm_m, X.sm_part, X.sm_S, 5);
    const TimeScalars ts = time_scalars(X.P, t);
    const int n = X.P.n;
    for (int cell = threadIdx.x; cell < X.nc; cell += blockDim.x) {
        double o[3];
        cell_rhs(X.P, arg, X.c0 + cell, &X.sm_S[cell * 3], ts, o);
        const int i = X.c0 + cell;
        out[i] = o[0]; out[n + i] = o[1]; out[2 * n + i] = o[2];
    }
    __syncthreads();
    s.f_count++;
}

MT_DEV void write_arg(Ctx& X, int argi, int q, int q32, double v)
{
    if (X.L) {   // every rank's copy, this rank's included
        const float f = (float)v;
        for (int p = 0; p < X.sworld; ++p) {
            X.L->pool[p][argi][q] = v;
            X.L->pool32[p][argi][q32] = f;
        }
        return;
    }
    X.B.pool[argi][q] = v;
    X.B.pool32[argi][q32] = (float)v;
}

// -------------------------------------------------------------------------
// step_r1: one attempt (with phase-2 restarts) of a step of size htry.
// Returns false on abort.  err receives the weighted error norm.
// -------------------------------------------------------------------------
MT_DEV bool rk_step(Ctx& X, RKS& s, double tnow, double& htry, double hmin, double& err)
{
    const double* y = X.B.pool[s.iy];
    const double* yp = X.B.deriv[s.dyp];
    double* es = X.B.errest;
    double* w = X.B.weights;
    const double thr = X.Q.thres;
    for (;;) {
        if (s.phase2) {
            FOR_OWN(X, q, q32) w[q] = fmax(thr, fabs(ldcg(&y[q])));
            __syncthreads();
        }
        bool restart = false;
        for (int i = 2; i <= 8; ++i) {
            const int argi = (i & 1) ? s.ia1 : s.ia0;
            double lm = 0.0;
            FOR_OWN(X, q, q32) {
                double e = xmul(cT.a[i][1], ldcg(&yp[q]));
                for (int j = 2; j <= i - 1; ++j) {
                    const double aij = cT.a[i][j];
                    if (aij == 0.0) continue;
                    e = xadd(e, xmul(aij, ldcg(&X.B.stg[j][q])));
                }
                const double yq = ldcg(&y[q]);
                const double yn = xadd(yq, xmul(htry, e));
                write_arg(X, argi, q, q32, yn);
                if (i == 8) es[q] = e;
                if (i == 7) {   // stepb: early estimate from the embedded 4th-order formula
                    double v = xmul(cT.e[1], ldcg(&yp[q]));
                    v = xadd(v, xmul(cT.e[3], ldcg(&X.B.stg[3][q])));
                    v = xadd(v, xmul(cT.e[4], ldcg(&X.B.stg[4][q])));
                    v = xadd(v, xmul(cT.e[5], ldcg(&X.B.stg[5][q])));
                    v = xadd(v, xmul(cT.e[6], ldcg(&X.B.stg[6][q])));
                    const double wq = fmax(xmul(0.5, xadd(fabs(yq), fabs(yn))), thr);
                    lm = fmax(lm, fabs(v) / wq);
                }
            }
            if (i == 7) {
                double v1[1] = {lm};
                if (!grid_reduce<true, 1>(X, v1, 70)) return false;
                err = xmul(fabs(s.h), v1[0]);
                if (err > s.tol) return true;
            } else {
                if (!barrier(X, 60 + i)) return false;
            }
            double tstg = xadd(tnow, xmul(cT.c[i], htry));
            if (s.at_t_end && cT.c[i] == 1.0) tstg = s.t_end;
            double* out = (i == 8) ? X.B.deriv[s.d8] : X.B.stg[i];
            feval(X, s, tstg, argi, out);
            if (s.phase2 && i <= 3 && fabs(htry) > hmin) {   // stepa
                const double* yn = X.B.pool[argi];
                double m4[4] = {0.0, 0.0, 0.0, 0.0};
                FOR_OWN(X, q, q32) {
                    const double ynq = ldcg(&yn[q]), yq = ldcg(&y[q]);
                    const double wq = fmax(ldcg(&w[q]), fabs(ynq));
                    w[q] = wq;
                    m4[0] = fmax(m4[0], fabs(yq) / wq);
                    m4[1] = fmax(m4[1], fabs(ynq) / wq);
                    m4[2] = fmax(m4[2], fabs(xsub(ynq, yq)) / wq);
                    m4[3] = fmax(m4[3], fabs(xsub(ldcg(&out[q]), ldcg(&yp[q]))) / wq);
                }
                if (!grid_reduce<true, 4>(X, m4, 80 + i)) return false;
                double ynrm = m4[0], ystgnm = m4[1], argdif = m4[2], fdiff = m4[3];
                const double tdiff = xsub(tstg, tnow);
                const double twt = fabs(xsub(s.t_end, tnow));
                ynrm = fmax(ynrm, fabs(tnow) / twt);
                ystgnm = fmax(ystgnm, fabs(tstg) / twt);
                argdif = fmax(argdif, fabs(tdiff) / twt);
                bool cutbak = false;
                if (argdif > xmul(X.Q.round_off, fmax(ynrm, ystgnm))) {
                    if (xmul(fabs(htry), fdiff) > xmul(3.9, argdif)) {
                        const double scl = fmax(0.125, fmin(0.5, xmul(3.9, argdif) / xmul(fabs(htry), fdiff)));
                        htry = xmul(scl, htry);
                        cutbak = true;
                    }
                }
                if (cutbak) {
                    s.at_t_end = 0;
                    if (fabs(htry) <= hmin) { htry = copysign(hmin, htry); s.phase2 = 0; }
                    restart = true;
                    break;
                }
            }
        }
        if (restart) continue;
        // local error estimate of the 4th-order formula against the 5th-order result
        const double* yn = X.B.pool[s.ia0];
        const double* k8 = X.B.deriv[s.d8];
        double lm = 0.0;
        FOR_OWN(X, q, q32) {
            double v = ldcg(&es[q]);
            v = xsub(v, xmul(cT.b[1], ldcg(&yp[q])));
            for (int i = 2; i <= 7; ++i) {
                if (cT.b[i] == 0.0) continue;
                v = xsub(v, xmul(cT.b[i], ldcg(&X.B.stg[i][q])));
            }
            v = xsub(v, xmul(cT.b[8], ldcg(&k8[q])));
            v = xmul(htry, v);
            es[q] = v;
            const double wq = fmax(xmul(0.5, xadd(fabs(ldcg(&y[q])), fabs(ldcg(&yn[q])))), thr);
            w[q] = wq;
            lm = fmax(lm, fabs(v) / wq);
        }
        double v1[1] = {lm};
        if (!grid_reduce<true, 1>(X, v1, 90)) return false;
        err = v1[0];
        return true;
    }
}

// weighted inner products for the stiffness test
MT_DEV bool wip3(Ctx& X, const double* a0, const double* b0, const double* a1, const double* b1,
                 const double* a2, const double* b2, int K, double out[3], int where)
{
    double v[3] = {0.0, 0.0, 0.0};
    const double* w = X.B.weights;
    FOR_OWN(X, q, q32) {
        const double wq = ldcg(&w[q]);
        v[0] += (ldcg(&a0[q]) / wq) * (ldcg(&b0[q]) / wq);
        if (K > 1) v[1] += (ldcg(&a1[q]) / wq) * (ldcg(&b1[q]) / wq);
        if (K > 2) v[2] += (ldcg(&a2[q]) / wq) * (ldcg(&b2[q]) / wq);
    }
    if (!grid_reduce<false, 3>(X, v, where)) return false;
    out[0] = v[0]; out[1] = v[1]; out[2] = v[2];
    return true;
}

// vout = (h_average/temp1) * (f(t, y + temp1*vin) - yp)
MT_DEV bool approx_jacobian(Ctx& X, RKS& s, double scale, const double* vin, double vdotv, double* vout)
{
    const double temp1 = scale / sqrt(vdotv);
    const double* y = X.B.pool[s.iy];
    const int argi = s.ia1;
    FOR_OWN(X, q, q32) write_arg(X, argi, q, q32, xadd(ldcg(&y[q]), xmul(temp1, ldcg(&vin[q]))));
    if (!barrier(X, 100)) return false;
    feval(X, s, s.t, argi, vout);
    const double fac = s.h_average / temp1;
    const double* yp = X.B.deriv[s.dyp];
    FOR_OWN(X, q, q32) vout[q] = xmul(fac, xsub(ldcg(&vout[q]), ldcg(&yp[q])));
    __syncthreads();
    return true;
}

struct Cplx { double re, im; };
MT_DEV double cabs_(Cplx z) { return hypot(z.re, z.im); }
MT_DEV Cplx csub_(Cplx a, Cplx b) { return {a.re - b.re, a.im - b.im}; }
// principal square root of (x + i*s0) where s0 is a signed zero
MT_DEV Cplx csqrt_real(double x, double signed_zero)
{
    if (x >= 0.0) return {sqrt(x), signed_zero};
    double r = sqrt(-x);
    return {0.0, signbit(signed_zero) ? -r : r};
}
MT_DEV void quad_roots(double alpha, double beta, Cplx r[2])
{
    const double tmp = alpha / 2.0;
    const double im0 = tmp * 0.0 + 0.0 * tmp;
    const Cplx sq = csqrt_real(tmp * tmp - beta, im0 - 0.0);
    const Cplx mt = {-tmp, 0.0};
    if (sq.re == 0.0 && sq.im == 0.0) { r[0] = mt; r[1] = mt; return; }
    const Cplx r1 = {-tmp + sq.re, sq.im};     // both roots as tabulated in the vendored code
    r[0] = r1; r[1] = r1;
}

// stiff_r1: returns false on abort; sure receives the diagnosis
MT_DEV bool rk_stiff(Ctx& X, RKS& s, int toomch, int& sure)
{
    sure = 0;
    int lots_of_fails = 0;
    if ((s.step_count - 10) % 40 == 0) {
        lots_of_fails = s.stiff_bad_step_count >= 10;
        s.stiff_bad_step_count = 0;
    }
    int maybe = toomch || lots_of_fails;
    double v0v0 = 0.0, scale = 0.0;
    double* w = X.B.weights;
    const double* y = X.B.pool[s.iy];
    const double* yo = X.B.pool[s.iyold];
    double* v0 = X.B.errest;
    double* v1 = X.B.stg[2];
    double* v2 = X.B.stg[3];
    double* v3 = X.B.stg[4];
    if (maybe) {
        FOR_OWN(X, q, q32) w[q] = fmax(xmul(0.5, xadd(fabs(ldcg(&y[q])), fabs(ldcg(&yo[q])))), X.Q.thres);
        __syncthreads();
        const double rat = fabs(s.h / s.h_average);
        maybe = 0.2 < rat && rat < 5.0;
        if (maybe) {
            maybe = xmul(7.0, fabs(xsub(s.t_end, s.t) / s.h_average)) > 5000.0;
            if (maybe) {
                double o[3];
                if (!wip3(X, v0, v0, y, y, nullptr, nullptr, 2, o, 110)) return false;
                v0v0 = o[0];
                const double ynrm = sqrt(o[1]);
                scale = xmul(ynrm, X.Q.sqrrmc);
                if (scale == 0.0) { scale = xmul(v0v0, X.Q.sqrrmc); maybe = scale > 0.0; }
            }
        }
    }
    if (!maybe) return true;
    if (v0v0 == 0.0) {
        FOR_OWN(X, q, q32) v0[q] = 1.0;
        __syncthreads();
        double o[3];
        if (!wip3(X, v0, v0, nullptr, nullptr, nullptr, nullptr, 1, o, 111)) return false;
        v0v0 = o[0];
    }
    const double v0nrm = sqrt(v0v0);
    FOR_OWN(X, q, q32) v0[q] = ldcg(&v0[q]) / v0nrm;
    __syncthreads();
    v0v0 = 1.0;
    double rold = 0.0, rho = 0.0;
    Cplx root[2] = {{0, 0}, {0, 0}}, prv[2] = {{0, 0}, {0, 0}};
    int ntry = 1;
    auto dominant = [&](double a11, double a10, double a00) -> bool {
        const double ratio = a10 / a00;
        rho = fabs(ratio);
        const double det = a00 * a11 - a10 * a10;
        const double res = fabs(det / a00);
        const bool big = det == 0.0 || (res <= fabs(a11) * 1e-6 && fabs(ratio - rold) <= 0.001 * rho);
        if (big) { root[0] = {ratio, 0.0}; root[1] = {0.0, 0.0}; }
        rold = ratio;
        return big;
    };
    for (;;) {
        double o[3];
        if (!approx_jacobian(X, s, scale, v0, v0v0, v1)) return false;
        if (!wip3(X, v1, v1, v1, v0, nullptr, nullptr, 2, o, 112)) return false;
        const double v1v1 = o[0], v1v0 = o[1];
        if (sqrt(v1v1) > 1.0e10 * sqrt(v0v0)) return true;
        if (ntry == 1) {
            rold = v1v0 / v0v0;
            if (fabs(rold) < X.Q.cubrmc) return true;
        } else {
            if (dominant(v1v1, v1v0, v0v0)) break;
        }
        if (!approx_jacobian(X, s, scale, v1, v1v1, v2)) return false;
        if (!wip3(X, v2, v2, v2, v0, v2, v1, 3, o, 113)) return false;
        const double v2v2 = o[0], v2v0 = o[1], v2v1 = o[2];
        if (dominant(v2v2, v2v1, v1v1)) break;
        const double det1 = v0v0 * v1v1 - v1v0 * v1v0;
        const double alpha1 = (-v0v0 * v2v1 + v1v0 * v2v0) / det1;
        const double beta1 = (v1v0 * v2v1 - v1v1 * v2v0) / det1;
        if (!approx_jacobian(X, s, scale, v2, v2v2, v3)) return false;
        if (!wip3(X, v3, v3, v3, v1, v3, v2, 3, o, 114)) return false;
        const double v3v3 = o[0], v3v1 = o[1], v3v2 = o[2];
        if (dominant(v3v3, v3v2, v2v2)) break;
        const double det2 = v1v1 * v2v2 - v2v1 * v2v1;
        const double alpha2 = (-v1v1 * v3v2 + v2v1 * v3v1) / det2;
        const double beta2 = (v2v1 * v3v2 - v2v2 * v3v1) / det2;
        const double res2 = fabs(v3v3 + alpha2 * v3v2 + beta2 * v3v1 + alpha2 * v3v2 + alpha2 * alpha2 * v2v2 +
                                 alpha2 * beta2 * v2v1 + beta2 * v3v1 + beta2 * alpha2 * v2v1 + beta2 * beta2 * v1v1);
        if (res2 <= fabs(v3v3) * 1e-6) {
            quad_roots(alpha1, beta1, prv);
            quad_roots(alpha2, beta2, root);
            rho = cabs_(prv[0]);
            const double dist = fmin(cabs_(csub_(root[0], prv[0])), cabs_(csub_(root[0], prv[1])));
            if (dist <= 0.001 * rho) break;
        }
        ntry++;
        if (ntry > 8) return true;
        const double v3nrm = sqrt(v3v3);
        FOR_OWN(X, q, q32) v0[q] = ldcg(&v3[q]) / v3nrm;
        __syncthreads();
        v0v0 = 1.0;
    }
    if (root[0].re < 0.0) {
        if (!(cabs_(root[1]) >= 0.9 * rho && root[1].re > 0.0)) {
            if (fabs(root[0].im) <= fabs(root[0].re) * 5.2) sure = rho >= 0.9 * 3.9;
        }
    }
    return true;
}

MT_DEV void renorm_own(Ctx& X, int pi)
{
    double* v = X.B.pool[pi];
    float* v32 = X.B.pool32[pi];
    const int n = X.P.n, ldk = X.P.ldk;
    for (int cell = threadIdx.x; cell < X.nc; cell += blockDim.x) {
        const int i = X.c0 + cell;
        const double x = v[i], y = v[n + i], z = v[2 * n + i];
        const double r = sqrt(xadd(xadd(xmul(x, x), xmul(y, y)), xmul(z, z)));
        if (r > 0.0) {
            const double a = x / r, b = y / r, c = z / r;
            if (X.L) {
                write_arg(X, pi, i, i, a);
                write_arg(X, pi, n + i, ldk + i, b);
                write_arg(X, pi, 2 * n + i, 2 * ldk + i, c);
            } else {
                v[i] = a; v[n + i] = b; v[2 * n + i] = c;
                v32[i] = (float)a; v32[ldk + i] = (float)b; v32[2 * ldk + i] = (float)c;
            }
        }
    }
    __syncthreads();
}

// step_integrate_r1: returns the flag (1 ok, 3, 4, 5, 911) or -1 on abort
MT_DEV int rk_step_integrate(Ctx& X, RKS& s)
{
    int ier = 1;
    double hmin = 0.0;
    if (s.at_t_start) {
        feval(X, s, s.t, s.iy, X.B.deriv[s.dyp]);
        double* w = X.B.weights;
        const double* y = X.B.pool[s.iy];
        const double* yp = X.B.deriv[s.dyp];
        double mx = -1.0;    // -1: no component with y != 0
        FOR_OWN(X, q, q32) {
            const double yq = ldcg(&y[q]);
            const double wq = fmax(fabs(yq), X.Q.thres);
            w[q] = wq;
            if (yq != 0.0) mx = fmax(mx, fabs(ldcg(&yp[q])) / wq);
        }
        double v1[1] = {mx};
        if (!grid_reduce<true, 1>(X, v1, 10)) return -1;
        s.phase2 = 1;
        s.h = fabs(s.h);
        const double ypnorm = fmax(0.0, v1[0] < 0.0 ? -1.0 : v1[0]);
        const double tau = root5(s.tol);
        if (xmul(s.h, ypnorm) > tau) s.h = tau / ypnorm;
        hmin = fmax(X.Q.sqtiny, xmul(X.Q.toosml, fmax(fabs(s.t_start), fabs(s.t_end))));
        s.h = xmul(s.dir, fmax(s.h, hmin));
    } else if (s.at_t_end) {
        return 911;
    }
    int phase3 = 1, failed = 0;
    for (;;) {
        s.h = copysign(fabs(s.h), s.dir);
        s.at_t_end = xmul(s.dir, xsub(xadd(s.t, s.h), s.t_end)) >= 0.0;
        if (s.at_t_end) s.h = xsub(s.t_end, s.t);
        else if (xmul(s.dir, xsub(xadd(s.t, xmul(2.0, s.h)), s.t_end)) >= 0.0) s.h = xsub(s.t_end, s.t) / 2.0;
        hmin = fmax(X.Q.sqtiny, xmul(X.Q.toosml, fmax(fabs(s.t), fabs(xadd(s.t, s.h)))));
        if (fabs(s.h) < hmin) { ier = 5; break; }
        if (s.chkeff) {
            s.hit_t_end_count++;
            if (s.hit_t_end_count >= 100 && s.hit_t_end_count >= s.step_count / 3) {
                ier = 2; s.hit_t_end_count = 0; break;
            }
        }
        if (!failed) {
            const int toomch = s.f_count > 5000;
            if (toomch) { ier = 3; s.full_f_count += s.f_count; s.f_count = 0; }
            int sure = 0;
            if (!rk_stiff(X, s, toomch, sure)) return -1;
            if (sure) ier = 4;
            if (ier != 1) break;
        }
        double htry = s.h, err = 0.0;
        if (!rk_step(X, s, s.t, htry, hmin, err)) return -1;
        s.h = htry;
        double alpha;
        if (err > s.tol) {
            if (s.at_t_start) { phase3 = 0; alpha = 0.5; }
            else {
                s.bad_step_count++;
                s.stiff_bad_step_count++;
                if (failed) alpha = 0.5;
                else alpha = fmax(xmul(0.8, root5(s.tol / err)), 0.5);
            }
            s.h = xmul(alpha, s.h);
            failed = 1;
            continue;
        }
        double beta = root5(err / s.tol);
        if (!s.at_t_start) {
            const double t1 = root5(err) / s.h;
            const double t2 = root5(s.errold) / s.h_old;
            if (t1 < xmul(t2, 100.0) && t2 < xmul(t1, 100.0)) beta = xmul(beta, t1 / t2);
        }
        alpha = 8.0;
        if (0.8 < xmul(beta, alpha)) alpha = 0.8 / beta;
        if (s.at_t_start) {
            s.phase2 = 0;
            phase3 = phase3 && !s.at_t_end && (alpha > 4.0);
            if (phase3) { s.h = xmul(alpha, s.h); continue; }
        }
        alpha = fmin(alpha, 2.0);
        if (failed) alpha = fmin(alpha, 1.0);
        alpha = fmax(alpha, 0.5);
        s.h_old = s.h;
        s.h = xmul(alpha, s.h);
        if (s.at_t_start) s.h_average = s.h_old;
        else s.h_average = xadd(xmul(0.9, s.h_average), xmul(0.1, s.h_old));
        s.at_t_start = 0;
        s.errold = err;
        s.t_old = s.t;
        if (s.at_t_end) s.t = s.t_end; else s.t = xadd(s.t, s.h_old);
        s.step_count++;
        // y_old <- y, y <- stage-8 argument, spare <- old y_old ; yp rotation
        const int oy = s.iy, oyo = s.iyold, oa0 = s.ia0;
        s.iyold = oy; s.iy = oa0; s.ia0 = oyo;
        const int dp = s.dyp, dpo = s.dypold, d8 = s.d8;
        s.dypold = dp; s.dyp = d8; s.d8 = dpo;
        if (X.Q.renorm) renorm_own(X, s.iy);
        break;
    }
    s.at_t_end = s.t == s.t_end;
    s.chkeff = s.at_t_end;
    if (ier == 1) s.intrp_ready = 0;
    return ier;
}

// interpolate_r1: y_want (own elements) at t_want; false on abort
MT_DEV bool rk_interpolate(Ctx& X, RKS& s, double t_want, double* y_want)
{
    const int n = X.P.n;
    (void)n;
    double* const* P5 = X.B.p;
    if (!s.intrp_ready) {
        const double* yold = X.B.pool[s.iyold];
        const double* k1 = X.B.deriv[s.dypold];
        const double* k8 = X.B.deriv[s.dyp];
        for (int i = 9; i <= 11; ++i) {
            const int argi = (i & 1) ? s.ia0 : s.ia1;
            FOR_OWN(X, q, q32) {
                double e = xmul(cT.a[i][1], ldcg(&k1[q]));
                for (int j = 2; j <= i - 1; ++j) {
                    const double* sj = (j == 8) ? k8 : X.B.stg[j];
                    e = xadd(e, xmul(cT.a[i][j], ldcg(&sj[q])));
                }
                write_arg(X, argi, q, q32, xadd(ldcg(&yold[q]), xmul(s.h_old, e)));
            }
            if (!barrier(X, 120 + i)) return false;
            feval(X, s, xadd(s.t_old, xmul(cT.c[i], s.h_old)), argi, X.B.stg[i]);
        }
        const double ho = s.h_old;
        FOR_OWN(X, q, q32) {
            const double K1 = ldcg(&k1[q]), K3 = ldcg(&X.B.stg[3][q]), K4 = ldcg(&X.B.stg[4][q]);
            const double K5 = ldcg(&X.B.stg[5][q]), K6 = ldcg(&X.B.stg[6][q]), K7 = ldcg(&X.B.stg[7][q]);
            const double K8 = ldcg(&k8[q]), K9 = ldcg(&X.B.stg[9][q]), K10 = ldcg(&X.B.stg[10][q]);
            const double K11 = ldcg(&X.B.stg[11][q]);
#define R(i, j) cT.r[i][j]
#define M(a, b) xmul(a, b)
#define A(a, b) xadd(a, b)
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
            P5[5][q] = xmul(ho, p5); P5[4][q] = xmul(ho, p4); P5[3][q] = xmul(ho, p3);
            P5[2][q] = xmul(ho, p2); P5[1][q] = xmul(ho, p1);
        }
        __syncthreads();
        s.intrp_ready = 1;
    }
    const double sigma = xsub(t_want, s.t) / s.h_old;
    const double* y = X.B.pool[s.iy];
    const double* yp = X.B.deriv[s.dyp];
    FOR_OWN(X, q, q32) {
        double v = xmul(ldcg(&P5[5][q]), sigma);
        v = xmul(xadd(v, ldcg(&P5[4][q])), sigma);
        v = xmul(xadd(v, ldcg(&P5[3][q])), sigma);
        v = xmul(xadd(v, ldcg(&P5[2][q])), sigma);
        v = xmul(xadd(v, ldcg(&P5[1][q])), sigma);
        y_want[q] = xadd(xmul(xadd(v, xmul(s.h_old, ldcg(&yp[q]))), sigma), ldcg(&y[q]));
    }
    __syncthreads();
    return true;
}

// range_integrate_r1 (resumable across launches): returns flag, -1 abort, -2 budget
MT_DEV int rk_range_integrate(Ctx& X, RKS& s, double t_want, double* y_got, double& t_got)
{
    if (!s.in_range) {
        if (s.at_t_start) {
            s.range_t_end = s.t_end;
            s.tlast = s.t_start;
            t_got = s.t_start;
            s.h = fmin(fabs(s.h), fabs(xsub(t_want, s.t_start)));
            const double hmin = fmax(X.Q.sqtiny, xmul(X.Q.toosml, fmax(fabs(s.t_start), fabs(s.t_end))));
            s.h = fmax(s.h, hmin);
        } else if (s.tlast == s.range_t_end) {
            return 911;
        }
        if (xmul(s.dir, xsub(t_want, s.tlast)) <= 0.0) return 911;
        if (xmul(s.dir, xsub(t_want, s.range_t_end)) > 0.0) return 911;
        s.in_range = 1;
    }
    int flag = 1;
    for (;;) {
        if (xmul(s.dir, xsub(s.t, t_want)) >= 0.0) {
            if (!rk_interpolate(X, s, t_want, y_got)) return -1;
            t_got = t_want;
            break;
        }
        if (s.full_f_count + s.f_count >= X.budget_end) return -2;
        flag = rk_step_integrate(X, s);
        if (flag < 0) return -1;
        if (flag == 1) continue;
        if (flag >= 911) { s.in_range = 0; return flag; }
        t_got = s.t;
        const double* y = X.B.pool[s.iy];
        FOR_OWN(X, q, q32) y_got[q] = ldcg(&y[q]);
        __syncthreads();
        break;
    }
    s.in_range = 0;
    s.tlast = t_got;
    return flag;
}

// The integrator of one instance on its CTA group (X.P, X.B, X.Q, X.grank, X.gsize set).
MT_DEV void integrate_body(Ctx& X, unsigned char* smem)
{
    const DevProb& P = X.P;
    const IntegBufs& B = X.B;
    const IntegParams& Q = X.Q;
    const int G = X.gsize;
    X.L = B.link;
    int cell0 = 0, ncell = P.n;
    X.srank = 0; X.sworld = 1; X.slot0 = 0; X.nslots = G;
    if (X.L) {
        X.srank = X.L->rank; X.sworld = X.L->world;
        cell0 = X.L->cell0; ncell = X.L->ncell;
        X.slot0 = X.L->cta_base; X.nslots = X.L->cta_total;
    }
    X.c0 = cell0 + (int)(((long long)ncell * X.grank) / G);
    X.nc = cell0 + (int)(((long long)ncell * (X.grank + 1)) / G) - X.c0;
    const int ncmax = (ncell + G - 1) / G;
    const int JC = P.ldk < kDemagJC ? P.ldk : kDemagJC;
    X.sm_m = reinterpret_cast<float*>(smem);
    X.sm_part = X.sm_m + 3 * JC;
    X.sm_S = X.sm_part + 3 * kDemagMaxUnits;
    X.sm_scr = reinterpret_cast<double*>(X.sm_S + ((3 * ncmax + 3) & ~3));
    X.sm_red = X.sm_scr + 32;
    X.abort = false;

    RKS s = *B.state;                  // identical copy in every thread
    X.rcount = (int)(s.rseq & 1);
    X.xseq = s.xseq;
    X.budget_end = s.full_f_count + s.f_count + Q.evals_per_launch;
    const int n3 = 3 * P.n;
    while (!s.finished && !X.abort) {
        if (s.ci >= Q.ncomb) { s.finished = 1; break; }
        const double t_want = Q.comb_t[s.ci];
        const int cf = Q.comb_flags[s.ci];
        const bool save = (cf & 1) && s.ko < Q.nt;
        double* dst = save ? B.y_out + (size_t)s.ko * n3 : B.ystep;
        double t_got = 0.0;
        const int flag = rk_range_integrate(X, s, t_want, dst, t_got);
        if (flag == -1) break;       // abort
        if (flag == -2) break;       // budget: state saved, relaunch continues inside range_integrate
        if (flag >= 911) { s.status = flag; s.finished = 1; break; }
        if (flag == 3) s.n_flag3++;
        if (flag == 4) s.n_flag4++;
        if (flag == 5 || flag == 2) s.status = flag;
        if (cf & 2) {       // convergence check against the last checked sample
            double ce = 0.0;
            FOR_OWN(X, q, q32) ce = fmax(ce, fabs(xsub(ldcg(&dst[q]), ldcg(&B.ylast[q]))));
            double v1[1] = {ce};
            if (!grid_reduce<true, 1>(X, v1, 130)) break;
            if (v1[0] < Q.conv_tol) {
                if (s.ko < Q.nt) {
                    if (!save) {
                        double* slot = B.y_out + (size_t)s.ko * n3;
                        FOR_OWN(X, q, q32) slot[q] = ldcg(&dst[q]);
                        __syncthreads();
                    }
                    if (X.grank == 0 && threadIdx.x == 0) { Q.t_out[s.ko] = t_got; Q.flags_out[s.ko] = flag; }
                }
                s.converged_at = s.ko;
                s.finished = 1;
                s.ci++;
                break;
            }
            FOR_OWN(X, q, q32) B.ylast[q] = ldcg(&dst[q]);
            __syncthreads();
        }
        if (save) {
            if (X.grank == 0 && threadIdx.x == 0) { Q.t_out[s.ko] = t_got; Q.flags_out[s.ko] = flag; }
            s.ko++;
        }
        s.ci++;
        if (s.status) { s.finished = 1; break; }
        if (s.full_f_count + s.f_count >= X.budget_end) break;
    }
    // row shards: all ranks finish at the same point (their states are identical), so
    // they meet once more; after it no rank stores into a peer's region for this run,
    // whichever exit (output, convergence or an RKSUITE error flag) ended it
    if (X.L && s.finished && !X.abort) sync_all(X, 140);
    // every CTA holds the same state; the group's first CTA publishes it
    s.rseq = X.rcount;
    s.xseq = X.xseq;
    if (X.grank == 0 && threadIdx.x == 0 && !X.abort) *B.state = s;
}

__global__ void __launch_bounds__(kIntegThreads, 1)
integrate_kernel(DevProb P, IntegBufs B, IntegParams Q)
{
    extern __shared__ __align__(16) unsigned char smem[];
    Ctx X;
    X.P = P; X.B = B; X.Q = Q;
    X.grank = blockIdx.x;
    X.gsize = gridDim.x;
    integrate_body(X, smem);
}

// Ragged batch: instances of different grids in one launch.  Instance k owns the
// CTAs [inst[k].cta0, inst[k].cta0 + inst[k].ncta) and runs the single-instance
// integrator on them with its own barrier, buffers and budget; the groups never
// wait for each other, so a group whose instance finishes simply returns.
__global__ void __launch_bounds__(kIntegThreads, 1)
integrate_ragged_kernel(const RaggedInst* __restrict__ inst, const int* __restrict__ cta_inst)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const int k = cta_inst[blockIdx.x];
    Ctx X;
    X.P = inst[k].P; X.B = inst[k].B; X.Q = inst[k].Q;
    X.grank = blockIdx.x - inst[k].cta0;
    X.gsize = inst[k].ncta;
    integrate_body(X, smem);
}

}  // namespace

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
static void bs45_fill(BS45& T)
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
    a[8][1] = 587.0 / 8064.0; a[8][2] = 0.0; a[8][3] = 4440339.0 / 15491840.0;
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

cudaError_t integrate_upload_tables()
{
    static BS45 T;
    bs45_fill(T);
    return cudaMemcpyToSymbol(cT, &T, sizeof(T));
}

int integrate_grid_size(int n, int num_sms)
{
    int g = n / 8;
    if (g < 1) g = 1;
    if (g > num_sms) g = num_sms;
    return g;
}

size_t integrate_smem_bytes(int n, int ldk, int grid)
{
    // n: the cells the grid's CTAs share (a rank's cells for a row-sharded instance)
    const int ncmax = (n + grid - 1) / grid;
    return demag_smem_bytes(ldk, ncmax) + 16 + sizeof(double) * (32 + kRed + 2);
}

cudaError_t launch_integrate_ragged(const RaggedInst* inst_dev, const int* cta_inst_dev, int grid, size_t smem,
                                    cudaStream_t stream)
{
    cudaError_t e = cudaFuncSetAttribute(integrate_ragged_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    const RaggedInst* a = inst_dev;
    const int* b = cta_inst_dev;
    void* args[] = {&a, &b};
    return cudaLaunchCooperativeKernel((const void*)integrate_ragged_kernel, dim3(grid), dim3(kIntegThreads), args, smem,
                                       stream);
}

cudaError_t launch_integrate(const DevProb& P, const IntegBufs& B, const IntegParams& Q, int grid,
                             cudaStream_t stream)
{
    const size_t smem = integrate_smem_bytes(P.n, P.ldk, grid);
    cudaError_t e = cudaFuncSetAttribute(integrate_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    DevProb p = P;
    IntegBufs b = B;
    IntegParams q = Q;
    void* args[] = {&p, &b, &q};
    return cudaLaunchCooperativeKernel((const void*)integrate_kernel, dim3(grid), dim3(kIntegThreads), args, smem,
                                       stream);
}
