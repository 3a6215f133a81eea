// Shared device helpers: bounded grid barrier, block reductions, cache-global
// loads, exact (non-contracted) FP64 arithmetic.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define MT_DEV __device__ __forceinline__

// Error codes recorded by kernels in GridSync::err (host maps them to MT_ERR_*).
enum { KERR_NONE = 0, KERR_BARRIER_TIMEOUT = 1, KERR_BAD_CONFIG = 2, KERR_RANGE = 3, KERR_PEER_TIMEOUT = 4,
       KERR_PEER_ABORT = 5 };

// Grid-wide barrier state for the persistent cooperative kernels.  The host
// zeroes it before every launch (count then holds the arrivals of the launch so
// far; gen is unused).
struct GridSync {
    unsigned int count;
    unsigned int gen;
    int abort;
    int err;
    int err_where;
    int pad[3];
};

MT_DEV unsigned ld_acquire_u32(const unsigned* p)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
MT_DEV void st_release_u32(unsigned* p, unsigned v)
{
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
MT_DEV unsigned ld_acquire_sys_u32(const unsigned* p)
{
    unsigned v;
    asm volatile("ld.acquire.sys.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
MT_DEV void st_release_sys_u32(unsigned* p, unsigned v)
{
    asm volatile("st.release.sys.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
MT_DEV unsigned atom_add_acq_rel_u32(unsigned* p, unsigned v)
{
    unsigned old;
    asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}
MT_DEV int ld_volatile_i32(const int* p) { return *(volatile const int*)p; }
MT_DEV uint64_t globaltimer_ns()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Barrier across all CTAs of a cooperative launch.  Every wait is bounded: after
// kSpinLimit polls or kTimeoutNs nanoseconds the waiting CTA records
// KERR_BARRIER_TIMEOUT, raises abort and returns false; CTAs that see abort
// return false at once.  Returns true when all CTAs arrived.
constexpr long long kSpinLimit = 20000000LL;
constexpr uint64_t kTimeoutNs = 4000000000ULL;

// The same for a group of nctas CTAs that share one GridSync (the CTA groups
// of a ragged launch; every CTA of a group calls it the same number of times).
MT_DEV bool group_sync(GridSync* gs, unsigned nctas, int where)
{
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        if (ld_volatile_i32(&gs->abort)) {
            ok = 0;
        } else {
            // count only grows within a launch: every CTA arrives at barrier k before any
            // CTA can arrive at barrier k + 1, so the arrivals at barrier k return values in
            // [k nctas, (k + 1) nctas) and the barrier is complete once count reaches
            // (k + 1) nctas; the last arriver needs no reset and no second store
            // acq_rel: releases the CTA's writes (ordered before by the __syncthreads above)
            // and, for the last arriver, acquires everyone else's
            const unsigned prev = atom_add_acq_rel_u32(&gs->count, 1u);
            const unsigned target = (prev / nctas + 1u) * nctas;
            if (prev + 1u != target) {
                long long it = 0;
                uint64_t t0 = globaltimer_ns();
                while (ld_acquire_u32(&gs->count) < target) {
                    if (ld_volatile_i32(&gs->abort)) { ok = 0; break; }
                    if (++it > kSpinLimit || (it & 1023) == 0 && globaltimer_ns() - t0 > kTimeoutNs) {
                        if (atomicCAS(&gs->err, 0, KERR_BARRIER_TIMEOUT) == 0) gs->err_where = where;
                        atomicExch(&gs->abort, 1);
                        ok = 0;
                        break;
                    }
                    __nanosleep(32);
                }
            }
        }
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

MT_DEV bool grid_sync(GridSync* gs, int where) { return group_sync(gs, gridDim.x, where); }

// Block-wide reductions; the result is returned to every thread.  scratch must
// hold 32 doubles.  Deterministic (fixed tree).
MT_DEV double warp_max(double v)
{
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
MT_DEV double warp_sum(double v)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
template <bool IsMax>
MT_DEV double block_reduce(double v, double* scratch)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    v = IsMax ? warp_max(v) : warp_sum(v);
    __syncthreads();
    if (lane == 0) scratch[wid] = v;
    __syncthreads();
    if (wid == 0) {
        double w = (lane < nw) ? scratch[lane] : (IsMax ? -1.0 : 0.0);
        if (IsMax && lane >= nw) w = scratch[0];
        w = IsMax ? warp_max(w) : warp_sum(w);
        if (lane == 0) scratch[0] = w;
    }
    __syncthreads();
    double r = scratch[0];
    __syncthreads();
    return r;
}

// Exact IEEE double arithmetic with no FMA contraction, so that elementwise
// results match a CPU evaluation of the same expression bit for bit.
MT_DEV double xmul(double a, double b) { return __dmul_rn(a, b); }
MT_DEV double xadd(double a, double b) { return __dadd_rn(a, b); }
MT_DEV double xsub(double a, double b) { return __dsub_rn(a, b); }

// x^(1/5) for the RKSUITE step-size control, from IEEE operations only (so the
// host oracle, which runs the same iteration, rounds identically): x = f 2^e,
// e = 5 q + r, y = f 2^r in [0.5, 16), twelve Newton steps z <- z + (y / z^4 - z) / 5
// from z = 1 (y < 2) or 1.5, then 2^q z.  Agrees with pow(x, 0.2) to a few ulp
// (pow's exponent 0.2 is itself 1/5 + 1.1e-17).
MT_DEV double root5(double x)
{
    if (!(x > 0.0)) return 0.0;
    if (isinf(x)) return x;
    int e = 0;
    const double f = frexp(x, &e);
    const int q = (e >= 0) ? e / 5 : -((-e + 4) / 5);
    const double y = ldexp(f, e - 5 * q);
    double z = (y < 2.0) ? 1.0 : 1.5;
    for (int k = 0; k < 12; ++k) {
        const double z2 = __dmul_rn(z, z);
        const double z4 = __dmul_rn(z2, z2);
        z = __dadd_rn(z, __ddiv_rn(__dsub_rn(__ddiv_rn(y, z4), z), 5.0));
    }
    return ldexp(z, q);
}

MT_DEV double ldcg(const double* p) { return __ldcg(p); }
MT_DEV float ldcg(const float* p) { return __ldcg(p); }

static inline int ceil_div(long long a, long long b) { return (int)((a + b - 1) / b); }
