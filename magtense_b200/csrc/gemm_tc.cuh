// tcgen05 (5th-generation tensor core) demag GEMM tile for the batched
// integrator: H[a][cell][inst] = sum_k Khi/lo[(a, cell), k] * Mhi/lo[inst, k]
// for the three field components a of 128 receiver cells and 128 instances,
// over one split of the 3n-long source dimension.
//
// Split-BF16: K32 = Khi + Klo and m32 = Mhi + Mlo (each part BF16, the low
// part the BF16 rounding of the remainder), products accumulated in FP32 in
// TMEM:  bf16x3 = Khi*Mhi + Khi*Mlo + Klo*Mhi ;  bf16x2 = Khi*Mhi + Klo*Mhi.
// Split-FP16 with row scaling (fp16s): every tensor row r is multiplied by a
// power of two s_r that puts its largest entry in [2^13, 2^14), then split
// into FP16 hi+lo (22 significant bits); m splits into FP16 hi+lo; the three
// products are accumulated in FP32 and the epilogue multiplies row r by 1/s_r
// (exact).  Small entries of a row fall into the FP16 subnormal range, where
// the absolute error stays below 2^-24 / s_r.
//
// Per k-block of 32 sources a stage holds A_hi[3], A_lo[3] (3 x 128 x 32 BF16
// each), B_hi, B_lo (128 x 32 BF16), loaded by TMA (SWIZZLE_64B, no multicast)
// into a 3-stage shared-memory ring.  Warp 4 (one lane) issues the TMA loads,
// warp 5 (one lane) issues tcgen05.mma (M=128, N=128, K=16) into three TMEM
// accumulators (columns 0/128/256) and commits each stage back to its empty
// barrier; warps 0-3 read the accumulators with tcgen05.ld and store them.
// Every mbarrier wait is bounded; on a timeout the kernel's abort flag is set.
#pragma once
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include "common.cuh"

struct TcMaps {
    CUtensorMap ahi, alo, bhi, blo;
};

struct TcState {
    long long kb_done;   // k-blocks consumed so far in this launch (ring position)
    long long tiles;     // tiles finished so far (accumulator barrier phase)
    uint32_t tmem;       // TMEM base address of the accumulators
};

constexpr int kTcStages = 3;
constexpr int kTcN = 128;                                    // instances per tile (MMA N)
constexpr int kTcKB = 32;                                    // k elements per stage (64 B rows)
constexpr int kTcABytes = 128 * kTcKB * 2;                   // one A tile
constexpr int kTcBBytes = kTcN * kTcKB * 2;                  // one B tile
constexpr int kTcStageBytes = 6 * kTcABytes + 2 * kTcBBytes; // 64 KB
constexpr int kTcTmemCols = 512;                             // three N-column accumulators

static inline size_t tc_smem_bytes() { return 1024 + (size_t)kTcStages * kTcStageBytes + 256; }

MT_DEV uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

MT_DEV void mbar_init(uint32_t bar, int count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
MT_DEV void mbar_expect_tx(uint32_t bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
// bounded wait on the given phase parity; false after the limit.  sleep_ns > 0:
// a patient waiter (the accumulator readers wait a whole segment of MMAs) that
// backs off between polls, so it does not take issue slots from the warps that
// drive the copies and the MMAs on the same SM sub-partition.
MT_DEV bool mbar_wait(uint32_t bar, uint32_t parity, GridSync* gs, int where, unsigned sleep_ns = 0)
{
    uint32_t done = 0;
    const uint64_t t0 = globaltimer_ns();
    for (long long it = 0; it < 4000000LL; ++it) {
        asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
                     : "=r"(done)
                     : "r"(bar), "r"(parity)
                     : "memory");
        if (done) return true;
        if (sleep_ns && it >= 4) __nanosleep(sleep_ns);
        if ((it & 255) == 255) {
            if (ld_volatile_i32(&gs->abort)) return false;
            if (globaltimer_ns() - t0 > 2000000000ULL) break;
        }
    }
    if (atomicCAS(&gs->err, 0, KERR_BARRIER_TIMEOUT) == 0) gs->err_where = where;
    atomicExch(&gs->abort, 1);
    return false;
}

MT_DEV void tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y, uint32_t bar)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
        "l"(map), "r"(x), "r"(y), "r"(bar)
        : "memory");
}

// shared-memory matrix descriptor: K-major tile of 64-byte rows with the
// 64-byte swizzle, 8-row groups 512 bytes apart (SBO), version 1 (tcgen05)
MT_DEV uint64_t sdesc_sw64(uint32_t saddr)
{
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)1 << 16;                  // LBO (unused for swizzled K-major)
    d |= (uint64_t)(512 >> 4) << 32;          // SBO
    d |= (uint64_t)1 << 46;                   // descriptor version
    d |= (uint64_t)4 << 61;                   // SWIZZLE_64B
    return d;
}

// instruction descriptors: D F32, A/B BF16 (or F16), both K-major, M = 128, N = kTcN
constexpr uint32_t kIdescBF16 = (1u << 4) | (1u << 7) | (1u << 10) | (((uint32_t)kTcN >> 3) << 17) | ((128u >> 4) << 24);
constexpr uint32_t kIdescF16 = (1u << 4) | (0u << 7) | (0u << 10) | (((uint32_t)kTcN >> 3) << 17) | ((128u >> 4) << 24);

MT_DEV void umma(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t accumulate)
{
    asm volatile("{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                 " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}" ::"r"(tmem_d),
                 "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
                 : "memory");
}

MT_DEV void umma_commit(uint32_t bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

MT_DEV void tmem_ld32(uint32_t taddr, float (&v)[32])
{
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
          "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
          "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int k = 0; k < 32; ++k) v[k] = __uint_as_float(r[k]);
}

// shared-memory layout of the GEMM area (1024-aligned base)
struct TcSmem {
    uint8_t* stages;     // kTcStages x kTcStageBytes
    uint64_t* full;      // kTcStages
    uint64_t* empty;     // kTcStages
    uint64_t* accum;     // 1
    uint32_t* tmem_slot; // 1
};

MT_DEV TcSmem tc_layout(unsigned char* smem)
{
    TcSmem L;
    const uint32_t base = smem_u32(smem);
    const uint32_t pad = (1024u - (base & 1023u)) & 1023u;
    L.stages = smem + pad;
    uint64_t* bars = reinterpret_cast<uint64_t*>(L.stages + (size_t)kTcStages * kTcStageBytes);
    L.full = bars;
    L.empty = bars + kTcStages;
    L.accum = bars + 2 * kTcStages;
    L.tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * kTcStages + 1);
    return L;
}

MT_DEV void tc_init_impl(unsigned char* smem, TcState& st)
{
    TcSmem L = tc_layout(smem);
    const int warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) {
        for (int k = 0; k < kTcStages; ++k) {
            mbar_init(smem_u32(&L.full[k]), 1);
            mbar_init(smem_u32(&L.empty[k]), 1);
        }
        mbar_init(smem_u32(L.accum), 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(L.tmem_slot)),
                     "r"(kTcTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    st.tmem = *reinterpret_cast<volatile uint32_t*>(L.tmem_slot);
    st.kb_done = 0;
    st.tiles = 0;
}

MT_DEV void tc_finish_impl(unsigned char* smem, TcState& st)
{
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if ((threadIdx.x >> 5) == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(st.tmem), "r"(kTcTmemCols) : "memory");
    (void)smem;
}

// One GEMM tile (cb, ib, s) of the current tick.  Q/F are BatchParams/BatchBufs.
// Returns a CTA-uniform ok flag.
template <typename QT, typename FT>
MT_DEV bool tc_gemm_tile_impl(unsigned char* smem, const QT& Q, const FT& F, const TcMaps& maps, int cb, int ib, int s,
                              bool three, bool f16, const float* row_inv, TcState& st)
{
    TcSmem L = tc_layout(smem);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int kseg = Q.Kd / Q.S;
    const int k0 = s * kseg;
    const int nkb = kseg / kTcKB;
    const uint32_t tx = three ? (uint32_t)kTcStageBytes : (uint32_t)(6 * kTcABytes + kTcBBytes);
    bool ok = true;
    if (warp == 4 && lane == 0) {
        for (int kb = 0; kb < nkb; ++kb) {
            const long long g = st.kb_done + kb;
            const int stg = (int)(g % kTcStages);
            const uint32_t ph = (uint32_t)((g / kTcStages) & 1);
            if (!mbar_wait(smem_u32(&L.empty[stg]), ph ^ 1u, F.gs, 200)) { ok = false; break; }
            uint8_t* base = L.stages + (size_t)stg * kTcStageBytes;
            const uint32_t fb = smem_u32(&L.full[stg]);
            mbar_expect_tx(fb, tx);
            const int x = k0 + kb * kTcKB;
            for (int a = 0; a < 3; ++a) {
                const int y = a * Q.np + cb * 128;
                tma_load_2d(smem_u32(base + a * kTcABytes), &maps.ahi, x, y, fb);
                tma_load_2d(smem_u32(base + (3 + a) * kTcABytes), &maps.alo, x, y, fb);
            }
            tma_load_2d(smem_u32(base + 6 * kTcABytes), &maps.bhi, x, ib * kTcN, fb);
            if (three) tma_load_2d(smem_u32(base + 6 * kTcABytes + kTcBBytes), &maps.blo, x, ib * kTcN, fb);
        }
        if (!ok) {   // let loads already in flight land before the CTA moves on
            const long long issued = st.kb_done + nkb;
            for (long long g = issued - kTcStages; g < issued; ++g) {
                if (g < 0) continue;
                mbar_wait(smem_u32(&L.full[g % kTcStages]), (uint32_t)((g / kTcStages) & 1), F.gs, 203);
            }
        }
    } else if (warp == 5 && lane == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t idesc = f16 ? kIdescF16 : kIdescBF16;
        for (int kb = 0; kb < nkb; ++kb) {
            const long long g = st.kb_done + kb;
            const int stg = (int)(g % kTcStages);
            const uint32_t ph = (uint32_t)((g / kTcStages) & 1);
            if (!mbar_wait(smem_u32(&L.full[stg]), ph, F.gs, 201)) { ok = false; break; }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t base = smem_u32(L.stages + (size_t)stg * kTcStageBytes);
#pragma unroll
            for (int kk = 0; kk < kTcKB / 16; ++kk) {
                const uint32_t koff = kk * 32;
                const uint64_t bh = sdesc_sw64(base + 6 * kTcABytes + koff);
                const uint64_t bl = sdesc_sw64(base + 6 * kTcABytes + kTcBBytes + koff);
#pragma unroll
                for (int a = 0; a < 3; ++a) {
                    const uint32_t d = st.tmem + a * kTcN;
                    const uint64_t ah = sdesc_sw64(base + a * kTcABytes + koff);
                    const uint64_t al = sdesc_sw64(base + (3 + a) * kTcABytes + koff);
                    umma(d, ah, bh, idesc, (kb > 0 || kk > 0) ? 1u : 0u);
                    if (three) umma(d, ah, bl, idesc, 1u);
                    umma(d, al, bh, idesc, 1u);
                }
            }
            umma_commit(smem_u32(&L.empty[stg]));
        }
        if (ok) umma_commit(smem_u32(L.accum));
    }
    if (warp < 4) {
        const uint32_t ph = (uint32_t)(st.tiles & 1);
        bool w = mbar_wait(smem_u32(L.accum), ph, F.gs, 202, 200);
        w = __all_sync(0xffffffffu, w);
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (w) {
            const int cell = cb * 128 + warp * 32 + lane;
#pragma unroll 1
            for (int a = 0; a < 3; ++a) {
                const float sc = row_inv ? __ldg(&row_inv[a * Q.np + cell]) : 1.0f;
#pragma unroll 1
                for (int half = 0; half < kTcN / 32; ++half) {
                    float v[32];
                    tmem_ld32(st.tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(a * kTcN + half * 32), v);
#pragma unroll
                    for (int k = 0; k < 32; ++k) {
                        const int inst = ib * kTcN + half * 32 + k;
                        F.hpart[(((size_t)s * Q.Bp + inst) * 3 + a) * Q.np + cell] = v[k] * sc;
                    }
                }
            }
        } else {
            ok = false;
        }
    }
    st.kb_done += nkb;
    st.tiles++;
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    return __syncthreads_and(ok ? 1 : 0) != 0;
}

// ---------------------------------------------------------------------------
// Exact fixed-point demag product on the integer tensor pipe (kind::i8).
//
// Tensor row r (component a, cell i; 3np rows) is scaled by 2^e_r so that its
// largest entry lies in [2^29, 2^30) and rounded to an integer Kq (|Kq| < 2^30),
// written as four signed 8-bit limbs Kq = k0 2^24 + k1 2^16 + k2 2^8 + k3.
// Every source value m_j (|m_j| < 1.96) is rounded to mq = rint(m_j 2^30) and
// written as four limbs mq = m0 2^24 + m1 2^16 + m2 2^8 + m3.  All sixteen limb
// products are accumulated exactly in int32 TMEM accumulators grouped by
// s = a + b (D_s, columns 64 s .. 64 s + 63) and combined in two int64 parts,
// Hhi = sum_{s<=3} 2^(8 (3 - s)) D_s and Hlo = sum_{s>=4} 2^(8 (6 - s)) D_s, so
// that sum_j Kq_rj mq_j = 2^24 Hhi + Hlo exactly and neither part can
// overflow: the sum over sources carries no rounding, does not depend on the
// order or split of the k range, and the field 2^(-30 - e_r) RN(2^24 Hhi + Hlo)
// is the same bit pattern on every run.
//
// Work split (Stream-K): tile = 128 tensor rows x 64 instances, unit = one
// 128-wide k step of a tile; the units of all active tiles are split into
// contiguous non-empty ranges, one per CTA, so every SM gets the same number of
// MMAs.  A CTA's range covers pieces ("segments") of one or more tiles; each
// segment's exact int64 partials go to its own slot [CTA][segment][part][inst][row],
// and the reader sums the slots of the CTAs that cover the tile.
// ---------------------------------------------------------------------------
constexpr int kI8Stages = 2;
constexpr int kI8KB = 128;                                   // int8 sources per stage (128-byte rows, 128-byte swizzle)
constexpr int kI8N = 64;                                     // instances per tile (MMA N)
constexpr int kI8ATile = 128 * kI8KB;                        // one 128-row K limb tile, 16 KB
constexpr int kI8BTile = kI8N * kI8KB;                       // one 64-row m limb tile, 8 KB
constexpr int kI8KLimbs = 4, kI8MLimbs = 4, kI8Acc = 7;
constexpr int kI8StageBytes = kI8KLimbs * kI8ATile + kI8MLimbs * kI8BTile;   // 96 KB

// shared-memory matrix descriptor: K-major tile of 128-byte rows with the
// 128-byte swizzle, 8-row groups 1024 bytes apart (SBO), version 1 (tcgen05)
MT_DEV uint64_t sdesc_sw128(uint32_t saddr)
{
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)1 << 16;                  // LBO (unused for swizzled K-major)
    d |= (uint64_t)(1024 >> 4) << 32;         // SBO
    d |= (uint64_t)1 << 46;                   // descriptor version
    d |= (uint64_t)2 << 61;                   // SWIZZLE_128B
    return d;
}
constexpr int kI8SlotElems = 2 * kI8N * 128;                 // int64 per segment slot (hi and lo parts)
// D S32 (2 at bit 4), A and B signed 8-bit (1 at bits 7 and 10), M = 128, N at bits 17-22 (N / 8)
constexpr uint32_t idesc_i8(uint32_t n) { return (2u << 4) | (1u << 7) | (1u << 10) | ((n >> 3) << 17) | ((128u >> 4) << 24); }
constexpr uint32_t kIdescI8 = idesc_i8(kI8N);

static inline size_t tc_i8_smem_bytes() { return 1024 + (size_t)kI8Stages * kI8StageBytes + 256; }

struct I8Smem {
    uint8_t* stages;
    uint64_t* full;      // kI8Stages
    uint64_t* empty;     // kI8Stages
    uint64_t* accum;     // segment accumulators complete
    uint64_t* tfree;     // segment accumulators drained (4 epilogue warps)
    uint32_t* tmem_slot;
};

MT_DEV I8Smem i8_layout(unsigned char* smem)
{
    I8Smem L;
    const uint32_t base = smem_u32(smem);
    const uint32_t pad = (1024u - (base & 1023u)) & 1023u;
    L.stages = smem + pad;
    uint64_t* bars = reinterpret_cast<uint64_t*>(L.stages + (size_t)kI8Stages * kI8StageBytes);
    L.full = bars;
    L.empty = bars + kI8Stages;
    L.accum = bars + 2 * kI8Stages;
    L.tfree = bars + 2 * kI8Stages + 1;
    L.tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * kI8Stages + 2);
    return L;
}

MT_DEV void tc_i8_init(unsigned char* smem, TcState& st)
{
    I8Smem L = i8_layout(smem);
    const int warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) {
        for (int k = 0; k < kI8Stages; ++k) {
            mbar_init(smem_u32(&L.full[k]), 1);
            mbar_init(smem_u32(&L.empty[k]), 1);
        }
        mbar_init(smem_u32(L.accum), 1);
        mbar_init(smem_u32(L.tfree), 4);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(L.tmem_slot)),
                     "r"(kTcTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    st.tmem = *reinterpret_cast<volatile uint32_t*>(L.tmem_slot);
    st.kb_done = 0;
    st.tiles = 0;
}

// the same with an L2 cache policy (createpolicy): the tensor limbs stream through L2
// with evict_first, so they do not push the instances' state out of L2
MT_DEV uint64_t l2_evict_first_policy()
{
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}

MT_DEV void tma_load_3d_hint(uint32_t dst, const CUtensorMap* map, int x, int y, int z, uint32_t bar, uint64_t policy)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1, {%2, %3, %4}], [%5], %6;" ::"r"(dst),
        "l"(map), "r"(x), "r"(y), "r"(z), "r"(bar), "l"(policy)
        : "memory");
}

MT_DEV void tma_load_3d(uint32_t dst, const CUtensorMap* map, int x, int y, int z, uint32_t bar)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(dst),
        "l"(map), "r"(x), "r"(y), "r"(z), "r"(bar)
        : "memory");
}

MT_DEV void umma_i8(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate, uint32_t idesc = kIdescI8)
{
    asm volatile("{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                 " tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n}" ::"r"(tmem_d),
                 "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
                 : "memory");
}

MT_DEV void tmem_ld32_i(uint32_t taddr, int (&v)[32])
{
    float f[32];
    tmem_ld32(taddr, f);
#pragma unroll
    for (int k = 0; k < 32; ++k) v[k] = __float_as_int(f[k]);
}

MT_DEV void mbar_arrive(uint32_t bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

// Stream-K over U units on G = min(Gsel, U) CTAs (every range non-empty):
// CTA c owns units [sk_start(c), sk_start(c + 1)).  Gsel (at most gridDim.x) and the
// unit order come from the schedule the autotuner picked for the active tile count.
MT_DEV long long sk_ctas(long long U, long long Gsel) { return U < Gsel ? U : Gsel; }
MT_DEV long long sk_start(long long c, long long U, long long G) { return c * U / G; }

// Schedule word: Stream-K CTA count in the low 16 bits, unit order in bit 16
// (0: tile-major, the units of one 64-instance tile and row block after another;
// 1: row-major, the active tiles of one row block after another, so a row block of
// the tensor is read for all active tiles close together in time).
constexpr int kSkOrderBit = 16;
MT_DEV int sk_sched_ctas(int w) { return w & 0xffff; }
MT_DEV int sk_sched_order(int w) { return (w >> kSkOrderBit) & 1; }

// "tile" index tt of (active position pos, row block rb) in the unit order; unit u
// belongs to tile tt = u / nks
MT_DEV long long sk_tile(int order, int pos, int rb, int nact, int RB)
{
    return order ? (long long)rb * nact + pos : (long long)pos * RB + rb;
}
MT_DEV void sk_tile_coords(int order, long long tt, int nact, int RB, int* pos, int* rb)
{
    if (order) { *rb = (int)(tt / nact); *pos = (int)(tt - (long long)*rb * nact); }
    else { *pos = (int)(tt / RB); *rb = (int)(tt - (long long)*pos * RB); }
}

// The CTAs whose ranges touch tile t (units [t nks, (t+1) nks)) are first..last;
// the tile is the jf-th segment of CTA first and the first segment (slot 0) of
// every later one, because their ranges start inside it.
struct SkCover { int first, last, jf; };

MT_DEV SkCover sk_cover(long long t, long long nks, long long U, long long Gsel)
{
    const long long G = sk_ctas(U, Gsel);
    const long long x0 = t * nks, x1 = (t + 1) * nks;
    long long f = ((x0 + 1) * G + U - 1) / U - 1;
    long long l = (x1 * G + U - 1) / U - 1;
    if (f > G - 1) f = G - 1;
    if (l > G - 1) l = G - 1;
    if (f < 0) f = 0;
    SkCover cv;
    cv.first = (int)f;
    cv.last = (int)l;
    cv.jf = (int)(t - sk_start(f, U, G) / nks);
    return cv;
}

// GEMM-internal timers of CTA 0 (prof slots 16..23) when profiling is on
MT_DEV void i8_prof_add(unsigned long long* prof, int slot, unsigned long long v)
{
    if (prof && blockIdx.x == 0) atomicAdd(&prof[slot], v);
}

// The Stream-K share of this CTA in one tick: nact active instance tiles
// (act_jb[0..nact), 64 instances each), RB row blocks, nks k steps per tile.
// part: int64 slots [gridDim.x][maxseg][64][128].  Returns a CTA-uniform ok flag.
template <typename FT>
MT_DEV bool tc_i8_streamk(unsigned char* smem, const FT& F, long long* part, int maxseg, const TcMaps& maps,
                          const CUtensorMap* bmap, int nact, const int* act_jb, int RB, int nks, int sched,
                          TcState& st)
{
    I8Smem L = i8_layout(smem);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long long U = (long long)nact * RB * nks;
    const int order = sk_sched_order(sched);
    const long long G = sk_ctas(U, sk_sched_ctas(sched)), c = blockIdx.x;
    bool ok = true;
    if (c >= G) return __syncthreads_and(1) != 0;
    const long long u0 = sk_start(c, U, G), u1 = sk_start(c + 1, U, G);
    unsigned long long* prof = F.prof;
    const uint64_t t_in = globaltimer_ns();
    if (warp == 4 && lane == 0) {
        long long g = st.kb_done;
        unsigned long long wait_empty = 0;
        const uint64_t kpol = l2_evict_first_policy();
        for (long long u = u0; u < u1 && ok;) {
            const int t = (int)(u / nks), ks0 = (int)(u - (long long)t * nks);
            const long long ue = min(u1, (long long)(t + 1) * nks);
            int pos, rb;
            sk_tile_coords(order, t, nact, RB, &pos, &rb);
            const int jb = act_jb[pos];
            for (int ks = ks0; ks < ks0 + (int)(ue - u); ++ks, ++g) {
                const int stg = (int)(g % kI8Stages);
                const uint32_t ph = (uint32_t)((g / kI8Stages) & 1);
                const uint64_t tw = globaltimer_ns();
                if (!mbar_wait(smem_u32(&L.empty[stg]), ph ^ 1u, F.gs, 210)) { ok = false; break; }
                wait_empty += globaltimer_ns() - tw;
                uint8_t* base = L.stages + (size_t)stg * kI8StageBytes;
                const uint32_t fb = smem_u32(&L.full[stg]);
                mbar_expect_tx(fb, (uint32_t)kI8StageBytes);
                const int x = ks * kI8KB;
                for (int a = 0; a < kI8KLimbs; ++a)
                    tma_load_3d_hint(smem_u32(base + a * kI8ATile), &maps.ahi, x, rb * 128, a, fb, kpol);
                for (int b = 0; b < kI8MLimbs; ++b)
                    tma_load_3d(smem_u32(base + kI8KLimbs * kI8ATile + b * kI8BTile), bmap, x, jb * kI8N, b, fb);
            }
            u = ue;
        }
        i8_prof_add(prof, 20, wait_empty);
        i8_prof_add(prof, 21, (unsigned long long)(u1 - u0));
        if (!ok) {   // let loads already in flight land before the CTA moves on
            for (long long q = g - kI8Stages; q < g; ++q) {
                if (q < st.kb_done) continue;
                mbar_wait(smem_u32(&L.full[q % kI8Stages]), (uint32_t)((q / kI8Stages) & 1), F.gs, 213);
            }
        }
    } else if (warp == 5 && lane == 0) {
        long long g = st.kb_done, seg = st.tiles;
        unsigned long long wait_full = 0, wait_free = 0;
        for (long long u = u0; u < u1 && ok; ++seg) {
            const int t = (int)(u / nks), ks0 = (int)(u - (long long)t * nks);
            const long long ue = min(u1, (long long)(t + 1) * nks);
            // the accumulators of the previous segment must be drained first
            const uint64_t tf = globaltimer_ns();
            if (seg > 0 && !mbar_wait(smem_u32(L.tfree), (uint32_t)((seg - 1) & 1), F.gs, 214)) { ok = false; break; }
            wait_free += globaltimer_ns() - tf;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            for (int ks = ks0; ks < ks0 + (int)(ue - u); ++ks, ++g) {
                const int stg = (int)(g % kI8Stages);
                const uint32_t ph = (uint32_t)((g / kI8Stages) & 1);
                const uint64_t tw = globaltimer_ns();
                if (!mbar_wait(smem_u32(&L.full[stg]), ph, F.gs, 211)) { ok = false; break; }
                wait_full += globaltimer_ns() - tw;
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t base = smem_u32(L.stages + (size_t)stg * kI8StageBytes);
                // The four m-limb tiles of a stage lie back to back as one K-major operand of
                // 4 x 64 rows (8-row groups 1024 bytes apart), and accumulator D_s sits at
                // columns 64 s, so one MMA of K limb a against m limbs b0..b1 (N = 64 (b1 - b0 + 1))
                // adds K_a m_b into D_{a+b} for every b at once.  Five MMAs per 32-wide k step
                // cover the sixteen limb pairs: (0, 0..3) and (3, 1..3) open D0..D3 and D4..D6
                // at the first k step of a segment, then (1, 0..3), (2, 0..3) and (3, 0).
                const uint32_t bbase = base + kI8KLimbs * kI8ATile;
#pragma unroll
                for (int kk = 0; kk < kI8KB / 32; ++kk) {
                    const uint32_t open = (ks == ks0 && kk == 0) ? 0u : 1u;
                    const uint64_t b0 = sdesc_sw128(bbase + kk * 32);
                    const uint64_t b1 = sdesc_sw128(bbase + kI8BTile + kk * 32);
                    umma_i8(st.tmem, sdesc_sw128(base + kk * 32), b0, open, idesc_i8(4 * kI8N));
                    umma_i8(st.tmem + 4u * kI8N, sdesc_sw128(base + 3 * kI8ATile + kk * 32), b1, open,
                            idesc_i8(3 * kI8N));
                    umma_i8(st.tmem + 1u * kI8N, sdesc_sw128(base + 1 * kI8ATile + kk * 32), b0, 1u, idesc_i8(4 * kI8N));
                    umma_i8(st.tmem + 2u * kI8N, sdesc_sw128(base + 2 * kI8ATile + kk * 32), b0, 1u, idesc_i8(4 * kI8N));
                    umma_i8(st.tmem + 3u * kI8N, sdesc_sw128(base + 3 * kI8ATile + kk * 32), b0, 1u, idesc_i8(kI8N));
                }
                umma_commit(smem_u32(&L.empty[stg]));
            }
            if (ok) umma_commit(smem_u32(L.accum));
            u = ue;
        }
        i8_prof_add(prof, 16, wait_full);
        i8_prof_add(prof, 17, wait_free);
        i8_prof_add(prof, 22, (unsigned long long)(seg - st.tiles));
    }
    if (warp < 4) {
        long long seg = st.tiles;
        const long long tfirst = u0 / nks;
        unsigned long long wait_acc = 0, drain = 0;
        for (long long u = u0; u < u1; ++seg) {
            const int t = (int)(u / nks);
            const long long ue = min(u1, (long long)(t + 1) * nks);
            const uint64_t ta0 = globaltimer_ns();
            bool w = ok && mbar_wait(smem_u32(L.accum), (uint32_t)(seg & 1), F.gs, 212, 200);
            w = __all_sync(0xffffffffu, w);
            const uint64_t ta1 = globaltimer_ns();
            wait_acc += ta1 - ta0;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            if (!w) { ok = false; break; }
            const int row = warp * 32 + lane;
            long long* slot = part + ((size_t)c * maxseg + (size_t)(t - tfirst)) * kI8SlotElems;
#pragma unroll 1
            for (int grp = 0; grp < kI8N / 32; ++grp) {
                long long h[32];
                int d[32];
                const uint32_t ta = st.tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(grp * 32);
#pragma unroll 1
                for (int part = 0; part < 2; ++part) {
                    // part 0: D0..D3 (hi), part 1: D4..D6 (lo)
                    const int s0 = part ? 4 : 0, s1 = part ? kI8Acc : 4;
                    tmem_ld32_i(ta + (uint32_t)(s0 * kI8N), d);
#pragma unroll
                    for (int k = 0; k < 32; ++k) h[k] = (long long)d[k];
#pragma unroll 1
                    for (int s = s0 + 1; s < s1; ++s) {
                        tmem_ld32_i(ta + (uint32_t)(s * kI8N), d);
#pragma unroll
                        for (int k = 0; k < 32; ++k) h[k] = h[k] * 256 + (long long)d[k];
                    }
#pragma unroll
                    for (int k = 0; k < 32; ++k) slot[(size_t)part * kI8N * 128 + (size_t)(grp * 32 + k) * 128 + row] = h[k];
                }
            }
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive(smem_u32(L.tfree));
            drain += globaltimer_ns() - ta1;
            u = ue;
        }
        if (warp == 0 && lane == 0) { i8_prof_add(prof, 18, wait_acc); i8_prof_add(prof, 19, drain); }
    }
    const uint64_t t_body = globaltimer_ns();
    // every role walked the same segment list
    {
        long long nseg = 0, nk = 0;
        for (long long u = u0; u < u1; ++nseg) {
            const int t = (int)(u / nks);
            const long long ue = min(u1, (long long)(t + 1) * nks);
            nk += ue - u;
            u = ue;
        }
        st.kb_done += nk;
        st.tiles += nseg;
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    const bool all_ok = __syncthreads_and(ok ? 1 : 0) != 0;
    if (threadIdx.x == 0) { i8_prof_add(prof, 23, t_body - t_in); i8_prof_add(prof, 24, globaltimer_ns() - t_in); }
    return all_ok;
}

// exact demag sum of row lr of a tile for instance lj, rounded once to double:
// the hi and lo parts of the slots of the CTAs cv.first..cv.last that cover the
// tile are summed exactly in int64 and combined as RN(2^24 hi + lo).
// i8_tile_load issues the loads of the first three covering slots (most tiles have
// at most three; slots past the last cover are not loaded), i8_tile_finish adds the
// rest and rounds.
MT_DEV void i8_tile_load(const long long* part, int maxseg, const SkCover& cv, int lr, int lj, long long v[6])
{
    const size_t off = (size_t)lj * 128 + (size_t)lr, lo = (size_t)kI8N * 128;
    const long long* p0 = part + ((size_t)cv.first * maxseg + (size_t)cv.jf) * kI8SlotElems + off;
    const bool has1 = cv.first + 1 <= cv.last, has2 = cv.first + 2 <= cv.last;
    const long long* p1 = part + (size_t)(cv.first + 1) * maxseg * kI8SlotElems + off;
    const long long* p2 = part + (size_t)(cv.first + 2) * maxseg * kI8SlotElems + off;
    v[0] = __ldcg(p0);
    v[1] = __ldcg(p0 + lo);
    v[2] = has1 ? __ldcg(p1) : 0ll;
    v[3] = has1 ? __ldcg(p1 + lo) : 0ll;
    v[4] = has2 ? __ldcg(p2) : 0ll;
    v[5] = has2 ? __ldcg(p2 + lo) : 0ll;
}

MT_DEV double i8_tile_finish(const long long* part, int maxseg, const SkCover& cv, int lr, int lj, const long long v[6])
{
    const size_t off = (size_t)lj * 128 + (size_t)lr, lo = (size_t)kI8N * 128;
    long long hi_s = v[0] + v[2] + v[4], lo_s = v[1] + v[3] + v[5];
    for (int c = cv.first + 3; c <= cv.last; ++c) {
        const long long* pc = part + (size_t)c * maxseg * kI8SlotElems + off;
        hi_s += __ldcg(pc);
        lo_s += __ldcg(pc + lo);
    }
    return __dadd_rn(__dmul_rn((double)hi_s, 16777216.0), (double)lo_s);
}

MT_DEV double i8_tile_sum(const long long* part, int maxseg, const SkCover& cv, int lr, int lj)
{
    long long v[6];
    i8_tile_load(part, maxseg, cv, lr, lj, v);
    return i8_tile_finish(part, maxseg, cv, lr, lj, v);
}
