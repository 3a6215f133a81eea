// Batched integration: B instances that share one geometry (tensor, material)
// and differ in applied field, damping and initial state.  Declarations shared
// by batch.cu (persistent kernel), gemm_tc.cuh (tcgen05 demag GEMM) and capi.cu.
#pragma once
#include "common.cuh"
#include "integrate.cuh"
#include "llg.cuh"

constexpr int kBatchThreads = 512;
constexpr int kCellBlock = 128;   // receiver cells per tile (tcgen05 M = 128)
constexpr int kInstBlock = 128;   // instances per tile (tcgen05 N = 128)
constexpr int kRedSlots = 4;      // values per reduction

enum BatchPrecision { kPrecFP32 = 0, kPrecBF16x3 = 1, kPrecBF16x2 = 2, kPrecFP16x3S = 3, kPrecI8 = 4 };
constexpr int kMaxIB = 64;        // instance blocks (B <= 8192)

// Per-instance coroutine state: RKSUITE scalars plus the resume point and the
// locals that live across a yield.  One private copy per owning CTA.
struct BInst {
    RKS s;
    int pc;            // resume label
    int req;           // 0 none, 1 right-hand side, 2 reduction, 3 done
    int rhs_arg;       // pool index of the argument
    int rhs_dst;       // destination vector id (see batch.cu)
    double t_rhs;
    int red_k, red_max;
    int red_seq, red_pad;   // reductions completed in this launch (arrival-counter target)
    double red[kRedSlots];
    // locals of the synchronous formulation
    int i_stage, failed, phase3, ier, ntry, maybe, lots, sure, dst_slot, cf, flag, argi;
    double htry, hmin, err, tstg, t_want, t_got, scale, v0v0, v1v1, v1v0, v2v2, v2v0, v2v1, v3v3, v3v1, v3v2;
    double rold, rho, alpha1, beta1;
    double root_re[2], root_im[2];
    long long budget_mark;
};

struct BatchBufs {
    // per-instance vectors [k][Bp][3n] FP64 unless noted
    double* pool;      // 4 rotating state/argument buffers
    double* deriv;     // 3 rotating derivative buffers
    double* stg;       // stages 2..7, 9..11 (12 slots, index = stage)
    double* p;         // interpolant coefficients 1..5 (6 slots)
    double* errest;
    double* weights;
    double* ylast;
    double* ystep;
    double* y_out;     // [Bp][nt][3n] or nullptr
    double* mavg_out;  // [Bp][nt][3] (spatial average of each sample) or nullptr
    double* t_out;     // [Bp][nt]
    int* flags_out;    // [Bp][nt]
    // GEMM operands/results
    float* m32;        // [Bp][3][ldk] FP32 argument (fp32 backend)
    uint16_t* mhi;     // [Bp][Kd] BF16 argument, K-major (tcgen05 backends)
    uint16_t* mlo;
    int8_t* mlimb;     // [4][Bp][Kd] int8 limbs of the argument (int8 backend)
    int8_t* mcomp;     // [4][Bp][Kd] the limbs of this tick's requesting instances, packed (int8 backend)
    unsigned* reqbits; // [3][Bp / 32] instances that request a right-hand side (int8 backend)
    float* hpart;      // [S][Bp][3][np] partial demag sums
    long long* part;   // [G][maxseg][64][128] exact int64 segment sums (int8 backend)
    double* partials;  // [2][Bp][kRedSlots][CB] reduction partials (two halves by reduction parity)
    unsigned* redcnt;  // [Bp] arrivals of the instance's cell-block CTAs at its reductions (zero per launch)
    BInst* inst;       // [CB][Bp] private coroutine copies
    GridSync* gs;
    unsigned* counters;  // [3][2]: active instances, right-hand-side requests
    unsigned* ibreq;     // [3][2 IB]: right-hand-side requests per 64-instance tile
    unsigned long long* prof;  // [48] phase times (ns) and counters seen by CTA 0, or nullptr
    // per-instance inputs
    const double* hext;    // [Bp][nt_hext][4]
    const double* alpha0;  // [Bp]
};

struct BatchParams {
    int Bp, B, CB, IB, S, np, Kd, nt, ncomb, nt_hext;
    int prec;
    double thres, round_off, sqrrmc, cubrmc, sqtiny, toosml, conv_tol;
    const double* comb_t;
    const int* comb_flags;
    long long ticks_per_launch;
    long long evals_budget;   // per instance per launch
    int renorm;
    int demag_only;           // 1: one GEMM, write -Ms*H to out_h and return
    double* out_h;            // [B][3n] when demag_only
    // tcgen05 operands
    const uint16_t* khi;      // [3np][Kd] BF16 tensor (rows (a,i), cols (b,j))
    const uint16_t* klo;
    const float* row_inv;     // [3np] 1/s_r of the fp16s tensor rows
    // int8 backend: Stream-K geometry and the per-row scale 2^(-30 - e_r)
    int RB, nks, maxseg;
    const double* row_scale;  // [3np]
    // Stream-K schedule word (CTA count, unit order) per active tile count 0..2 kMaxIB,
    // picked by the autotuner (mt_batch_tune) or the default (all CTAs, tile-major)
    int sk_sched[2 * kMaxIB + 1];
    int tune_nact;            // > 0: demag_only times the product over this many tiles with tune_sched
    int tune_sched;
    // coroutine copies in dynamic shared memory at this offset (0: local memory), per warp
    int inst_smem_off, inst_per_warp;
    size_t inst_smem_bytes;
};

cudaError_t batch_upload_tables();
int batch_grid(int n, int B, int num_sms, int prec, int* CB, int* IB, int* S);
size_t batch_smem_bytes(int n, int ldk, int prec);
size_t batch_inst_smem(int n, int ldk, int prec, int per_cta, int* off, int* per_warp);
cudaError_t launch_batch(const DevProb& P, const BatchBufs& Bf, const BatchParams& Q, int grid, const void* tmaps,
                         cudaStream_t s, const void* l2_base = nullptr, size_t l2_bytes = 0, float l2_hit = 0.f);
cudaError_t launch_split_tensor(const float* K, int n, int ldk, int np, int prec, uint16_t* khi, uint16_t* klo,
                                float* row_inv, cudaStream_t s);
cudaError_t launch_batch_operand(const double* m, int B, int n, int ldk, int np, int prec, float* m32, uint16_t* mhi,
                                 uint16_t* mlo, int8_t* mlimb, int Bp, GridSync* gs, cudaStream_t s);
cudaError_t launch_limb_tensor(const float* K, int n, int ldk, int np, int8_t* klimb, double* row_scale,
                               cudaStream_t s);
int batch_i8_maxseg(int RB, int nks, int JB, int G);
