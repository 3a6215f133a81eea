// Shared declarations of the persistent integrator (integrate.cu) and its host driver (capi.cu).
#pragma once
#include "common.cuh"
#include "llg.cuh"

constexpr int kIntegThreads = 512;

// Scalar state of RKSUITE (rk_comm_real_1d, RKSuitef90.f90:41-100) plus the
// output driver position.  Kept identical in every thread of the persistent
// kernel and stored in global memory between launches.
struct RKS {
    double t, t_old, t_start, t_end, dir, h, h_old, h_average, tol, errold, tlast, range_t_end;
    long long f_count, full_f_count, step_count, bad_step_count, stiff_bad_step_count;
    long long n_flag3, n_flag4;
    int at_t_start, at_t_end, phase2, chkeff, hit_t_end_count, intrp_ready;
    int iy, iyold, ia0, ia1;       // roles of the four state/argument buffers
    int dyp, dypold, d8;           // roles of the three derivative buffers
    int in_range;                  // a range_integrate call is in progress
    int ci;                        // next entry of the merged output-time list
    int ko;                        // next output slot
    int finished, status, converged_at;
    long long xseq;                // row shards: cross-rank barriers passed since the exchange region was made
    long long rseq;                // reductions since then (parity of the partials buffer)
};

// Row shards of one instance (one rank per GPU).  Rank r owns the receiver cells
// [cell0, cell0 + ncell) and the tensor rows of those cells only.  Every rank keeps a
// full copy of the stage arguments: a rank writes its own cells' values into all
// ranks' exchange regions (peer stores), and the group barrier becomes local barrier,
// release/acquire flags between ranks at system scope.  Reductions
// write each CTA's partial into every region and combine all ranks' partials in the
// same order everywhere, so all ranks take identical steps.
constexpr int kMaxShards = 8;
constexpr int kShardMaxCtas = 256;   // per rank, for the partials slots

struct ShardLink {
    int rank, world;
    int cell0, ncell;              // this rank's receiver cells
    int cta_base, cta_total;       // this rank's first global CTA index; CTAs over all ranks
    double* pool[kMaxShards][4];   // each rank's stage-argument buffers (3n FP64)
    float* pool32[kMaxShards][4];  // each rank's FP32 shadows [3][ldk]
    double* partials[kMaxShards];  // each rank's reduction slots [2][cta_total][4]
    unsigned* flags[kMaxShards];   // each rank's barrier flags: slot p is written by rank p; slot
                                   // kMaxShards is the rank's sticky abort word (any rank may raise it)
    unsigned long long timeout_ns; // bound on one wait for the other ranks
};

// Byte offsets inside one rank's exchange region (identical on every rank).
struct ShardLayout {
    size_t pool, pool32, partials, flags, bytes;
};
inline ShardLayout shard_layout(int n, int ldk, int world)
{
    auto up = [](size_t v) { return (v + 255) & ~(size_t)255; };
    ShardLayout L;
    L.pool = 0;
    L.pool32 = up(L.pool + sizeof(double) * 4 * 3 * (size_t)n);
    L.partials = up(L.pool32 + sizeof(float) * 4 * 3 * (size_t)ldk);
    L.flags = up(L.partials + sizeof(double) * 2 * (size_t)world * kShardMaxCtas * 4);
    L.bytes = up(L.flags + sizeof(unsigned) * (kMaxShards + 1));
    return L;
}

struct IntegBufs {
    double* pool[4];       // 3n FP64: y, y_old and two stage-argument buffers (rotating)
    float* pool32[4];      // FP32 shadows [3][ldk] of pool (demag product input)
    double* deriv[3];      // 3n FP64: yp, yp_old, stage 8 (rotating)
    double* stg[12];       // stages 2..7 and 9..11 (index = stage number)
    double* p[6];          // interpolant coefficients 1..5
    double* errest;
    double* weights;
    double* ylast;         // last sample checked for convergence
    double* ystep;         // sample buffer when the sample is not stored
    double* y_out;         // nt * 3n
    double* partials;      // 2 * grid * 4 reduction partials
    GridSync* gs;
    RKS* state;
    const ShardLink* link;  // row shards (device memory), nullptr for a whole instance
};

struct IntegParams {
    double thres;
    double round_off, sqrrmc, cubrmc, sqtiny, toosml;
    double conv_tol;
    const double* comb_t;      // merged, unique, sorted output + convergence times
    const int* comb_flags;     // bit 0: store sample, bit 1: convergence check
    int ncomb, nt;
    double* t_out;             // device, nt
    int* flags_out;            // device, nt
    long long evals_per_launch;
    int renorm;
};

// one instance of a ragged launch and its CTA group
struct RaggedInst {
    DevProb P;
    IntegBufs B;
    IntegParams Q;
    int cta0, ncta;
};

cudaError_t integrate_upload_tables();
int integrate_grid_size(int n, int num_sms);
size_t integrate_smem_bytes(int n, int ldk, int grid);
cudaError_t launch_integrate(const DevProb& P, const IntegBufs& B, const IntegParams& Q, int grid,
                             cudaStream_t stream);
cudaError_t launch_integrate_ragged(const RaggedInst* inst_dev, const int* cta_inst_dev, int grid, size_t smem,
                                    cudaStream_t stream);
