/*
 * magtense_b200.h -- C ABI of libmagtense_b200.so, the B200-native micromagnetic
 * hot path of MagTense (Landau-Lifshitz right-hand side, dense prism demag
 * tensor, adaptive Runge-Kutta integration).
 *
 * Conventions (all as in the reference, MagTense source/MagTenseMicroMag):
 *  - n = nx*ny*nz cells on a uniform grid, cell index i + j*nx + k*nx*ny.
 *  - A magnetisation state is one FP64 vector [mx(0..n-1), my(..), mz(..)].
 *  - "H" arrays are the reference's internal fields, i.e. MINUS the physical
 *    field (LandauLifshitzEquationSolver.f90:453,494-507,542-544,715-754).
 *  - alpha is the reference's damping coefficient gamma*alpha_Gilbert.
 *
 * Every function returns an int status: 0 on success, a negative MT_ERR_* code
 * otherwise; nothing here exits, aborts or traps.  mt_last_error() gives a
 * message for the calling thread's last failure.  Pointers named *_dev are
 * device pointers (any allocator); everything else is host memory.  Streams
 * are passed as void* (a cudaStream_t; NULL = legacy default stream).
 * Distinct handles may be used from different threads concurrently; one handle
 * must not be used concurrently.
 */
#ifndef MAGTENSE_B200_H
#define MAGTENSE_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define MT_OK 0
#define MT_ERR_ARG (-1)          /* invalid argument */
#define MT_ERR_CUDA (-2)         /* CUDA runtime error */
#define MT_ERR_NOMEM (-3)        /* device allocation failed */
#define MT_ERR_STATE (-4)        /* call out of order (e.g. no tensor yet) */
#define MT_ERR_UNSUPPORTED (-5)  /* feature not on this path */
#define MT_ERR_SOLVER (-6)       /* integrator stopped (see mt_stats.status) */
#define MT_ERR_TIMEOUT (-7)      /* a bounded device wait gave up */

typedef struct mt_handle mt_handle;

/* Uniform grid; mirrors MicroMagGrid (MicroMagParameters.f90:57-70). */
typedef struct {
    int nx, ny, nz;
    double Lx, Ly, Lz;
} mt_grid;

/* Integrator statistics (RKSUITE counters, RKSuitef90.f90:41-100). */
typedef struct {
    long long f_evals;     /* right-hand-side evaluations */
    long long steps;       /* accepted steps */
    long long bad_steps;   /* rejected steps (after the first step) */
    long long n_flag3;     /* "too much work" returns (every 5000 evaluations) */
    long long n_flag4;     /* "problem looks stiff" returns */
    long long n_out;       /* output samples written */
    int status;            /* 0 ok; 5 step size underflow; 911 fatal argument */
    int converged_at;      /* output index where the t_conv test ended the run, -1 if none */
    long long launches;    /* persistent-kernel launches used */
    double kernel_ms;      /* device time of those launches (CUDA events on the stream) */
} mt_stats;

/* ---------------- handle life cycle ---------------- */

/* Replaces the per-process globals of MagTenseCudaBlas.cu:29-92 with a handle.
 * Allocates nothing on the device yet. */
int mt_create(const mt_grid* grid, mt_handle** out);
int mt_destroy(mt_handle* h);
const char* mt_last_error(void);
const char* mt_version(void);

/* Per-cell material (loadMicroMagProblem, MagTenseMicroMagPyIO.f90:91-100;
 * initializeSolution :415-422).  Ms, K0: n values; u_ea: n*3 row-major
 * (u_ea[i*3+c]); A0 scalar.  Host arrays. */
int mt_set_material(mt_handle* h, double A0, const double* Ms, const double* K0, const double* u_ea);

/* Time dependence (updateExternalField :485-514, alpha() :281-294).
 * solver: 1 explicit (field row hext_row, 0-based), 2 dynamic (interpolated).
 * hext: nt_hext rows of {t, Hx, Hy, Hz} (A/m); alpha_tab: nt_alpha rows of
 * {t, alpha}, used when alpha0 == 0.  renormalize: rescale each cell's m to
 * unit length after every accepted step (off in the reference's RKSUITE path). */
int mt_set_dynamics(mt_handle* h, int solver, double gamma, double alpha0,
                    const double* alpha_tab, int nt_alpha, const double* hext, int nt_hext,
                    int hext_row, int renormalize);

/* ---------------- demag tensor ---------------- */

/* Analytical prism tensor of every (receiver, source) pair, FP64 on the GPU and
 * rounded to FP32 (ComputeDemagfieldTensor uniform branch,
 * LandauLifshitzEquationSolver.f90:883-986; getN_prism_3D,
 * TileNComponents.f90:629-724). */
int mt_assemble_demag(mt_handle* h, void* stream);

/* Reference layout in/out: six column-major n*n FP32 blocks Kxx Kxy Kxz Kyy Kyz
 * Kzz, K(:,src) = field at every receiver from source src (host memory).  This
 * is the record layout of writeDemagTensorToDisk/loadDemagTensorFromDisk
 * (MagTenseMicroMagPyIO.f90:221-271). */
int mt_load_demag_colmajor(mt_handle* h, const float* Kxx, const float* Kxy, const float* Kxz,
                           const float* Kyy, const float* Kyz, const float* Kzz);
int mt_get_demag_colmajor(mt_handle* h, float* Kxx, float* Kxy, float* Kxz,
                          float* Kyy, float* Kyz, float* Kzz);

/* Thresholded-sparse demag (dem_appr "threshold" = 2 / "threshold_fraction" = 4 of
 * MagTenseMicroMagPyIO.f90; ApplyThresholdDense, DemagAuxFunctions.f90:20-122, and
 * ConvertDenseToSparse_s, util_micromag.f90:81-138): keeps the entries of the
 * assembled or loaded tensor with |K| > threshold and from then on computes every
 * demag product (fields, right-hand side, integration) on those entries only.
 * approx 2: value is the threshold; approx 4: value is the fraction of the positive
 * entries to remove, turned into a threshold by the bisection of FindThresholdFraction
 * (:353-428; a fraction >= 1 removes everything); approx 1 returns to the dense
 * product.  Reports the kept entries (of the 9 block rows per cell; the symmetric
 * blocks count twice) and the threshold used.  Assembling or loading a tensor
 * again drops the sparse one.  Not for row shards or batches. */
int mt_set_demag_threshold(mt_handle* h, int approx, double value, long long* nnz_out, float* threshold_out,
                           void* stream);

/* ---------------- fields and right-hand side ---------------- */

/* Internal demag field Hm = Ms * (-K m) with m rounded to FP32 and an FP32
 * product (updateDemagfield dense branch :706-767).  m_dev, H_dev: 3n FP64. */
int mt_demag_field(mt_handle* h, const double* m_dev, double* H_dev, void* stream);

/* All four internal field terms at time t (StoreHeffComponents :306-349). */
int mt_fields(mt_handle* h, double t, const double* m_dev, double* Hj_dev, double* Hh_dev,
              double* Hk_dev, double* Hm_dev, void* stream);

/* dm/dt of the Landau-Lifshitz equation (dmdt_fct :220-273). */
int mt_rhs(mt_handle* h, double t, const double* m_dev, double* dmdt_dev, void* stream);

/* Vector-Jacobian product of mt_rhs at (t, m) for the cotangent lam (3n): the
 * gradient with respect to m (gm, 3n), the cotangent of the internal field
 * he = Hh + Hj + Hm + Hk (ghe, 3n; the applied-field gradient is -sum over
 * cells of ghe) and the gradient with respect to the per-cell Ms (gms, n).
 * The demag and exchange operators are symmetric, so their transposes run the
 * forward kernels.  No counterpart in the reference (it has no derivatives);
 * used by the adjoint of a trajectory (magtense_b200.adjoint). */
int mt_rhs_vjp(mt_handle* h, double t, const double* m_dev, const double* lam_dev, double* gm_dev,
               double* ghe_dev, double* gms_dev, void* stream);

/* Ragged batch: ninst independent instances, each with its own handle (grid,
 * tensor, material, dynamics), integrated like mt_integrate over the same
 * output times in ONE cooperative launch (relaunched in slices of about 0.25 s).
 * Instance k runs on its own group of CTAs, sized by its demag work n_k^2, with
 * its own barrier and adaptive steps; ninst must not exceed the SM count.
 * m0_dev[k], y_out_dev[k] (nt * 3 n_k): device buffers of instance k; t_out,
 * flags: ninst * nt; stats: ninst (launches and kernel_ms in stats[0]).
 * options: MT_RAGGED_GRAPH captures the launch sequence in a CUDA graph once
 * and replays it.  No counterpart in the reference (one problem per process). */
#define MT_RAGGED_GRAPH 1
int mt_integrate_ragged(mt_handle* const* hs, int ninst, const double* t, int nt, const double* const* m0_dev,
                        double tol, double thres, double* t_out, double* const* y_out_dev, int* flags,
                        mt_stats* stats, int options, void* stream);

/* Row shards of ONE instance over `world` ranks, one GPU each (1 < world <= 8).
 * Rank r keeps the tensor rows of the receiver cells
 * [n*r/world, n*(r+1)/world) only (24 n^2 / world bytes), and integrates those
 * cells; each stage argument is all-gathered by peer stores into every rank's
 * exchange region, and the error norms are combined over all ranks, so every
 * rank takes the same adaptive steps as the whole instance.  No counterpart in
 * the reference, which holds the whole tensor in one process
 * (LandauLifshitzEquationSolver.f90:881-986, MagTenseCudaBlas.cu:29-92).
 *
 * Order on each rank: mt_create, mt_set_row_shard, mt_set_material,
 * mt_set_dynamics, mt_assemble_demag (own rows), mt_shard_region, then the
 * peers' regions through mt_shard_open_peers (IPC handles from
 * mt_shard_ipc_handle, one process per GPU) or mt_shard_set_peers (pointers
 * the caller has mapped), then mt_integrate on every rank at the same time:
 * each rank fills its own cells' rows of y_out (and the whole first sample).
 * A sharded handle serves no other compute entry point (MT_ERR_UNSUPPORTED).
 * A wait for the other ranks gives up after 10 s (environment variable
 * MAGTENSE_B200_SHARD_TIMEOUT_S, read by mt_integrate, sets another bound) with
 * MT_ERR_TIMEOUT; the ranks' barrier epochs then differ: destroy the handles. */
int mt_set_row_shard(mt_handle* h, int rank, int world);
/* This rank's exchange region (device memory, allocated on the first call). */
int mt_shard_region(mt_handle* h, void** region_dev, size_t* bytes);
/* cudaIpcMemHandle_t of the region (64 bytes into handle_out). */
int mt_shard_ipc_handle(mt_handle* h, void* handle_out);
/* Map the peers' regions from their IPC handles (world * 64 bytes, rank order;
 * this rank's entry is ignored). */
int mt_shard_open_peers(mt_handle* h, const void* handles);
/* Peer regions given as device pointers valid in this process (world entries,
 * rank order; this rank's entry must be its own region). */
int mt_shard_set_peers(mt_handle* h, void* const* regions_dev);
/* All `world` ranks of a row-sharded instance on ONE device, as CTA groups of one
 * cooperative launch (the multi-GPU code path, with peer stores into local
 * memory).  hs: the ranks' handles in rank order, peers set with
 * mt_shard_set_peers; y_out_dev (nt * 3n) is shared, each rank writing its own
 * rows; other arguments as mt_integrate, statistics of rank 0. */
int mt_integrate_shards_local(mt_handle* const* hs, int world, const double* t, int nt, const double* m0_dev,
                              double tol, double thres, const double* t_conv, int nt_conv, double conv_tol,
                              double* t_out, double* y_out_dev, int* flags, mt_stats* stats, void* stream);

/* Allocation-free dm/dt.  No counterpart in the reference: it exists for
 * callers that may not allocate device memory (for example a host framework
 * that owns all device memory through its own pool, or a host program whose
 * device-memory budget is fixed once it has started).  Same result as mt_rhs,
 * but the FP32 copy of m that
 * the demag product reads lives in a fixed array inside the library
 * (3 * MT_NOALLOC_MAX_CELLS floats, held on every GPU that loads the library
 * until the process exits) instead of memory allocated on first use; the call
 * allocates nothing and rejects grids with more than MT_NOALLOC_MAX_CELLS
 * cells (MT_ERR_ARG).  The handle must already hold the tensor, material and
 * dynamics.  The first call on a device looks up the array's device address
 * (once per device, with that device current); make that first call before
 * any stream capture.  All calls share the one array: calls that overlap on
 * the GPU (different streams, or different handles on the same device) race
 * and must be serialised by the caller.  Each call rewrites the whole array
 * region it uses before reading it. */
#define MT_NOALLOC_MAX_CELLS 16384
int mt_rhs_noalloc(mt_handle* h, double t, const double* m_dev, double* dmdt_dev, void* stream);

/* ---------------- time integration ---------------- */

/* MagTense_ODE_RKSuite (ODE_Solvers.f90:124-237) driving RKSUITE-90 method 'M'
 * (RKSuitef90.f90), executed on the device by one persistent cooperative
 * kernel.  t: nt requested output times (host); m0_dev: 3n FP64; y_out_dev:
 * nt*3n FP64 (sample k at y_out_dev + k*3n); t_out, flags: nt host values (the
 * time each sample was taken at, and the RKSUITE flag of the call that produced
 * it: 1 normal, 3/4 warning return before t_want was reached).  t_conv: times
 * at which max|m - m_last| < conv_tol stops the run (ODE_Solvers.f90:210-222).
 * Blocks the calling thread until done. */
int mt_integrate(mt_handle* h, const double* t, int nt, const double* m0_dev, double tol,
                 double thres, const double* t_conv, int nt_conv, double conv_tol,
                 double* t_out, double* y_out_dev, int* flags, mt_stats* stats, void* stream);

/* ---------------- batched instances sharing one geometry ---------------- */
/* B independent problems on the same grid, material and demag tensor, each
 * with its own applied-field table, damping and initial state (the dataset
 * workflow of python/scripts/database.py:19-87 and db_utils.py:50-82, run as
 * one call).  Every instance keeps its own RKSUITE 'M' step control; the demag
 * products of all instances form one GEMM per right-hand-side evaluation. */
typedef struct mt_batch mt_batch;

#define MT_PREC_FP32 0     /* FP32 SIMT product, same arithmetic as the single-instance path */
#define MT_PREC_BF16X3 1   /* tcgen05, K and m split into BF16 hi+lo, 3 products, FP32 accumulate */
#define MT_PREC_BF16X2 2   /* tcgen05, K split hi+lo, m in BF16, 2 products, FP32 accumulate */
#define MT_PREC_FP16X3S 3  /* tcgen05, rows of K scaled by powers of two, K and m split into FP16 hi+lo,
                              3 products, FP32 accumulate (about FP32 accuracy) */
#define MT_PREC_INT8 4     /* tcgen05 kind::i8, rows of K as 32-bit fixed point (4 int8 limbs), m as
                              rint(m 2^30) (4 limbs), all 16 limb products accumulated exactly in
                              int32/int64: the product is exact for the quantised operands, so it
                              carries no rounding noise; needs |m| < 1.96 (MT_ERR_ARG otherwise) and
                              at most 10624 cells */

int mt_batch_create(const mt_grid* grid, int B, int precision, mt_batch** out);
int mt_batch_destroy(mt_batch* b);
/* shared material, as mt_set_material */
int mt_batch_set_material(mt_batch* b, double A0, const double* Ms, const double* K0, const double* u_ea);
/* per-instance time dependence: alpha0[B]; hext[B][nt_hext][4] (rows {t,Hx,Hy,Hz});
 * solver 1 (explicit) uses row 0 of each instance's table */
int mt_batch_set_dynamics(mt_batch* b, int solver, double gamma, const double* alpha0, const double* hext,
                          int nt_hext, int renormalize);
/* damping table alpha_tab[nt_alpha][2] (rows {t, alpha}) shared by the instances whose
 * alpha0 is 0: alpha() of LandauLifshitzEquationSolver.f90:281-294 (interp1 of the table,
 * 0 outside it), as mt_set_dynamics's alpha_tab; may come before or after
 * mt_batch_set_dynamics */
int mt_batch_set_alpha_table(mt_batch* b, const double* alpha_tab, int nt_alpha);
int mt_batch_assemble_demag(mt_batch* b, void* stream);
/* Autotuner of the int8 product's GEMM schedule (no counterpart in the reference,
 * whose product is an MKL/cuBLAS SGEMV, LandauLifshitzEquationSolver.f90:718-747):
 * for every count of active 64-instance tiles, times the candidate schedules on the
 * device (Stream-K CTA count, tile-major or row-major unit order) and keeps the
 * fastest for the integrations of this handle; cached per device and geometry for
 * the process.  Every schedule gives the same bits.  A no-op for the other
 * precisions.  Needs the assembled tensor. */
int mt_batch_tune(mt_batch* b, void* stream);
/* the schedule in use: per active tile count k = 1..n_tiles, ctas[k-1] and order[k-1]
 * (0 tile-major, 1 row-major); fills at most max_tiles entries */
int mt_batch_get_schedule(mt_batch* b, int* ctas, int* order, int max_tiles, int* n_tiles);
/* set the schedule by hand (n_tiles entries; CTA counts from two thirds of the SMs up
 * to all of them, order 0 or 1), for example to replay a tuned one */
int mt_batch_set_schedule(mt_batch* b, const int* ctas, const int* order, int n_tiles);
/* m0_dev: B*3n FP64; y_out_dev: B*nt*3n FP64 or NULL; t_out, flags: B*nt host;
 * stats: B entries (kernel_ms/launches of the whole batch in stats[0]). */
int mt_batch_integrate(mt_batch* b, const double* t, int nt, const double* m0_dev, double tol, double thres,
                       const double* t_conv, int nt_conv, double conv_tol, double* t_out, double* y_out_dev,
                       int* flags, mt_stats* stats, void* stream);
/* the same, with the trajectories also delivered to page-locked host memory y_out_host
 * ([B][nt][3n] FP64), as the reference returns M(t) in host arrays
 * (MagTenseMicroMagPyIO.f90:200-206, the intent(out) M of runMicroMagSimulation): after
 * every relaunch of the persistent kernel the samples that all unfinished instances have
 * passed are copied there on a stream of their own while the next launch runs.
 * y_out_dev is still required as the device copy.  MT_ERR_ARG if y_out_host is not
 * page-locked. */
int mt_batch_integrate_host(mt_batch* b, const double* t, int nt, const double* m0_dev, double tol, double thres,
                            const double* t_conv, int nt_conv, double conv_tol, double* t_out, double* y_out_dev,
                            double* y_out_host, int* flags, mt_stats* stats, void* stream);
/* demag field of all instances with the batch's precision: H_dev = -Ms K m, B*3n FP64 */
int mt_batch_demag_field(mt_batch* b, const double* m_dev, double* H_dev, void* stream);

/* ---------------- reference compatibility shims ---------------- */
/* Exact signatures of the reference's C shim (MagTenseCudaBlasICLWrapper.cxx:13-59,
 * bound from Fortran in FortranCuda.f90:15-60).  They act on one process-wide
 * problem like the reference, but return a status instead of exiting. */

/* replaces cu_initDemagMatrices (MagTenseCudaBlas.cu:306-352) */
int icl_initDemagMatrices(const float* Kxx, const float* Kxy, const float* Kxz,
                          const float* Kyy, const float* Kyz, const float* Kzz, int* n);
/* replaces cu_MVMult_GetH (MagTenseCudaBlas.cu:367-407): H = pref * K * M, FP32 host vectors */
int icl_MVMult_GetH(const float* Mx, const float* My, const float* Mz, float* Hx, float* Hy,
                    float* Hz, int* n, float* pref);
/* replaces cu_destroy (MagTenseCudaBlas.cu:420-497) */
int icl_destroy(void);
/* replace cu_initDemagMatrices_sparse / cu_MVMult_GetH_sparse (MagTenseCudaBlas.cu:106-297):
 * called six times, once per block (mat_no 1..6 = xx xy xz yy yz zz), with 1-based CSR
 * (rowInds of n + 1 entries, rowInds[n] = nnz + rowInds[0]); when all six are in, the
 * product H = pref * K * M (FP32 host vectors) runs on the kept entries. */
int icl_initDemagMatrices_sparse(int* n, int* nnz, int* mat_no, float* values, int* colInds,
                                 int* rowInds);
int icl_MVMult_GetH_sparse(const float* Mx, const float* My, const float* Mz, float* Hx, float* Hy,
                           float* Hz, const int* n, const float* pref);

#ifdef __cplusplus
}
#endif
#endif /* MAGTENSE_B200_H */
