// Host launchers of the stand-alone field kernels (fields.cu) and the tensor assembly (assemble.cu).
#pragma once
#include "llg.cuh"

constexpr int kFieldThreads = 256;

cudaError_t launch_m_to_f32(const double* m, int n, int ldk, float* m32, cudaStream_t s);
cudaError_t launch_pack3_f32(const float* x, const float* y, const float* z, int n, int ldk, float* m32,
                             cudaStream_t s);
int field_cells_per_cta(int n, int num_sms);
// mode 0: internal demag field (o0); 1: Hj,Hh,Hk,Hm (o0..o3); 2: dm/dt (o0); 3: pref*K*m32 -> h32 (FP32);
// 4, 5: the two passes of the vector-Jacobian product of dm/dt (see fields.cu)
cudaError_t launch_field(int mode, const DevProb& P, const double* m, const float* m32, double t, double* o0,
                         double* o1, double* o2, double* o3, float* h32, float pref, int num_sms, cudaStream_t s);

// tensor rows of the receiver cells [row0, row0 + nrows) into K (nrows * 6 * ldk floats)
cudaError_t launch_assemble(int nx, int ny, int nz, const double L[3], const double d[3], int n, int ldk, int row0,
                            int nrows, float* K,
                            cudaStream_t s);
cudaError_t launch_colmajor_to_rows(const float* blk, int c, int n, int ldk, float* K, cudaStream_t s);
cudaError_t launch_rows_to_colmajor(const float* K, int c, int n, int ldk, float* blk, cudaStream_t s);
