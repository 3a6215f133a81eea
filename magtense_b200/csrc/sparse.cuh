// Thresholded-sparse demag tensor: device kernels of its construction (sparse.cu).
#pragma once
#include <cuda_runtime.h>

// kept entries (|K| > thr) of every receiver row 3 i + a of the cell-row tensor
cudaError_t sparse_count_rows(const float* K, int n, int ldk, float thr, int* counts, cudaStream_t s);
// the kept entries in CSR order (rowptr: exclusive scan of the counts)
cudaError_t sparse_fill_rows(const float* K, int n, int ldk, float thr, const int* rowptr, int* col, float* val,
                             cudaStream_t s);
// over the positive entries of the six blocks: out[0] = their count, out[1] = those <= f
cudaError_t sparse_count_positive(const float* K, int n, int ldk, float f, unsigned long long* out, cudaStream_t s);
// smallest and largest positive entry, as float bit patterns: out[0], out[1]
cudaError_t sparse_positive_minmax(const float* K, int n, int ldk, unsigned* out, cudaStream_t s);
