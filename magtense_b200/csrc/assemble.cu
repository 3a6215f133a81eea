// Analytical prism demag tensor, assembled on the GPU in FP64 and rounded to FP32.
//
// Restates getN_prism_3D (source/TileDemagTensor/TileDemagTensor/TileNComponents.f90:629-724)
// and its helpers f_3D, g_3D, h_3D, FF_3D, GG_3D, HH_3D, getF_limit
// (TileRectangularPrismTensor.f90:7-149), evaluated for every (receiver,
// source) pair of the uniform grid as ComputeDemagfieldTensor does
// (LandauLifshitzEquationSolver.f90:929-986: tile centred on the source cell,
// diffPos = pts(receiver) - offset, identity rotation).
//
// This translation unit is compiled with --fmad=false so that every multiply
// and add is rounded separately, as in the reference build.
#include "common.cuh"
#include "llg.cuh"

namespace {

constexpr double kPi = 3.141592653589793;

__device__ double f3(double a, double b, double c, double x, double y, double z)
{
    const double bb = b / 2.0 - y, cc = c / 2.0 - z;
    if (a / 2.0 - x == 0.0) {
        const double xh = x * 1.0001, xl = x * 0.9999;
        const double ah = a / 2.0 - xh, al = a / 2.0 - xl;
        const double fh = bb * cc / (ah * sqrt(ah * ah + bb * bb + cc * cc));
        const double fl = bb * cc / (al * sqrt(al * al + bb * bb + cc * cc));
        return 0.5 * (fh + fl);
    }
    const double aa = a / 2.0 - x;
    return bb * cc / (aa * sqrt(aa * aa + bb * bb + cc * cc));
}

__device__ double g3(double a, double b, double c, double x, double y, double z)
{
    const double aa = a / 2.0 - x, cc = c / 2.0 - z;
    if (b / 2.0 - y == 0.0) {
        const double yh = y * 1.0001, yl = y * 0.9999;
        const double bh = b / 2.0 - yh, bl = b / 2.0 - yl;
        const double gh = aa * cc / (bh * sqrt(aa * aa + bh * bh + cc * cc));
        const double gl = aa * cc / (bl * sqrt(aa * aa + bl * bl + cc * cc));
        return 0.5 * (gh + gl);
    }
    const double bb = b / 2.0 - y;
    return aa * cc / (bb * sqrt(aa * aa + bb * bb + cc * cc));
}

__device__ double h3(double a, double b, double c, double x, double y, double z)
{
    const double aa = a / 2.0 - x, bb = b / 2.0 - y;
    if (c / 2.0 - z == 0.0) {
        const double zh = z * 1.0001, zl = z * 0.9999;
        const double ch = c / 2.0 - zh, cl = c / 2.0 - zl;
        const double hh = aa * bb / (ch * sqrt(aa * aa + bb * bb + ch * ch));
        const double hl = aa * bb / (cl * sqrt(aa * aa + bb * bb + cl * cl));
        return 0.5 * (hl + hh);
    }
    const double cc = c / 2.0 - z;
    return aa * bb / (cc * sqrt(aa * aa + bb * bb + cc * cc));
}

// FF (c-axis), GG (a-axis), HH (b-axis) of the off-diagonal logarithms
template <int AX>
__device__ double FGH(double a, double b, double c, double x, double y, double z)
{
    const double aa = a / 2.0 - x, bb = b / 2.0 - y, cc = c / 2.0 - z;
    const double r = sqrt(aa * aa + bb * bb + cc * cc);
    return (AX == 2 ? cc : (AX == 0 ? aa : bb)) + r;
}

template <int AX>
__device__ double prod_nom(double a, double b, double c, double x, double y, double z)
{
    return FGH<AX>(a, b, c, x, y, z) * FGH<AX>(-a, -b, c, x, y, z) * FGH<AX>(a, -b, -c, x, y, z) *
           FGH<AX>(-a, b, -c, x, y, z);
}
template <int AX>
__device__ double prod_den(double a, double b, double c, double x, double y, double z)
{
    return FGH<AX>(a, -b, c, x, y, z) * FGH<AX>(-a, b, c, x, y, z) * FGH<AX>(a, b, -c, x, y, z) *
           FGH<AX>(-a, -b, -c, x, y, z);
}

template <int AX>
__device__ double offdiag(double a, double b, double c, double x, double y, double z)
{
    const double nom = prod_nom<AX>(a, b, c, x, y, z);
    const double den = prod_den<AX>(a, b, c, x, y, z);
    const double k = 1.0 / (4.0 * kPi);
    double v;
    if (den == 0.0 || nom == 0.0) {
        const double xh = x * 1.0001, yh = y * 1.0001, zh = z * 1.0001;
        const double xl = x * 0.9999, yl = y * 0.9999, zl = z * 0.9999;
        const double nl = prod_nom<AX>(a, b, c, xl, yl, zl), nh = prod_nom<AX>(a, b, c, xh, yh, zh);
        const double dl = prod_den<AX>(a, b, c, xl, yl, zl), dh = prod_den<AX>(a, b, c, xh, yh, zh);
        const double lim = (0.5 * (nl + nh)) / (0.5 * (dl + dh));
        v = -(k * log(lim));
    } else {
        v = -(k * log(nom / den));
    }
    if (fabs((nom - den) / den) < 10.0 * 2.220446049250313e-16) v = 0.0;
    return v;
}

template <typename Fn>
__device__ double diag_sum(Fn F, double a, double b, double c, double x, double y, double z)
{
    const double s = atan(F(a, b, c, x, y, z)) + atan(F(a, b, c, -x, y, z)) + atan(F(a, b, c, x, -y, z)) +
                     atan(F(a, b, c, x, y, -z)) + atan(F(a, b, c, -x, -y, z)) + atan(F(a, b, c, x, -y, -z)) +
                     atan(F(a, b, c, -x, y, -z)) + atan(F(a, b, c, -x, -y, -z));
    return (1.0 / (4.0 * kPi)) * s;
}

struct F3 { __device__ double operator()(double a, double b, double c, double x, double y, double z) const { return f3(a, b, c, x, y, z); } };
struct G3 { __device__ double operator()(double a, double b, double c, double x, double y, double z) const { return g3(a, b, c, x, y, z); } };
struct H3 { __device__ double operator()(double a, double b, double c, double x, double y, double z) const { return h3(a, b, c, x, y, z); } };

__device__ void prism_tensor(double a, double b, double c, double x, double y, double z, double N6[6])
{
    const double n11 = diag_sum(F3{}, a, b, c, x, y, z);
    const double n22 = diag_sum(G3{}, a, b, c, x, y, z);
    const double n33 = diag_sum(H3{}, a, b, c, x, y, z);
    const double n12 = offdiag<2>(a, b, c, x, y, z);   // FF
    const double n23 = offdiag<0>(a, b, c, x, y, z);   // GG
    const double n13 = offdiag<1>(a, b, c, x, y, z);   // HH
    N6[0] = -1.0 * n11; N6[1] = -1.0 * n12; N6[2] = -1.0 * n13;
    N6[3] = -1.0 * n22; N6[4] = -1.0 * n23; N6[5] = -1.0 * n33;
}

// cell-centre coordinate along one axis (setupGrid, :828-857)
__device__ double axis_coord(int i, int nn, double L, double d)
{
    if (nn > 1) return (-(L / 2.0) + (double)i * d) + d / 2.0;
    return 0.0;
}

struct GridDesc { int nx, ny, nz; double L[3], d[3]; };

// One thread per (receiver i, source j); blockIdx.y = receiver - row0.
__global__ void __launch_bounds__(128) assemble_kernel(GridDesc g, int n, int ldk, int row0, float* __restrict__ K)
{
    const int i = row0 + blockIdx.y;
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= ldk) return;
    float* rowbase = K + ((size_t)blockIdx.y * 6) * ldk + j;
    if (j >= n) {
        for (int c = 0; c < 6; ++c) rowbase[(size_t)c * ldk] = 0.0f;
        return;
    }
    const int ix = i % g.nx, iy = (i / g.nx) % g.ny, iz = i / (g.nx * g.ny);
    const int jx = j % g.nx, jy = (j / g.nx) % g.ny, jz = j / (g.nx * g.ny);
    const double x = axis_coord(ix, g.nx, g.L[0], g.d[0]) - axis_coord(jx, g.nx, g.L[0], g.d[0]);
    const double y = axis_coord(iy, g.ny, g.L[1], g.d[1]) - axis_coord(jy, g.ny, g.L[1], g.d[1]);
    const double z = axis_coord(iz, g.nz, g.L[2], g.d[2]) - axis_coord(jz, g.nz, g.L[2], g.d[2]);
    double N6[6];
    prism_tensor(g.d[0], g.d[1], g.d[2], x, y, z, N6);
#pragma unroll
    for (int c = 0; c < 6; ++c) rowbase[(size_t)c * ldk] = (float)N6[c];
}

// Reference column-major blocks -> cell-row layout (and back).
__global__ void colmajor_to_rows(const float* __restrict__ blk, int c, int n, int ldk, float* __restrict__ K)
{
    // blk(i, j) at j*n + i ; write K[(i*6+c)*ldk + j]; tile transpose through shared memory
    __shared__ float tile[32][33];
    const int i0 = blockIdx.x * 32, j0 = blockIdx.y * 32;
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int j = j0 + r, i = i0 + threadIdx.x;
        tile[r][threadIdx.x] = (i < n && j < n) ? blk[(size_t)j * n + i] : 0.0f;
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int i = i0 + r, j = j0 + threadIdx.x;
        if (i < n && j < ldk) K[((size_t)i * 6 + c) * ldk + j] = (j < n) ? tile[threadIdx.x][r] : 0.0f;
    }
}

__global__ void rows_to_colmajor(const float* __restrict__ K, int c, int n, int ldk, float* __restrict__ blk)
{
    __shared__ float tile[32][33];
    const int i0 = blockIdx.x * 32, j0 = blockIdx.y * 32;
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int i = i0 + r, j = j0 + threadIdx.x;
        tile[r][threadIdx.x] = (i < n && j < n) ? K[((size_t)i * 6 + c) * ldk + j] : 0.0f;
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int j = j0 + r, i = i0 + threadIdx.x;
        if (i < n && j < n) blk[(size_t)j * n + i] = tile[threadIdx.x][r];
    }
}

}  // namespace

// Host launchers (called from capi.cu)
cudaError_t launch_assemble(int nx, int ny, int nz, const double L[3], const double d[3], int n, int ldk, int row0,
                            int nrows, float* K, cudaStream_t s)
{
    if (row0 < 0 || nrows < 1 || row0 + nrows > n) return cudaErrorInvalidValue;
    GridDesc g;
    g.nx = nx; g.ny = ny; g.nz = nz;
    for (int a = 0; a < 3; ++a) { g.L[a] = L[a]; g.d[a] = d[a]; }
    dim3 block(128);
    dim3 grid((ldk + 127) / 128, nrows);
    assemble_kernel<<<grid, block, 0, s>>>(g, n, ldk, row0, K);
    return cudaGetLastError();
}

cudaError_t launch_colmajor_to_rows(const float* blk, int c, int n, int ldk, float* K, cudaStream_t s)
{
    dim3 block(32, 8);
    dim3 grid((n + 31) / 32, (ldk + 31) / 32);
    colmajor_to_rows<<<grid, block, 0, s>>>(blk, c, n, ldk, K);
    return cudaGetLastError();
}

cudaError_t launch_rows_to_colmajor(const float* K, int c, int n, int ldk, float* blk, cudaStream_t s)
{
    dim3 block(32, 8);
    dim3 grid((n + 31) / 32, (n + 31) / 32);
    rows_to_colmajor<<<grid, block, 0, s>>>(K, c, n, ldk, blk);
    return cudaGetLastError();
}
