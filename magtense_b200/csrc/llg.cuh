// Problem description on the device, the streaming FP32 demag product and the
// per-cell Landau-Lifshitz right-hand side.
//
// Demag tensor layout in HBM ("cell rows"): for receiver cell i the six
// components xx,xy,xz,yy,yz,zz are six consecutive rows of ldk floats,
//   K[((size_t)i*6 + c)*ldk + j]  (source j, zero for n <= j < ldk).
// A CTA that owns a range of receiver cells therefore streams one contiguous
// 24*ldk-byte record per cell.  ldk = n rounded up to a multiple of 4 so that
// every row starts 16-byte aligned for 128-bit loads.
#pragma once
#include "common.cuh"

struct DevProb {
    int n, nx, ny, nz, ldk;
    const float* K;          // tensor rows of cells [krow0, ...): K[((i - krow0)*6 + c)*ldk + j]
    int krow0;               // first cell whose rows K holds (0 unless the instance is row-sharded)
    double lapc[3];          // 1/(d*d) per axis
    double diag_b[3];        // boundary-row diagonal -1/(d*d), 0 when the axis has one cell
    double diag_i[3];        // interior-row diagonal -2/(d*d), 0 when the axis has one cell
    const double* Jfact;     // A0/(mu0 Ms_i)
    const double* Kfact;     // K0_i/(mu0 Ms_i)
    const float* Mfact;      // Ms_i in FP32
    const double* A6;        // u u^T: [c*n + i], c = xx,xy,xz,yy,yz,zz
    int solver;              // 1 explicit, 2 dynamic
    int hext_row;
    int nt_hext, nt_alpha;
    const double* hext;      // [k*4 + {t,hx,hy,hz}]
    const double* alpha_tab; // [k*2 + {t,alpha}]
    double gamma, alpha0;
    // thresholded-sparse demag (nullptr: the dense tensor): receiver row r = 3 i + a holds
    // the kept entries K_ab(i, j) of blocks b = x, y, z in that order, column b*ldk + j
    const int* sp_rowptr;    // [3n + 1]
    const int* sp_col;
    const float* sp_val;
    // fraction of the dense tensor's lines loaded with the L2 evict_last policy (0: plain
    // streaming loads): a tensor about as large as one die's half of L2 is read in the same
    // order every evaluation, which evicts each line just before its next use
    float l2_keep;
};

// locate + interp1_MagTense (util.f90:39-85): 0 outside the table.
MT_DEV double interp1_dev(const double* tab, int stride, int col, int nt, double xv)
{
    if (nt < 2) return 0.0;
    int jl = 0, ju = nt + 1;
    const bool asc = __ldg(&tab[(nt - 1) * stride]) >= __ldg(&tab[0]);
    while (ju - jl > 1) {
        int jm = (ju + jl) >> 1;
        bool ge = xv >= __ldg(&tab[(jm - 1) * stride]);
        if (asc == ge) jl = jm; else ju = jm;
    }
    int j;
    if (xv == __ldg(&tab[0])) j = 1;
    else if (xv == __ldg(&tab[(nt - 1) * stride])) j = nt - 1;
    else j = jl;
    if (j == 0 || j >= nt) return 0.0;
    double x0 = __ldg(&tab[(j - 1) * stride]), x1 = __ldg(&tab[j * stride]);
    double y0 = __ldg(&tab[(j - 1) * stride + col]), y1 = __ldg(&tab[j * stride + col]);
    double xl = __ddiv_rn(xsub(xv, x0), xsub(x1, x0));
    return xadd(xmul(xsub(1.0, xl), y0), xmul(xl, y1));
}

struct TimeScalars { double hx, hy, hz, alpha; };

MT_DEV TimeScalars time_scalars(const DevProb& P, double t)
{
    TimeScalars s;
    if (P.solver == 1) {
        s.hx = __ldg(&P.hext[P.hext_row * 4 + 1]);
        s.hy = __ldg(&P.hext[P.hext_row * 4 + 2]);
        s.hz = __ldg(&P.hext[P.hext_row * 4 + 3]);
    } else if (P.solver == 2) {
        s.hx = interp1_dev(P.hext, 4, 1, P.nt_hext, t);
        s.hy = interp1_dev(P.hext, 4, 2, P.nt_hext, t);
        s.hz = interp1_dev(P.hext, 4, 3, P.nt_hext, t);
    } else {
        s.hx = s.hy = s.hz = 0.0;
    }
    s.alpha = (P.alpha0 == 0.0) ? interp1_dev(P.alpha_tab, 2, 1, P.nt_alpha, t) : P.alpha0;
    return s;
}

// Neumann Laplacian of one component at cell i (ComputeExchangeTerm3D_Uniform,
// LandauLifshitzEquationSolver.f90:1194-1522): merged diagonal plus the
// neighbour terms in increasing column order.  v is read through L2 because
// other CTAs wrote it during the same launch.  lap_load issues the loads (only
// of neighbours that exist, all in flight together: o = z0 y0 x0 c x1 y1 z1),
// lap_from sums them.
MT_DEV void lap_load(const DevProb& P, const double* v, int i, double o[7])
{
    const int nx = P.nx, ny = P.ny, nz = P.nz;
    const int ix = i % nx, iy = (i / nx) % ny, iz = i / (nx * ny);
    o[0] = (nz > 1 && iz > 0) ? ldcg(&v[i - nx * ny]) : 0.0;
    o[1] = (ny > 1 && iy > 0) ? ldcg(&v[i - nx]) : 0.0;
    o[2] = (nx > 1 && ix > 0) ? ldcg(&v[i - 1]) : 0.0;
    o[3] = ldcg(&v[i]);
    o[4] = (nx > 1 && ix < nx - 1) ? ldcg(&v[i + 1]) : 0.0;
    o[5] = (ny > 1 && iy < ny - 1) ? ldcg(&v[i + nx]) : 0.0;
    o[6] = (nz > 1 && iz < nz - 1) ? ldcg(&v[i + nx * ny]) : 0.0;
}

MT_DEV double lap_from(const DevProb& P, const double o[7], int i)
{
    const int nx = P.nx, ny = P.ny, nz = P.nz;
    const int ix = i % nx, iy = (i / nx) % ny, iz = i / (nx * ny);
    double dgx = (nx > 1) ? ((ix == 0 || ix == nx - 1) ? P.diag_b[0] : P.diag_i[0]) : 0.0;
    double dgy = (ny > 1) ? ((iy == 0 || iy == ny - 1) ? P.diag_b[1] : P.diag_i[1]) : 0.0;
    double dgz = (nz > 1) ? ((iz == 0 || iz == nz - 1) ? P.diag_b[2] : P.diag_i[2]) : 0.0;
    double diag = xadd(dgx, dgy);
    if (nz > 1) diag = xadd(diag, dgz);
    const bool hz0 = nz > 1 && iz > 0, hy0 = ny > 1 && iy > 0, hx0 = nx > 1 && ix > 0;
    const bool hx1 = nx > 1 && ix < nx - 1, hy1 = ny > 1 && iy < ny - 1, hz1 = nz > 1 && iz < nz - 1;
    double s = 0.0;
    bool first = true;
#define MT_ACC(term)                              \
    do {                                          \
        double _t = (term);                       \
        if (first) { s = _t; first = false; }     \
        else s = xadd(s, _t);                     \
    } while (0)
    if (hz0) MT_ACC(xmul(P.lapc[2], o[0]));
    if (hy0) MT_ACC(xmul(P.lapc[1], o[1]));
    if (hx0) MT_ACC(xmul(P.lapc[0], o[2]));
    MT_ACC(xmul(diag, o[3]));
    if (hx1) MT_ACC(xmul(P.lapc[0], o[4]));
    if (hy1) MT_ACC(xmul(P.lapc[1], o[5]));
    if (hz1) MT_ACC(xmul(P.lapc[2], o[6]));
#undef MT_ACC
    return s;
}

MT_DEV double lap_cell_dev(const DevProb& P, const double* v, int i)
{
    double o[7];
    lap_load(P, v, i, o);
    return lap_from(P, o, i);
}

// anisotropy field of one cell: -2 K0/(mu0 Ms) (u u^T) m.  aniso_load reads the cell's
// constants (K0/(mu0 Ms), then u u^T as xx xy xz yy yz zz), aniso_from applies them.
MT_DEV void aniso_load(const DevProb& P, int i, double c[7])
{
    const int n = P.n;
    c[0] = __ldg(&P.Kfact[i]);
#pragma unroll
    for (int k = 0; k < 6; ++k) c[1 + k] = __ldg(&P.A6[k * (size_t)n + i]);
}

MT_DEV void aniso_from(const double c[7], double mx, double my, double mz, double hk[3])
{
    const double k2 = xmul(-2.0, c[0]);
    const double axx = c[1], axy = c[2], axz = c[3], ayy = c[4], ayz = c[5], azz = c[6];
    hk[0] = xmul(k2, xadd(xadd(xmul(axx, mx), xmul(axy, my)), xmul(axz, mz)));
    hk[1] = xmul(k2, xadd(xadd(xmul(axy, mx), xmul(ayy, my)), xmul(ayz, mz)));
    hk[2] = xmul(k2, xadd(xadd(xmul(axz, mx), xmul(ayz, my)), xmul(azz, mz)));
}

MT_DEV void aniso_field(const DevProb& P, int i, double mx, double my, double mz, double hk[3])
{
    double c[7];
    aniso_load(P, i, c);
    aniso_from(c, mx, my, mz, hk);
}

// dm/dt from m and the effective field he (dmdt_fct :251-271)
MT_DEV void ll_from_heff(const DevProb& P, double mx, double my, double mz, const double he[3], double alpha,
                         double out[3])
{
    const double cx = xmul(-1.0, xsub(xmul(my, he[2]), xmul(mz, he[1])));
    const double cy = xmul(-1.0, xsub(xmul(mz, he[0]), xmul(mx, he[2])));
    const double cz = xmul(-1.0, xsub(xmul(mx, he[1]), xmul(my, he[0])));
    const double h2x = xsub(xmul(my, cz), xmul(mz, cy));
    const double h2y = xsub(xmul(mz, cx), xmul(mx, cz));
    const double h2z = xsub(xmul(mx, cy), xmul(my, cx));
    const double g = -P.gamma;
    out[0] = xsub(xmul(g, cx), xmul(alpha, h2x));
    out[1] = xsub(xmul(g, cy), xmul(alpha, h2y));
    out[2] = xsub(xmul(g, cz), xmul(alpha, h2z));
}

// The four internal field terms of one cell (dmdt_fct :239-248).
// S = sum_j K m (FP32, this cell's three rows).
struct CellFields { double hj[3], hh[3], hk[3], hm[3]; };

MT_DEV CellFields cell_fields_local(const DevProb& P, const double* m, int i, const TimeScalars& ts)
{
    const int n = P.n;
    CellFields F;
    const double mx = ldcg(&m[i]), my = ldcg(&m[n + i]), mz = ldcg(&m[2 * n + i]);
    const double jf = __ldg(&P.Jfact[i]);
    for (int a = 0; a < 3; ++a) F.hj[a] = xmul(xmul(-2.0, lap_cell_dev(P, m + (size_t)a * n, i)), jf);
    F.hh[0] = -ts.hx; F.hh[1] = -ts.hy; F.hh[2] = -ts.hz;
    aniso_field(P, i, mx, my, mz, F.hk);
    return F;
}

MT_DEV CellFields cell_fields(const DevProb& P, const double* m, int i, const float S[3],
                              const TimeScalars& ts)
{
    CellFields F = cell_fields_local(P, m, i, ts);
    const float ms = __ldg(&P.Mfact[i]);
    for (int a = 0; a < 3; ++a) F.hm[a] = (double)__fmul_rn(-S[a], ms);
    return F;
}

// dm/dt for one cell (dmdt_fct :251-271).
MT_DEV void cell_rhs_from(const DevProb& P, const double* m, int i, const CellFields& F, const TimeScalars& ts,
                          double out[3])
{
    const int n = P.n;
    const double mx = ldcg(&m[i]), my = ldcg(&m[n + i]), mz = ldcg(&m[2 * n + i]);
    double he[3];
    for (int a = 0; a < 3; ++a) he[a] = xadd(xadd(xadd(F.hh[a], F.hj[a]), F.hm[a]), F.hk[a]);
    ll_from_heff(P, mx, my, mz, he, ts.alpha, out);
}

MT_DEV void cell_rhs(const DevProb& P, const double* m, int i, const float S[3], const TimeScalars& ts,
                     double out[3])
{
    cell_rhs_from(P, m, i, cell_fields(P, m, i, S, ts), ts, out);
}

// the same with the demagnetisation field given in FP64 (exact fixed-point product)
MT_DEV void cell_rhs_h(const DevProb& P, const double* m, int i, const double hm[3], const TimeScalars& ts,
                       double out[3])
{
    CellFields F = cell_fields_local(P, m, i, ts);
    F.hm[0] = hm[0]; F.hm[1] = hm[1]; F.hm[2] = hm[2];
    cell_rhs_from(P, m, i, F, ts, out);
}

// ------------------------------------------------------------------------
// Streaming FP32 demag product for the receiver cells [c0, c0+nc) of this CTA.
// S_out[cell*3 + a] = sum_j sum_b K_ab(cell, j) m32_b(j), a,b in {x,y,z}.
// m32: global [3][ldk] FP32 (written by other CTAs in this launch -> L2 loads).
// Shared memory: sm_m (3*JC floats), sm_part (3*max_units floats).
// Each warp takes (cell, segment) units; a lane streams float4 columns of the
// cell's six rows with non-coherent 128-bit loads and FMAs against the m slice
// in shared memory; partial sums are combined in a fixed order.
// ------------------------------------------------------------------------
constexpr int kDemagJC = 8192;       // source chunk held in shared memory (96 KB)
constexpr int kDemagMaxUnits = 2048; // (cell, segment) units per chunk

MT_DEV float4 ldg_keep(const float* p, uint64_t pol)
{
    float4 v;
    asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.f32 {%0,%1,%2,%3}, [%4], %5;"
                 : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
                 : "l"(p), "l"(pol));
    return v;
}

template <bool Keep>
MT_DEV float4 ldg_k(const float* p, uint64_t pol);

MT_DEV float4 ldg_stream(const float* p)
{
    float4 v;
    asm volatile("ld.global.nc.L1::no_allocate.v4.f32 {%0,%1,%2,%3}, [%4];"
                 : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
                 : "l"(p));
    return v;
}

template <>
MT_DEV float4 ldg_k<false>(const float* p, uint64_t) { return ldg_stream(p); }
template <>
MT_DEV float4 ldg_k<true>(const float* p, uint64_t pol) { return ldg_keep(p, pol); }

// Sparse demag product for the receiver cells [c0, c0+nc): one warp per receiver row
// (cell, component) sums its kept entries against m (staged in shared memory when
// the whole [3][ldk] vector fits the chunk, read through L2 otherwise), lanes
// strided over the row, then a fixed shuffle tree.
MT_DEV void demag_cta_sparse(const DevProb& P, const float* __restrict__ m32, int c0, int nc, float* sm_m,
                             float* S_out)
{
    const int ldk = P.ldk;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const bool staged = ldk <= kDemagJC;
    __syncthreads();
    if (staged) {
        const int l4 = (3 * ldk) >> 2;
        float4* d4 = reinterpret_cast<float4*>(sm_m);
        const float4* s4 = reinterpret_cast<const float4*>(m32);
        for (int e = threadIdx.x; e < l4; e += blockDim.x) d4[e] = __ldcg(s4 + e);
    }
    __syncthreads();
    for (int r = warp; r < 3 * nc; r += nwarps) {
        const int row = 3 * c0 + r;
        const int e0 = __ldg(&P.sp_rowptr[row]), e1 = __ldg(&P.sp_rowptr[row + 1]);
        float s = 0.f;
        for (int e = e0 + lane; e < e1; e += 32) {
            const int col = __ldg(&P.sp_col[e]);
            const float mv = staged ? sm_m[col] : __ldcg(&m32[col]);
            s = __fmaf_rn(__ldg(&P.sp_val[e]), mv, s);
        }
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) S_out[r] = s;   // r = cell * 3 + a
    }
    __syncthreads();
}

// the (cell, segment) units of one chunk: each warp streams a cell's six rows over a
// segment against the m slice in shared memory
template <bool Keep>
MT_DEV void demag_units(const DevProb& P, int c0, int ch0, int len, int nseg, int seglen, int units,
                        const float4* mx4, const float4* my4, const float4* mz4, float* sm_part, uint64_t pol)
{
    const int ldk = P.ldk;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    for (int u = warp; u < units; u += nwarps) {
        const int cell = u / nseg, seg = u - cell * nseg;
        const int js4 = (seg * seglen) >> 2;
        const int je4 = min(seg * seglen + seglen, len) >> 2;
        const float* row = P.K + ((size_t)(c0 + cell - P.krow0) * 6) * ldk + ch0;
        float sx = 0.f, sy = 0.f, sz = 0.f;
#pragma unroll 2
        for (int j4 = js4 + lane; j4 < je4; j4 += 32) {
            const float4 kxx = ldg_k<Keep>(row + 0 * (size_t)ldk + 4 * j4, pol);
            const float4 kxy = ldg_k<Keep>(row + 1 * (size_t)ldk + 4 * j4, pol);
            const float4 kxz = ldg_k<Keep>(row + 2 * (size_t)ldk + 4 * j4, pol);
            const float4 kyy = ldg_k<Keep>(row + 3 * (size_t)ldk + 4 * j4, pol);
            const float4 kyz = ldg_k<Keep>(row + 4 * (size_t)ldk + 4 * j4, pol);
            const float4 kzz = ldg_k<Keep>(row + 5 * (size_t)ldk + 4 * j4, pol);
            const float4 a = mx4[j4], b = my4[j4], c = mz4[j4];
            sx += kxx.x * a.x + kxy.x * b.x + kxz.x * c.x;
            sy += kxy.x * a.x + kyy.x * b.x + kyz.x * c.x;
            sz += kxz.x * a.x + kyz.x * b.x + kzz.x * c.x;
            sx += kxx.y * a.y + kxy.y * b.y + kxz.y * c.y;
            sy += kxy.y * a.y + kyy.y * b.y + kyz.y * c.y;
            sz += kxz.y * a.y + kyz.y * b.y + kzz.y * c.y;
            sx += kxx.z * a.z + kxy.z * b.z + kxz.z * c.z;
            sy += kxy.z * a.z + kyy.z * b.z + kyz.z * c.z;
            sz += kxz.z * a.z + kyz.z * b.z + kzz.z * c.z;
            sx += kxx.w * a.w + kxy.w * b.w + kxz.w * c.w;
            sy += kxy.w * a.w + kyy.w * b.w + kyz.w * c.w;
            sz += kxz.w * a.w + kyz.w * b.w + kzz.w * c.w;
        }
        for (int o = 16; o > 0; o >>= 1) {
            sx += __shfl_xor_sync(0xffffffffu, sx, o);
            sy += __shfl_xor_sync(0xffffffffu, sy, o);
            sz += __shfl_xor_sync(0xffffffffu, sz, o);
        }
        if (lane == 0) {
            sm_part[u * 3 + 0] = sx;
            sm_part[u * 3 + 1] = sy;
            sm_part[u * 3 + 2] = sz;
        }
    }
}

// units_per_warp sets how many (cell, segment) units a chunk aims for per warp: more,
// shorter segments cost more rounds of the unit loop but shorten the FP32 running sums
// of every lane.  The integrators take 5 (the noise of the product sets RKSUITE's
// step size), the stand-alone field kernel 2.
MT_DEV void demag_cta(const DevProb& P, const float* __restrict__ m32, int c0, int nc, float* sm_m,
                      float* sm_part, float* S_out, int units_per_warp)
{
    if (P.sp_rowptr) { demag_cta_sparse(P, m32, c0, nc, sm_m, S_out); return; }
    const int ldk = P.ldk;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const int JC = ldk < kDemagJC ? ldk : kDemagJC;
    for (int e = threadIdx.x; e < 3 * nc; e += blockDim.x) S_out[e] = 0.0f;
    for (int ch0 = 0; ch0 < ldk; ch0 += JC) {
        const int len = min(JC, ldk - ch0);          // multiple of 4
        // segments: enough units to keep all warps busy, each a multiple of 128 floats
        int nseg = (units_per_warp * nwarps + nc - 1) / max(nc, 1);
        if (nseg < 1) nseg = 1;
        int seglen = (len + nseg - 1) / nseg;
        seglen = (seglen + 127) & ~127;
        nseg = (len + seglen - 1) / seglen;
        while (nc * nseg > kDemagMaxUnits && nseg > 1) {
            seglen *= 2;
            nseg = (len + seglen - 1) / seglen;
        }
        __syncthreads();
        {   // stage the m slice
            const int l4 = len >> 2;
            float4* d4 = reinterpret_cast<float4*>(sm_m);
            for (int e = threadIdx.x; e < 3 * l4; e += blockDim.x) {
                const int a = e / l4, j4 = e - a * l4;
                const float4* src = reinterpret_cast<const float4*>(m32 + (size_t)a * ldk + ch0) + j4;
                d4[a * (JC >> 2) + j4] = __ldcg(src);
            }
        }
        __syncthreads();
        const int units = nc * nseg;
        const float4* mx4 = reinterpret_cast<const float4*>(sm_m);
        const float4* my4 = mx4 + (JC >> 2);
        const float4* mz4 = my4 + (JC >> 2);
        if (P.l2_keep > 0.f) {
            uint64_t pol;
            asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, %1;" : "=l"(pol) : "f"(P.l2_keep));
            demag_units<true>(P, c0, ch0, len, nseg, seglen, units, mx4, my4, mz4, sm_part, pol);
        } else {
            demag_units<false>(P, c0, ch0, len, nseg, seglen, units, mx4, my4, mz4, sm_part, 0);
        }
        __syncthreads();
        for (int e = threadIdx.x; e < 3 * nc; e += blockDim.x) {
            const int cell = e / 3, a = e - cell * 3;
            float s = 0.f;
            for (int sg = 0; sg < nseg; ++sg) s += sm_part[(cell * nseg + sg) * 3 + a];
            S_out[e] += s;
        }
    }
    __syncthreads();
}

// shared-memory bytes needed by demag_cta for a given ldk and cells per CTA
static inline size_t demag_smem_bytes(int ldk, int nc)
{
    const int JC = ldk < kDemagJC ? ldk : kDemagJC;
    return sizeof(float) * (3 * (size_t)JC + 3 * (size_t)kDemagMaxUnits + 3 * (size_t)nc);
}
