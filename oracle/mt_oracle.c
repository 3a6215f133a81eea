/*
 * mt_oracle.c -- CPU oracle for the MagTense micromagnetic hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product (magtense_b200/) links,
 * loads or calls this file; it is used by tests/, by __graft_entry__.smoke()
 * and by the cpu_baseline leg of bench.py, and only as the checker.
 *
 * It restates, in plain C with IEEE double/single arithmetic and no FMA
 * contraction (-ffp-contract=off), the reference Fortran of the path
 * (paths relative to the MagTense project root):
 *
 *   prism tensor   getN_prism_3D      source/TileDemagTensor/TileDemagTensor/TileNComponents.f90:629-724
 *                  f_3D g_3D h_3D FF_3D GG_3D HH_3D getF_limit
 *                                     source/TileDemagTensor/TileDemagTensor/TileRectangularPrismTensor.f90:7-149
 *   grid           setupGrid          source/MagTenseMicroMag/LandauLifshitzEquationSolver.f90:815-872
 *   demag tensor   ComputeDemagfieldTensor, uniform branch            same file :883-986
 *   exchange       ComputeExchangeTerm3D_Uniform :1194-1522, updateExchangeTerms :440-474
 *   anisotropy     ComputeAnisotropyTerm3D_General :1566-1587, updateAnisotropy :523-548
 *   Zeeman         updateExternalField :485-514; interp1_MagTense/locate
 *                                     source/NumericalIntegration/NumericalIntegration/util.f90:39-85
 *   demag field    updateDemagfield dense CPU branch :706-767
 *   RHS            dmdt_fct :220-273, alpha() :281-294, initializeSolution :359-430
 *   integrator     RKSUITE-90 (Brankin, Gladwell, Shampine 1994) method 'M', task 'R',
 *                  as vendored in source/NumericalIntegration/NumericalIntegration/RKSuitef90.f90:
 *                  method_const case 2 :223-412,:568-591; setup_r1 :596-856;
 *                  range_integrate_r1 :942-1183; step_integrate_r1 :1185-1587;
 *                  step_r1 :1726-1978; stiff_r1 :1981-2367; interpolate_r1 :2655-2997
 *   output driver  MagTense_ODE_RKSuite  source/NumericalIntegration/NumericalIntegration/ODE_Solvers.f90:124-237
 *                  simple_unique/simple_sort SpecialFunctions.f90:13-65
 *
 * Three precisions: mode 0 ("ref") keeps the reference's FP32 demag tensor and
 * FP32 demag product; mode 1 ("fp64") keeps the tensor and the product in
 * FP64 and serves the error statements against FP64; mode 2 ("int8") is the
 * exact fixed-point product of the GPU's int8 backend, restated from its
 * definition (rows of the FP32 tensor as 32-bit fixed point in four int8
 * limbs, m as rint(m 2^30) in four limbs, all sixteen limb products summed
 * exactly, one rounding to double), so the GPU must reproduce it bit for bit.
 *
 * Summation order of the FP32 demag product follows the reference BLAS SGEMV
 * column sweep (y(i) += (-x(j))*A(i,j), j = 1..n, one block after the other);
 * MKL's internal order is not pinned by anything in the reference.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <complex.h>
#include <float.h>
#include <omp.h>

#define OR_PI 3.141592653589793
/* mu0 = 4*pi*1e-7 evaluated left to right, TileTensorHelperFunctions.f90:5 */
static double or_mu0(void) { double v = 4.0 * OR_PI; return v * 1e-7; }

/* ------------------------------------------------------------------ */
/* prism tensor                                                       */
/* ------------------------------------------------------------------ */
static double f3(double a, double b, double c, double x, double y, double z)
{
    double bb = b / 2.0 - y, cc = c / 2.0 - z;
    if (a / 2.0 - x == 0.0) {
        double xh = x * 1.0001, xl = x * 0.9999;
        double ah = a / 2.0 - xh, al = a / 2.0 - xl;
        double fh = bb * cc / (ah * sqrt(ah * ah + bb * bb + cc * cc));
        double fl = bb * cc / (al * sqrt(al * al + bb * bb + cc * cc));
        return 0.5 * (fh + fl);
    }
    double aa = a / 2.0 - x;
    return bb * cc / (aa * sqrt(aa * aa + bb * bb + cc * cc));
}

static double g3(double a, double b, double c, double x, double y, double z)
{
    double aa = a / 2.0 - x, cc = c / 2.0 - z;
    if (b / 2.0 - y == 0.0) {
        double yh = y * 1.0001, yl = y * 0.9999;
        double bh = b / 2.0 - yh, bl = b / 2.0 - yl;
        double gh = aa * cc / (bh * sqrt(aa * aa + bh * bh + cc * cc));
        double gl = aa * cc / (bl * sqrt(aa * aa + bl * bl + cc * cc));
        return 0.5 * (gh + gl);
    }
    double bb = b / 2.0 - y;
    return aa * cc / (bb * sqrt(aa * aa + bb * bb + cc * cc));
}

static double h3(double a, double b, double c, double x, double y, double z)
{
    double aa = a / 2.0 - x, bb = b / 2.0 - y;
    if (c / 2.0 - z == 0.0) {
        double zh = z * 1.0001, zl = z * 0.9999;
        double ch = c / 2.0 - zh, cl = c / 2.0 - zl;
        double hh = aa * bb / (ch * sqrt(aa * aa + bb * bb + ch * ch));
        double hl = aa * bb / (cl * sqrt(aa * aa + bb * bb + cl * cl));
        return 0.5 * (hl + hh);
    }
    double cc = c / 2.0 - z;
    return aa * bb / (cc * sqrt(aa * aa + bb * bb + cc * cc));
}

static double FF3(double a, double b, double c, double x, double y, double z)
{
    double aa = a / 2.0 - x, bb = b / 2.0 - y, cc = c / 2.0 - z;
    return cc + sqrt(aa * aa + bb * bb + cc * cc);
}
static double GG3(double a, double b, double c, double x, double y, double z)
{
    double aa = a / 2.0 - x, bb = b / 2.0 - y, cc = c / 2.0 - z;
    return aa + sqrt(aa * aa + bb * bb + cc * cc);
}
static double HH3(double a, double b, double c, double x, double y, double z)
{
    double aa = a / 2.0 - x, bb = b / 2.0 - y, cc = c / 2.0 - z;
    return bb + sqrt(aa * aa + bb * bb + cc * cc);
}

typedef double (*or_fun6)(double, double, double, double, double, double);

static double prod_nom(or_fun6 F, double a, double b, double c, double x, double y, double z)
{
    return F(a, b, c, x, y, z) * F(-a, -b, c, x, y, z) * F(a, -b, -c, x, y, z) * F(-a, b, -c, x, y, z);
}
static double prod_den(or_fun6 F, double a, double b, double c, double x, double y, double z)
{
    return F(a, -b, c, x, y, z) * F(-a, b, c, x, y, z) * F(a, b, -c, x, y, z) * F(-a, -b, -c, x, y, z);
}

/* getF_limit: average of the ratio's numerator/denominator at +-0.01 % offsets */
static double f_limit(or_fun6 F, double a, double b, double c, double x, double y, double z)
{
    double xh = x * 1.0001, yh = y * 1.0001, zh = z * 1.0001;
    double xl = x * 0.9999, yl = y * 0.9999, zl = z * 0.9999;
    double nom_l = prod_nom(F, a, b, c, xl, yl, zl);
    double nom_h = prod_nom(F, a, b, c, xh, yh, zh);
    double den_l = prod_den(F, a, b, c, xl, yl, zl);
    double den_h = prod_den(F, a, b, c, xh, yh, zh);
    double nom = 0.5 * (nom_l + nom_h);
    double den = 0.5 * (den_l + den_h);
    return nom / den;
}

static double offdiag(or_fun6 F, double a, double b, double c, double x, double y, double z)
{
    double nom = prod_nom(F, a, b, c, x, y, z);
    double den = prod_den(F, a, b, c, x, y, z);
    double v;
    double k = 1.0 / (4.0 * OR_PI);
    if (den == 0.0 || nom == 0.0)
        v = -(k * log(f_limit(F, a, b, c, x, y, z)));
    else
        v = -(k * log(nom / den));
    if (fabs((nom - den) / den) < 10.0 * DBL_EPSILON) v = 0.0;
    return v;
}

static double diag_sum(or_fun6 F, double a, double b, double c, double x, double y, double z)
{
    double s = atan(F(a, b, c, x, y, z)) + atan(F(a, b, c, -x, y, z)) + atan(F(a, b, c, x, -y, z))
             + atan(F(a, b, c, x, y, -z)) + atan(F(a, b, c, -x, -y, z)) + atan(F(a, b, c, x, -y, -z))
             + atan(F(a, b, c, -x, y, -z)) + atan(F(a, b, c, -x, -y, -z));
    return (1.0 / (4.0 * OR_PI)) * s;
}

/* Demag tensor of a prism with side lengths (a,b,c) centred at the origin, at
 * offset (x,y,z).  Output order xx, xy, xz, yy, yz, zz, with the reference's
 * final sign flip (self term of a cube = -1/3 on the diagonal). */
void or_prism_tensor(double a, double b, double c, double x, double y, double z, double* N6)
{
    double n11 = diag_sum(f3, a, b, c, x, y, z);
    double n22 = diag_sum(g3, a, b, c, x, y, z);
    double n33 = diag_sum(h3, a, b, c, x, y, z);
    double n12 = offdiag(FF3, a, b, c, x, y, z);
    double n23 = offdiag(GG3, a, b, c, x, y, z);
    double n13 = offdiag(HH3, a, b, c, x, y, z);
    N6[0] = -1.0 * n11; N6[1] = -1.0 * n12; N6[2] = -1.0 * n13;
    N6[3] = -1.0 * n22; N6[4] = -1.0 * n23; N6[5] = -1.0 * n33;
}

/* ------------------------------------------------------------------ */
/* grid                                                               */
/* ------------------------------------------------------------------ */
static void axis_setup(int nn, double L, double* d, double* coord)
{
    if (nn > 1) {
        *d = L / nn;
        for (int i = 0; i < nn; ++i) coord[i] = (-(L / 2.0) + (double)i * (*d)) + (*d) / 2.0;
    } else {
        *d = L;
        coord[0] = 0.0;
    }
}

/* cell centres, x fastest (ind = i + j*nx + k*nx*ny), pts[ind*3 + c]; d[3] cell sizes */
void or_grid(int nx, int ny, int nz, double Lx, double Ly, double Lz, double* pts, double* d)
{
    double* xs = (double*)malloc(sizeof(double) * (nx + ny + nz));
    double* ys = xs + nx;
    double* zs = ys + ny;
    axis_setup(nx, Lx, &d[0], xs);
    axis_setup(ny, Ly, &d[1], ys);
    axis_setup(nz, Lz, &d[2], zs);
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                long ind = i + (long)j * nx + (long)k * nx * ny;
                pts[ind * 3 + 0] = xs[i];
                pts[ind * 3 + 1] = ys[j];
                pts[ind * 3 + 2] = zs[k];
            }
    free(xs);
}

/* Dense demag tensor rows for the receivers in rows[0..nrows) (all receivers if
 * rows == NULL).  Layout: K[(c*nrows + r)*n + j] for component c (xx,xy,xz,yy,yz,zz),
 * receiver row r, source j.  Either K32 (rounded to FP32, the reference's
 * sngl()) or K64 (unrounded) may be NULL. */
void or_assemble(int nx, int ny, int nz, double Lx, double Ly, double Lz,
                 const int* rows, int nrows, float* K32, double* K64)
{
    int n = nx * ny * nz;
    double d[3];
    double* pts = (double*)malloc(sizeof(double) * 3 * (size_t)n);
    or_grid(nx, ny, nz, Lx, Ly, Lz, pts, d);
    if (rows == NULL) nrows = n;
#pragma omp parallel for schedule(dynamic, 4)
    for (int r = 0; r < nrows; ++r) {
        int i = rows ? rows[r] : r;
        double N6[6];
        for (int j = 0; j < n; ++j) {
            double x = pts[i * 3 + 0] - pts[j * 3 + 0];
            double y = pts[i * 3 + 1] - pts[j * 3 + 1];
            double z = pts[i * 3 + 2] - pts[j * 3 + 2];
            or_prism_tensor(d[0], d[1], d[2], x, y, z, N6);
            for (int c = 0; c < 6; ++c) {
                size_t idx = ((size_t)c * nrows + r) * (size_t)n + j;
                if (K32) K32[idx] = (float)N6[c];
                if (K64) K64[idx] = N6[c];
            }
        }
    }
    free(pts);
}

/* x^(1/5) for the step-size control (RKSuitef90.f90 uses (tol/err)**expon
 * with expon = 1/5).  libm pow differs between the host and the device in the
 * last bits, so both sides use this fixed iteration of IEEE operations:
 * x = f 2^e, e = 5 q + r, y = f 2^r in [0.5, 16), twelve Newton steps
 * z <- z + (y / z^4 - z) / 5 from z = 1 (y < 2) or 1.5, result 2^q z. */
static double or_root5(double x)
{
    if (!(x > 0.0)) return 0.0;
    if (isinf(x)) return x;
    int e = 0;
    const double f = frexp(x, &e);
    const int q = (e >= 0) ? e / 5 : -((-e + 4) / 5);
    const double y = ldexp(f, e - 5 * q);
    double z = (y < 2.0) ? 1.0 : 1.5;
    for (int k = 0; k < 12; ++k) {
        const double z2 = z * z;
        const double z4 = z2 * z2;
        z = z + (y / z4 - z) / 5.0;
    }
    return ldexp(z, q);
}

/* ------------------------------------------------------------------ */
/* problem and right-hand side                                         */
/* ------------------------------------------------------------------ */
typedef struct {
    int nx, ny, nz, n;
    double d[3];
    int solver;              /* 1 explicit, 2 dynamic */
    int mode;                /* 0 ref (FP32 demag), 1 fp64 */
    double gamma, alpha0;
    int nt_alpha; double* alpha_tab;  /* [k*2 + {t, alpha}] */
    int nt_hext; double* hext;        /* [k*4 + {t, hx, hy, hz}] */
    int hext_ind;                     /* explicit-mode row, 0-based */
    double* Jfact; double* Kfact; float* Mfact;
    double* A6;                       /* [c*n + i]: Axx Axy Axz Ayy Ayz Azz */
    double lap_coef[3];               /* 1/d^2 per axis as the reference forms it */
    const float* K32;                 /* [c][i][j], owned by caller */
    const double* K64;
    float* KT32;                      /* [c][j][i]: the same tensors by source column, owned here */
    double* KT64;
    int renorm;                       /* per-cell |m| renormalisation after accepted steps */
    float* ms;                        /* FP32 copy of m for the demag product */
    long nrhs;
    /* mode 2: limbs [4][3n][3n] of the fixed-point tensor rows, 2^(-30-e_r) per row */
    signed char* klimb;
    double* row_scale;
    int* mlimb;                       /* [4][3n] limbs of the current m */
    int range_err;                    /* a component of m outside (-1.96, 1.96) was seen */
} or_problem;

or_problem* or_problem_create(int nx, int ny, int nz, double Lx, double Ly, double Lz,
                              int solver, int mode, double A0, const double* Ms, const double* K0,
                              const double* u_ea /* n*3, [i*3+c] */, double gamma, double alpha0,
                              const double* alpha_tab, int nt_alpha, const double* hext, int nt_hext)
{
    or_problem* p = (or_problem*)calloc(1, sizeof(or_problem));
    int n = nx * ny * nz;
    p->nx = nx; p->ny = ny; p->nz = nz; p->n = n;
    double* tmp = (double*)malloc(sizeof(double) * 3 * (size_t)n);
    or_grid(nx, ny, nz, Lx, Ly, Lz, tmp, p->d);
    free(tmp);
    p->solver = solver; p->mode = mode; p->gamma = gamma; p->alpha0 = alpha0;
    p->nt_alpha = nt_alpha;
    p->alpha_tab = (double*)malloc(sizeof(double) * 2 * (nt_alpha > 0 ? nt_alpha : 1));
    if (nt_alpha > 0) memcpy(p->alpha_tab, alpha_tab, sizeof(double) * 2 * nt_alpha);
    p->nt_hext = nt_hext;
    p->hext = (double*)malloc(sizeof(double) * 4 * (nt_hext > 0 ? nt_hext : 1));
    if (nt_hext > 0) memcpy(p->hext, hext, sizeof(double) * 4 * nt_hext);
    p->Jfact = (double*)malloc(sizeof(double) * n);
    p->Kfact = (double*)malloc(sizeof(double) * n);
    p->Mfact = (float*)malloc(sizeof(float) * n);
    p->A6 = (double*)malloc(sizeof(double) * 6 * (size_t)n);
    p->ms = (float*)malloc(sizeof(float) * 3 * (size_t)n);
    double mu0 = or_mu0();
    for (int i = 0; i < n; ++i) {
        p->Jfact[i] = A0 / (mu0 * Ms[i]);
        p->Kfact[i] = K0[i] / (mu0 * Ms[i]);
        p->Mfact[i] = (float)Ms[i];
        double ux = u_ea[i * 3 + 0], uy = u_ea[i * 3 + 1], uz = u_ea[i * 3 + 2];
        p->A6[0 * (size_t)n + i] = ux * ux;
        p->A6[1 * (size_t)n + i] = ux * uy;
        p->A6[2 * (size_t)n + i] = ux * uz;
        p->A6[3 * (size_t)n + i] = uy * uy;
        p->A6[4 * (size_t)n + i] = uy * uz;
        p->A6[5 * (size_t)n + i] = uz * uz;
    }
    for (int a = 0; a < 3; ++a) p->lap_coef[a] = 1.0 / (p->d[a] * p->d[a]);
    return p;
}

/* Source-column copies of the tensors for the column sweep of the demag product. */
static void *or_transpose(const void* src, int n, size_t es)
{
    if (!src) return NULL;
    char* dst = (char*)malloc(es * 6 * (size_t)n * n);
    const char* s = (const char*)src;
#pragma omp parallel for collapse(2) schedule(static)
    for (int c = 0; c < 6; ++c)
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i)
                memcpy(dst + es * (((size_t)c * n + j) * n + i), s + es * (((size_t)c * n + i) * n + j), es);
    return dst;
}

void or_problem_set_tensor(or_problem* p, const float* K32, const double* K64)
{
    p->K32 = K32; p->K64 = K64;
    free(p->KT32); free(p->KT64);
    p->KT32 = (float*)or_transpose(K32, p->n, sizeof(float));
    p->KT64 = (double*)or_transpose(K64, p->n, sizeof(double));
}
void or_problem_set_hext_ind(or_problem* p, int ind) { p->hext_ind = ind; }
void or_problem_set_renorm(or_problem* p, int on) { p->renorm = on; }
void or_problem_set_alpha0(or_problem* p, double a) { p->alpha0 = a; }
long or_problem_nrhs(const or_problem* p) { return p->nrhs; }

void or_problem_destroy(or_problem* p)
{
    if (!p) return;
    free(p->alpha_tab); free(p->hext); free(p->Jfact); free(p->Kfact); free(p->Mfact);
    free(p->A6); free(p->ms); free(p->klimb); free(p->row_scale); free(p->mlimb);
    free(p->KT32); free(p->KT64); free(p);
}
int or_problem_range_err(const or_problem* p) { return p->range_err; }

/* The demag product H_a(i) = Ms_i * sum_b sum_j (-m_b(j)) K_ab(i, j) as the reference
 * BLAS SGEMV sweeps it (LandauLifshitzEquationSolver.f90:718-747): for every
 * component a, y = 0, then for each block b = 1..3 and source j = 1..n in order,
 * y(i) = y(i) + (-m_b(j)) * K_ab(i, j), each multiply and add rounded separately;
 * finally Ms_i * y(i).  The sweep runs over source columns of the column-major
 * copy, so it vectorises across the receivers i in [i0, i1) without changing any
 * receiver's order of operations (blocks: x: xx xy xz; y: xy yy yz; z: xz yz zz). */
static const int or_blk[3][3] = {{0, 1, 2}, {1, 3, 4}, {2, 4, 5}};

__attribute__((target_clones("avx2", "default")))
static void colsweep_f32(const float* KT, int n, const float* ms, const float* Mfact, int i0, int i1, double* Hm)
{
    float* y = (float*)malloc(sizeof(float) * (size_t)(i1 > i0 ? i1 - i0 : 1));
    for (int a = 0; a < 3; ++a) {
        for (int i = i0; i < i1; ++i) y[i - i0] = 0.0f;
        for (int b = 0; b < 3; ++b) {
            const float* K = KT + (size_t)or_blk[a][b] * n * n;
            const float* xb = ms + (size_t)b * n;
            for (int j = 0; j < n; ++j) {
                const float tmp = -xb[j];
                const float* col = K + (size_t)j * n + i0;
                float* yy = y;
                const int len = i1 - i0;
#pragma omp simd
                for (int i = 0; i < len; ++i) yy[i] = yy[i] + tmp * col[i];
            }
        }
        for (int i = i0; i < i1; ++i) {
            const float hm = y[i - i0] * Mfact[i];
            Hm[(size_t)a * n + i] = (double)hm;
        }
    }
    free(y);
}

__attribute__((target_clones("avx2", "default")))
static void colsweep_f64(const double* KT, int n, const double* m, const float* Mfact, int i0, int i1, double* Hm)
{
    double* y = (double*)malloc(sizeof(double) * (size_t)(i1 > i0 ? i1 - i0 : 1));
    for (int a = 0; a < 3; ++a) {
        for (int i = i0; i < i1; ++i) y[i - i0] = 0.0;
        for (int b = 0; b < 3; ++b) {
            const double* K = KT + (size_t)or_blk[a][b] * n * n;
            const double* xb = m + (size_t)b * n;
            for (int j = 0; j < n; ++j) {
                const double tmp = -xb[j];
                const double* col = K + (size_t)j * n + i0;
                double* yy = y;
                const int len = i1 - i0;
#pragma omp simd
                for (int i = 0; i < len; ++i) yy[i] = yy[i] + tmp * col[i];
            }
        }
        for (int i = i0; i < i1; ++i) Hm[(size_t)a * n + i] = y[i - i0] * (double)Mfact[i];
    }
    free(y);
}

/* this thread's receivers of an OpenMP team: contiguous blocks of 16 */
static void or_thread_cells(int n, int* i0, int* i1)
{
    const int nth = omp_get_num_threads(), t = omp_get_thread_num();
    const int blocks = (n + 15) / 16;
    const int b0 = (int)((long long)blocks * t / nth), b1 = (int)((long long)blocks * (t + 1) / nth);
    *i0 = b0 * 16 < n ? b0 * 16 : n;
    *i1 = b1 * 16 < n ? b1 * 16 : n;
}

/* mode 2 tensor limbs from the FP32 tensor: row r = (a, i), column (b, j).
 * 2^e_r puts the row's largest |K| in [2^29, 2^30); Kq = rint(K 2^e_r) =
 * k0 2^24 + k1 2^16 + k2 2^8 + k3 with signed 8-bit digits (k3 the lowest);
 * row_scale = 2^(-30 - e_r). */
static void or_i8_build(or_problem* p)
{
    const int n = p->n, n3 = 3 * n;
    static const int blk[3][3] = {{0, 1, 2}, {1, 3, 4}, {2, 4, 5}};
    const size_t tot = (size_t)n3 * n3;
    p->klimb = (signed char*)malloc(4 * tot);
    p->row_scale = (double*)malloc(sizeof(double) * n3);
    p->mlimb = (int*)malloc(sizeof(int) * 4 * (size_t)n3);
#pragma omp parallel for schedule(static)
    for (int r = 0; r < n3; ++r) {
        const int a = r / n, i = r - a * n;
        float mx = 0.0f;
        for (int b = 0; b < 3; ++b)
            for (int j = 0; j < n; ++j) {
                float v = fabsf(p->K32[((size_t)blk[a][b] * n + i) * (size_t)n + j]);
                if (v > mx) mx = v;
            }
        int e = 0;
        if (mx > 0.0f) frexpf(mx, &e);
        const int ex = (mx > 0.0f) ? 30 - e : 0;
        p->row_scale[r] = (mx > 0.0f) ? ldexp(1.0, -30 - ex) : 0.0;
        for (int b = 0; b < 3; ++b)
            for (int j = 0; j < n; ++j) {
                const float v = p->K32[((size_t)blk[a][b] * n + i) * (size_t)n + j];
                long long x = llrint(ldexp((double)v, ex));
                const size_t e2 = (size_t)r * n3 + (size_t)b * n + j;
                for (int l = 3; l >= 1; --l) {
                    const int d = (int)(signed char)(x & 0xff);
                    p->klimb[(size_t)l * tot + e2] = (signed char)d;
                    x = (x - d) >> 8;
                }
                p->klimb[e2] = (signed char)x;
            }
    }
}

/* mode 2 demag field: Hm = -Ms_i * 2^(-30-e_r) * RN(H_int) with the exact
 * H_int = sum_j Kq_rj mq_j = sum_s 2^(8(6-s)) D_s, D_s = sum_j sum_{a+b=s} k_a m_b
 * (all sixteen limb products), kept as 2^24 Hhi + Hlo (Hhi from D0..D3, Hlo
 * from D4..D6) so that no int64 overflows, and rounded to double once */
static void or_i8_demag(or_problem* p, const double* m, double* Hm)
{
    const int n = p->n, n3 = 3 * n;
    const size_t tot = (size_t)n3 * n3;
    if (!p->klimb) or_i8_build(p);
    int* ml = p->mlimb;
    for (int j = 0; j < n3; ++j) {
        double v = m[j];
        if (!(fabs(v) <= 1.96)) { p->range_err = 1; v = 0.0; }
        long long x = llrint(v * 1073741824.0);
        int d[4];
        for (int l = 3; l >= 1; --l) {
            const int dl = (int)(signed char)(x & 0xff);
            d[l] = dl;
            x = (x - dl) >> 8;
        }
        d[0] = (int)x;
        for (int l = 0; l < 4; ++l) ml[(size_t)l * n3 + j] = d[l];
    }
#pragma omp parallel for schedule(static)
    for (int r = 0; r < n3; ++r) {
        int D[7] = {0, 0, 0, 0, 0, 0, 0};
        for (int a = 0; a < 4; ++a)
            for (int b = 0; b < 4; ++b) {
                const signed char* kr = p->klimb + (size_t)a * tot + (size_t)r * n3;
                const int* mr = ml + (size_t)b * n3;
                int acc = 0;
                for (int j = 0; j < n3; ++j) acc += (int)kr[j] * mr[j];
                D[a + b] += acc;
            }
        long long hi = (long long)D[0];
        for (int s2 = 1; s2 < 4; ++s2) hi = hi * 256 + (long long)D[s2];
        long long lo = (long long)D[4];
        for (int s2 = 5; s2 < 7; ++s2) lo = lo * 256 + (long long)D[s2];
        const double h = (double)hi * 16777216.0 + (double)lo;
        const int i = r % n;
        Hm[r] = (-(double)p->Mfact[i]) * (h * p->row_scale[r]);
    }
}

/* locate + interp1_MagTense (util.f90:39-85).  Outside the table the value is 0;
 * above the last knot the reference reads past the table (undefined), here 0. */
double or_interp1(const double* tab, int stride, int col, int nt, double xv)
{
    if (nt < 2) return 0.0;
    int jl = 0, ju = nt + 1;
    int ascending = tab[(nt - 1) * stride] >= tab[0];
    while (ju - jl > 1) {
        int jm = (ju + jl) / 2;
        int ge = xv >= tab[(jm - 1) * stride];
        if (ascending == ge) jl = jm; else ju = jm;
    }
    int j;
    if (xv == tab[0]) j = 1;
    else if (xv == tab[(nt - 1) * stride]) j = nt - 1;
    else j = jl;
    if (j == 0 || j >= nt) return 0.0;
    double x0 = tab[(j - 1) * stride], x1 = tab[j * stride];
    double y0 = tab[(j - 1) * stride + col], y1 = tab[j * stride + col];
    double xl = (xv - x0) / (x1 - x0);
    return (1.0 - xl) * y0 + xl * y1;
}

static double or_alpha(const or_problem* p, double t)
{
    if (p->alpha0 == 0.0) return or_interp1(p->alpha_tab, 2, 1, p->nt_alpha, t);
    return p->alpha0;
}

/* Exchange operator L m for one component (Neumann 7/5-point Laplacian).  The
 * diagonal is the sum of the per-axis diagonals, as mkl_sparse_d_add merges
 * them; off-diagonal terms are summed in increasing column order. */
static double lap_cell(const or_problem* p, const double* v, int i)
{
    int nx = p->nx, ny = p->ny, nz = p->nz;
    int ix = i % nx, iy = (i / nx) % ny, iz = i / (nx * ny);
    double cx = p->lap_coef[0], cy = p->lap_coef[1], cz = p->lap_coef[2];
    double dgx = 0.0, dgy = 0.0, dgz = 0.0;
    if (nx > 1) dgx = (ix == 0 || ix == nx - 1) ? -1.0 / (p->d[0] * p->d[0]) : -2.0 / (p->d[0] * p->d[0]);
    if (ny > 1) dgy = (iy == 0 || iy == ny - 1) ? -1.0 / (p->d[1] * p->d[1]) : -2.0 / (p->d[1] * p->d[1]);
    if (nz > 1) dgz = (iz == 0 || iz == nz - 1) ? -1.0 / (p->d[2] * p->d[2]) : -2.0 / (p->d[2] * p->d[2]);
    double diag = dgx + dgy;
    if (nz > 1) diag = diag + dgz;
    double s = 0.0;
    int first = 1;
#define ACC(term) do { double _t = (term); if (first) { s = _t; first = 0; } else s = s + _t; } while (0)
    if (nz > 1 && iz > 0) ACC(cz * v[i - nx * ny]);
    if (ny > 1 && iy > 0) ACC(cy * v[i - nx]);
    if (nx > 1 && ix > 0) ACC(cx * v[i - 1]);
    ACC(diag * v[i]);
    if (nx > 1 && ix < nx - 1) ACC(cx * v[i + 1]);
    if (ny > 1 && iy < ny - 1) ACC(cy * v[i + nx]);
    if (nz > 1 && iz < nz - 1) ACC(cz * v[i + nx * ny]);
#undef ACC
    return s;
}

/* All four field terms (the reference's internal "H" = minus the physical field). */
void or_fields(or_problem* p, double t, const double* m, double* Hj, double* Hh, double* Hk, double* Hm)
{
    int n = p->n;
    const double* mx = m;
    const double* my = m + n;
    const double* mz = m + 2 * (size_t)n;
    /* Zeeman */
    double hx = 0, hy = 0, hz = 0;
    if (p->solver == 1) {
        hx = p->hext[p->hext_ind * 4 + 1]; hy = p->hext[p->hext_ind * 4 + 2]; hz = p->hext[p->hext_ind * 4 + 3];
    } else if (p->solver == 2) {
        hx = or_interp1(p->hext, 4, 1, p->nt_hext, t);
        hy = or_interp1(p->hext, 4, 2, p->nt_hext, t);
        hz = or_interp1(p->hext, 4, 3, p->nt_hext, t);
    }
    for (int i = 0; i < n; ++i) {
        /* exchange: y = -2 * (A m), then * Jfact */
        Hj[i] = (-2.0 * lap_cell(p, mx, i)) * p->Jfact[i];
        Hj[n + i] = (-2.0 * lap_cell(p, my, i)) * p->Jfact[i];
        Hj[2 * n + i] = (-2.0 * lap_cell(p, mz, i)) * p->Jfact[i];
        Hh[i] = -hx; Hh[n + i] = -hy; Hh[2 * n + i] = -hz;
        const double* A = p->A6;
        double k2 = -2.0 * p->Kfact[i];
        Hk[i] = k2 * ((A[0 * n + i] * mx[i] + A[1 * n + i] * my[i]) + A[2 * n + i] * mz[i]);
        Hk[n + i] = k2 * ((A[1 * n + i] * mx[i] + A[3 * n + i] * my[i]) + A[4 * n + i] * mz[i]);
        Hk[2 * n + i] = k2 * ((A[2 * n + i] * mx[i] + A[4 * n + i] * my[i]) + A[5 * n + i] * mz[i]);
    }
    /* demag */
    if (p->mode == 2) {
        or_i8_demag(p, m, Hm);
    } else if (p->mode == 0) {
        float* ms = p->ms;
        for (int i = 0; i < 3 * n; ++i) ms[i] = (float)m[i];
#pragma omp parallel
        {
            int i0, i1;
            or_thread_cells(n, &i0, &i1);
            colsweep_f32(p->KT32, n, ms, p->Mfact, i0, i1, Hm);
        }
    } else {
#pragma omp parallel
        {
            int i0, i1;
            or_thread_cells(n, &i0, &i1);
            colsweep_f64(p->KT64, n, m, p->Mfact, i0, i1, Hm);
        }
    }
}

/* dmdt_fct: dm/dt = -gamma * (-(m x Heff)) - alpha * (m x (-(m x Heff))) */
void or_rhs(or_problem* p, double t, const double* m, double* dmdt)
{
    int n = p->n;
    double* H = (double*)malloc(sizeof(double) * 12 * (size_t)n);
    double *Hj = H, *Hh = H + 3 * n, *Hk = H + 6 * n, *Hm = H + 9 * n;
    or_fields(p, t, m, Hj, Hh, Hk, Hm);
    double al = or_alpha(p, t);
    double g = p->gamma;
    for (int i = 0; i < n; ++i) {
        double mx = m[i], my = m[n + i], mz = m[2 * n + i];
        double hx = ((Hh[i] + Hj[i]) + Hm[i]) + Hk[i];
        double hy = ((Hh[n + i] + Hj[n + i]) + Hm[n + i]) + Hk[n + i];
        double hz = ((Hh[2 * n + i] + Hj[2 * n + i]) + Hm[2 * n + i]) + Hk[2 * n + i];
        double cx = -1.0 * (my * hz - mz * hy);
        double cy = -1.0 * (mz * hx - mx * hz);
        double cz = -1.0 * (mx * hy - my * hx);
        double h2x = my * cz - mz * cy;
        double h2y = mz * cx - mx * cz;
        double h2z = mx * cy - my * cx;
        dmdt[i] = -g * cx - al * h2x;
        dmdt[n + i] = -g * cy - al * h2y;
        dmdt[2 * n + i] = -g * cz - al * h2z;
    }
    free(H);
    p->nrhs++;
}

/* ------------------------------------------------------------------ */
/* RKSUITE-90 method 'M' (Bogacki-Shampine 4(5), FSAL, 6th-degree     */
/* interpolant with three extra stages)                               */
/* ------------------------------------------------------------------ */
typedef void (*or_rhs_fn)(void* ctx, double t, const double* y, double* f);

/* Published Bogacki-Shampine (1989) 4(5) pair as tabulated by RKSUITE
 * (RKSuitef90.f90:252-411).  Indices are 1-based to match the publication. */
typedef struct { double a[12][12], b[9], c[12], e[8], r[12][7]; } bs45_tab;

static void bs45_init(bs45_tab* T)
{
    memset(T, 0, sizeof(*T));
    double (*a)[12] = T->a;
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
    T->b[1] = 2479.0 / 34992.0; T->b[2] = 0.0; T->b[3] = 123.0 / 416.0; T->b[4] = 612941.0 / 3411720.0;
    T->b[5] = 43.0 / 1440.0; T->b[6] = 2272.0 / 6561.0; T->b[7] = 79937.0 / 1113912.0;
    T->b[8] = 3293.0 / 556956.0;
    T->e[1] = -3.0 / 1280.0; T->e[2] = 0.0; T->e[3] = 6561.0 / 632320.0; T->e[4] = -343.0 / 20800.0;
    T->e[5] = 243.0 / 12800.0; T->e[6] = -1.0 / 95.0; T->e[7] = 0.0;
    T->c[1] = 0.0; T->c[2] = 1.0 / 6.0; T->c[3] = 2.0 / 9.0; T->c[4] = 3.0 / 7.0; T->c[5] = 2.0 / 3.0;
    T->c[6] = 3.0 / 4.0; T->c[7] = 1.0; T->c[8] = 1.0;
    T->c[9] = 1.0 / 2.0; T->c[10] = 5.0 / 6.0; T->c[11] = 1.0 / 9.0;
    a[9][1] = 455.0 / 6144.0; a[10][1] = -837888343715.0 / 13176988637184.0;
    a[11][1] = 98719073263.0 / 1551965184000.0;
    a[9][2] = 0.0; a[10][2] = 30409415.0 / 52955362.0; a[11][2] = 1307.0 / 123552.0;
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
    double (*r)[7] = T->r;
    r[1][6] = -12134338393.0 / 1050809760.0; r[1][5] = -1620741229.0 / 50038560.0;
    r[1][4] = -2048058893.0 / 59875200.0; r[1][3] = -87098480009.0 / 5254048800.0;
    r[1][2] = -11513270273.0 / 3502699200.0;
    r[3][6] = -33197340367.0 / 1218433216.0; r[3][5] = -539868024987.0 / 6092166080.0;
    r[3][4] = -39991188681.0 / 374902528.0; r[3][3] = -69509738227.0 / 1218433216.0;
    r[3][2] = -29327744613.0 / 2436866432.0;
    r[4][6] = -284800997201.0 / 19905339168.0; r[4][5] = -7896875450471.0 / 165877826400.0;
    r[4][4] = -333945812879.0 / 5671036800.0; r[4][3] = -16209923456237.0 / 497633479200.0;
    r[4][2] = -2382590741699.0 / 331755652800.0;
    r[5][6] = -540919.0 / 741312.0; r[5][5] = -103626067.0 / 43243200.0;
    r[5][4] = -633779.0 / 211200.0; r[5][3] = -32406787.0 / 18532800.0;
    r[5][2] = -36591193.0 / 86486400.0;
    r[6][6] = 7157998304.0 / 374350977.0; r[6][5] = 30405842464.0 / 623918295.0;
    r[6][4] = 183022264.0 / 5332635.0; r[6][3] = -3357024032.0 / 1871754885.0;
    r[6][2] = -611586736.0 / 89131185.0;
    r[7][6] = -138073.0 / 9408.0; r[7][5] = -719433.0 / 15680.0; r[7][4] = -1620541.0 / 31360.0;
    r[7][3] = -385151.0 / 15680.0; r[7][2] = -65403.0 / 15680.0;
    r[8][6] = 1245.0 / 64.0; r[8][5] = 3991.0 / 64.0; r[8][4] = 4715.0 / 64.0;
    r[8][3] = 2501.0 / 64.0; r[8][2] = 149.0 / 16.0; r[8][1] = 1.0;
    r[9][6] = 55.0 / 3.0; r[9][5] = 71.0; r[9][4] = 103.0; r[9][3] = 199.0 / 3.0; r[9][2] = 16.0;
    r[10][6] = -1774004627.0 / 75810735.0; r[10][5] = -1774004627.0 / 25270245.0;
    r[10][4] = -26477681.0 / 359975.0; r[10][3] = -11411880511.0 / 379053675.0;
    r[10][2] = -423642896.0 / 126351225.0;
    r[11][6] = 35.0; r[11][5] = 105.0; r[11][4] = 117.0; r[11][3] = 59.0; r[11][2] = 12.0;
}

/* Integrator state.  Vector naming follows the method: k[1] is the derivative at
 * the start of the step, k[2..8] the stages of the step (k[8] = derivative at the
 * end, FSAL), k[9..11] the extra stages of the interpolant. */
typedef struct {
    bs45_tab T;
    int neq;
    or_rhs_fn f; void* ctx;
    double t, t_old, t_start, t_end, dir;
    double h, h_old, h_average, tol;
    long f_count, full_f_count, step_count, bad_step_count, stiff_bad_step_count;
    int at_t_start, at_t_end, phase2, chkeff, hit_t_end_count;
    double errold;
    double round_off, sqrrmc, cubrmc, sqtiny, toosml;
    double expon, safety, stability_radius, tan_angle, rs, rs1, rs2, rs3, rs4, cost;
    int max_stiff_iters;
    double tlast, range_t_end;
    int intrp_ready;          /* interpolant formed for the current step */
    int last_step_flag;       /* state of STEP_INTEGRATE after its last call */
    int renorm;
    double *thresh, *weights, *y, *yp, *y_new, *y_old, *yp_old, *errest, *ymax;
    double *stg[12];          /* stg[2..11] */
    double *p[6];             /* p[1..5] interpolant coefficients */
    double *ytemp, *vtemp;
    int ncell;                /* for renormalisation: neq = 3*ncell */
} or_rk;

static void vmax_abs(int n, const double* a, const double* b, double* out)
{
    for (int i = 0; i < n; ++i) out[i] = fmax(fabs(a[i]), b[i]);
}

static void rk_renorm(or_rk* R, double* v)
{
    int nc = R->ncell;
    for (int i = 0; i < nc; ++i) {
        double x = v[i], y = v[nc + i], z = v[2 * nc + i];
        double s = sqrt(x * x + y * y + z * z);
        if (s > 0.0) { v[i] = x / s; v[nc + i] = y / s; v[2 * nc + i] = z / s; }
    }
}

/* status codes returned by the integrator routines */
enum { RK_OK = 1, RK_FATAL = 911 };

static int rk_setup(or_rk* R, or_rhs_fn f, void* ctx, int neq, double t_start, const double* y_start,
                    double t_end, double tol, const double* thresh)
{
    memset(R, 0, sizeof(*R));
    bs45_init(&R->T);
    R->f = f; R->ctx = ctx; R->neq = neq;
    double eps = DBL_EPSILON;
    R->round_off = 10.0 * eps;
    R->sqrrmc = sqrt(eps);
    R->cubrmc = pow(eps, 1.0 / 3.0);
    R->sqtiny = sqrt(DBL_MIN);
    /* method constants (RKSuitef90.f90:244-248, :568-591) */
    R->safety = 0.8; R->stability_radius = 3.9; R->tan_angle = 5.2;
    R->cost = 7.0;
    R->max_stiff_iters = 8;
    R->expon = 1.0 / (4.0 + 1.0);
    R->rs = 2.0; R->rs1 = 1.0 / R->rs; R->rs2 = R->rs * R->rs; R->rs3 = R->rs * R->rs2; R->rs4 = 1.0 / R->rs3;
    double cdiff = 1.0;
    for (int i = 1; i <= 7; ++i)
        for (int j = i + 1; j <= 8; ++j) {
            double dd = R->T.c[i] - R->T.c[j];
            if (dd != 0.0) cdiff = fmin(cdiff, fabs(dd));
        }
    R->toosml = R->round_off / cdiff;
    R->phase2 = 1; R->at_t_start = 1;
    if (t_start == t_end) return -1;
    R->t_end = t_end; R->t_start = t_start; R->t_old = t_start; R->t = t_start;
    R->dir = (t_end - t_start) >= 0 ? 1.0 : -1.0;
    if (tol > 0.01 || tol < R->round_off) return -2;
    R->tol = tol;
    double tmin = thresh[0];
    for (int i = 1; i < neq; ++i) tmin = fmin(tmin, thresh[i]);
    if (tmin < R->sqtiny) return -3;
    double hmin = fmax(R->sqtiny, R->toosml * fmax(fabs(t_start), fabs(t_end)));
    if (fabs(t_end - t_start) < hmin) return -4;
    R->h = fmax(fabs(t_end - t_start) / R->rs3, hmin);
    size_t sz = sizeof(double) * (size_t)neq;
    double** vecs[] = {&R->thresh, &R->weights, &R->y, &R->yp, &R->y_new, &R->y_old, &R->yp_old,
                       &R->errest, &R->ymax, &R->ytemp, &R->vtemp};
    for (size_t k = 0; k < sizeof(vecs) / sizeof(vecs[0]); ++k) *vecs[k] = (double*)calloc(1, sz);
    for (int k = 2; k <= 11; ++k) R->stg[k] = (double*)calloc(1, sz);
    for (int k = 1; k <= 5; ++k) R->p[k] = (double*)calloc(1, sz);
    memcpy(R->y, y_start, sz);
    for (int i = 0; i < neq; ++i) R->ymax[i] = fabs(y_start[i]);
    memcpy(R->thresh, thresh, sz);
    R->last_step_flag = 0;
    return 0;
}

static void rk_free(or_rk* R)
{
    double* vecs[] = {R->thresh, R->weights, R->y, R->yp, R->y_new, R->y_old, R->yp_old,
                      R->errest, R->ymax, R->ytemp, R->vtemp};
    for (size_t k = 0; k < sizeof(vecs) / sizeof(vecs[0]); ++k) free(vecs[k]);
    for (int k = 2; k <= 11; ++k) free(R->stg[k]);
    for (int k = 1; k <= 5; ++k) free(R->p[k]);
}

static double vnorm_max_w(int n, const double* v, const double* w)
{
    double m = fabs(v[0]) / w[0];
    for (int i = 1; i < n; ++i) m = fmax(m, fabs(v[i]) / w[i]);
    return m;
}

/* One attempt of the step of size *htry from (t, y, yp).  Returns err. */
static double rk_step(or_rk* R, double tnow, double* htry, double hmin)
{
    const bs45_tab* T = &R->T;
    int n = R->neq;
    double err = 0.0;
    double* y = R->y;
    double* yp = R->yp;
    double* es = R->errest;
    double* yn = R->y_new;
    for (;;) {                                     /* attempt_step */
        if (R->phase2) vmax_abs(n, y, R->thresh, R->weights);
        int restart = 0;
        for (int i = 2; i <= 8; ++i) {
            for (int q = 0; q < n; ++q) es[q] = T->a[i][1] * yp[q];
            for (int j = 2; j <= i - 1; ++j) {
                if (T->a[i][j] == 0.0) continue;
                const double* s = R->stg[j];
                for (int q = 0; q < n; ++q) es[q] = es[q] + T->a[i][j] * s[q];
            }
            for (int q = 0; q < n; ++q) yn[q] = y[q] + (*htry) * es[q];
            if (i == 7) {                                   /* stepb: early error estimate */
                double mx = 0.0;
                for (int q = 0; q < n; ++q) {
                    double v = T->e[1] * yp[q] + T->e[3] * R->stg[3][q] + T->e[4] * R->stg[4][q]
                             + T->e[5] * R->stg[5][q] + T->e[6] * R->stg[6][q];
                    double w = fmax(0.5 * (fabs(y[q]) + fabs(yn[q])), R->thresh[q]);
                    double r = fabs(v) / w;
                    mx = (q == 0) ? r : fmax(mx, r);
                }
                err = fabs(R->h) * mx;
                if (err > R->tol) return err;
            }
            double tstg = tnow + T->c[i] * (*htry);
            if (R->at_t_end && T->c[i] == 1.0) tstg = R->t_end;
            R->f(R->ctx, tstg, yn, R->stg[i]);
            R->f_count++;
            if (R->phase2 && i <= 3 && fabs(*htry) > hmin) {  /* stepa */
                double* w = R->weights;
                const double* ypn = R->stg[i];
                for (int q = 0; q < n; ++q) w[q] = fmax(w[q], fabs(yn[q]));
                double ynrm = 0, ystgnm = 0, argdif = 0, fdiff = 0;
                for (int q = 0; q < n; ++q) {
                    double a1 = fabs(y[q]) / w[q], a2 = fabs(yn[q]) / w[q];
                    double a3 = fabs(yn[q] - y[q]) / w[q], a4 = fabs(ypn[q] - yp[q]) / w[q];
                    if (q == 0) { ynrm = a1; ystgnm = a2; argdif = a3; fdiff = a4; }
                    else { ynrm = fmax(ynrm, a1); ystgnm = fmax(ystgnm, a2); argdif = fmax(argdif, a3); fdiff = fmax(fdiff, a4); }
                }
                double tdiff = tstg - tnow;
                double twt = fabs(R->t_end - tnow);
                ynrm = fmax(ynrm, fabs(tnow) / twt);
                ystgnm = fmax(ystgnm, fabs(tstg) / twt);
                argdif = fmax(argdif, fabs(tdiff) / twt);
                int cutbak = 0;
                if (argdif > R->round_off * fmax(ynrm, ystgnm)) {
                    if (fabs(*htry) * fdiff > R->stability_radius * argdif) {
                        double scl = fmax(R->rs4, fmin(R->rs1, (R->stability_radius * argdif) / (fabs(*htry) * fdiff)));
                        *htry = scl * (*htry);
                        cutbak = 1;
                    }
                }
                if (cutbak) {
                    R->at_t_end = 0;
                    if (fabs(*htry) <= hmin) { *htry = copysign(hmin, *htry); R->phase2 = 0; }
                    restart = 1;
                    break;
                }
            }
        }
        if (restart) continue;
        /* error estimate of the 4th-order formula against the 5th-order result */
        for (int q = 0; q < n; ++q) es[q] = es[q] - T->b[1] * yp[q];
        for (int i = 2; i <= 8; ++i) {
            if (T->b[i] == 0.0) continue;
            const double* s = R->stg[i];
            for (int q = 0; q < n; ++q) es[q] = es[q] - T->b[i] * s[q];
        }
        for (int q = 0; q < n; ++q) es[q] = (*htry) * es[q];
        for (int q = 0; q < n; ++q) R->weights[q] = fmax(0.5 * (fabs(y[q]) + fabs(yn[q])), R->thresh[q]);
        err = vnorm_max_w(n, es, R->weights);
        return err;
    }
}

static double wip(const or_rk* R, const double* a, const double* b)
{
    double s = 0.0;
    for (int i = 0; i < R->neq; ++i) s = s + (a[i] / R->weights[i]) * (b[i] / R->weights[i]);
    return s;
}

static void quad_roots(double alpha, double beta, double complex* r)
{
    double tmp = alpha / 2.0;
    double complex temp = tmp;
    /* temp**2 of a real-valued complex: imaginary part carries the sign of tmp*0 */
    double complex t2 = CMPLX(tmp * tmp, tmp * 0.0 + 0.0 * tmp);
    double complex disc = CMPLX(creal(t2) - beta, cimag(t2) - 0.0);
    double complex sq = csqrt(disc);
    if (sq == 0.0) { r[0] = -temp; r[1] = -temp; return; }
    double complex r1 = -temp + sq, r2 = -temp + sq;   /* as tabulated in the vendored code */
    if (cabs(r1) > cabs(r2)) { r[0] = r1; r[1] = r2; } else { r[0] = r2; r[1] = r1; }
}

/* stiffness diagnosis; returns 1 when the problem is diagnosed as stiff */
static int rk_stiff(or_rk* R, int toomch)
{
    int n = R->neq;
    int lots_of_fails = 0;
    if ((R->step_count - 10) % 40 == 0) {
        lots_of_fails = R->stiff_bad_step_count >= 10;
        R->stiff_bad_step_count = 0;
    }
    int maybe = toomch || lots_of_fails;
    double v0v0 = 0, scale = 0;
    if (maybe) {
        for (int q = 0; q < n; ++q) R->weights[q] = fmax(0.5 * (fabs(R->y[q]) + fabs(R->y_old[q])), R->thresh[q]);
        double rat = fabs(R->h / R->h_average);
        maybe = 0.2 < rat && rat < 5.0;
        if (maybe) {
            maybe = R->cost * fabs((R->t_end - R->t) / R->h_average) > 5000.0;
            if (maybe) {
                v0v0 = wip(R, R->errest, R->errest);
                double yy = wip(R, R->y, R->y);
                double ynrm = sqrt(yy);
                scale = ynrm * R->sqrrmc;
                if (scale == 0.0) { scale = v0v0 * R->sqrrmc; maybe = scale > 0.0; }
            }
        }
    }
    if (!maybe) return 0;
    double* v0 = R->errest;
    double* v1 = R->stg[2];
    double* v2 = R->stg[3];
    double* v3 = R->stg[4];
    if (v0v0 == 0.0) { for (int q = 0; q < n; ++q) v0[q] = 1.0; v0v0 = wip(R, v0, v0); }
    double v0nrm = sqrt(v0v0);
    for (int q = 0; q < n; ++q) v0[q] = v0[q] / v0nrm;
    v0v0 = 1.0;
    double rold = 0, rho = 0;
    double complex root[2] = {0, 0}, prv[2] = {0, 0};
    int ntry = 1;
    double v1v1, v1v0, v2v2, v2v0, v2v1, v3v3, v3v1, v3v2;
#define APPROX_JAC(vout, vin, vdotv) do { \
        double temp1 = scale / sqrt(vdotv); \
        for (int q = 0; q < n; ++q) R->vtemp[q] = R->y[q] + temp1 * (vin)[q]; \
        R->f(R->ctx, R->t, R->vtemp, (vout)); R->f_count++; \
        double fac = R->h_average / temp1; \
        for (int q = 0; q < n; ++q) (vout)[q] = fac * ((vout)[q] - R->yp[q]); \
    } while (0)
#define DOMINANT(a11, a10, a00, resflag) do { \
        double ratio = (a10) / (a00); rho = fabs(ratio); \
        double det = (a00) * (a11) - (a10) * (a10); double res = fabs(det / (a00)); \
        int big = det == 0.0 || (res <= fabs(a11) * 1e-6 && fabs(ratio - rold) <= 0.001 * rho); \
        if (big) { root[0] = ratio; root[1] = 0.0; } \
        rold = ratio; resflag = big; \
    } while (0)
    for (;;) {
        int dom;
        APPROX_JAC(v1, v0, v0v0);
        v1v1 = wip(R, v1, v1);
        if (sqrt(v1v1) > 1.0e10 * sqrt(v0v0)) return 0;
        v1v0 = wip(R, v1, v0);
        if (ntry == 1) {
            rold = v1v0 / v0v0;
            if (fabs(rold) < R->cubrmc) return 0;
        } else {
            DOMINANT(v1v1, v1v0, v0v0, dom);
            if (dom) break;
        }
        APPROX_JAC(v2, v1, v1v1);
        v2v2 = wip(R, v2, v2); v2v0 = wip(R, v2, v0); v2v1 = wip(R, v2, v1);
        DOMINANT(v2v2, v2v1, v1v1, dom);
        if (dom) break;
        double det1 = v0v0 * v1v1 - v1v0 * v1v0;
        double alpha1 = (-v0v0 * v2v1 + v1v0 * v2v0) / det1;
        double beta1 = (v1v0 * v2v1 - v1v1 * v2v0) / det1;
        APPROX_JAC(v3, v2, v2v2);
        v3v3 = wip(R, v3, v3); v3v1 = wip(R, v3, v1); v3v2 = wip(R, v3, v2);
        DOMINANT(v3v3, v3v2, v2v2, dom);
        if (dom) break;
        double det2 = v1v1 * v2v2 - v2v1 * v2v1;
        double alpha2 = (-v1v1 * v3v2 + v2v1 * v3v1) / det2;
        double beta2 = (v2v1 * v3v2 - v2v2 * v3v1) / det2;
        double res2 = fabs(v3v3 + alpha2 * v3v2 + beta2 * v3v1 + alpha2 * v3v2 + alpha2 * alpha2 * v2v2
                           + alpha2 * beta2 * v2v1 + beta2 * v3v1 + beta2 * alpha2 * v2v1 + beta2 * beta2 * v1v1);
        if (res2 <= fabs(v3v3) * 1e-6) {
            quad_roots(alpha1, beta1, prv);
            quad_roots(alpha2, beta2, root);
            rho = cabs(prv[0]);
            double dist = fmin(cabs(root[0] - prv[0]), cabs(root[0] - prv[1]));
            if (dist <= 0.001 * rho) break;
        }
        ntry++;
        if (ntry > R->max_stiff_iters) return 0;
        double v3nrm = sqrt(v3v3);
        for (int q = 0; q < n; ++q) v0[q] = v3[q] / v3nrm;
        v0v0 = 1.0;
    }
#undef APPROX_JAC
#undef DOMINANT
    int sure = 0;
    if (creal(root[0]) < 0.0) {
        if (!(cabs(root[1]) >= 0.9 * rho && creal(root[1]) > 0.0)) {
            if (fabs(cimag(root[0])) <= fabs(creal(root[0])) * R->tan_angle)
                sure = rho >= 0.9 * R->stability_radius;
        }
    }
    return sure;
}

/* STEP_INTEGRATE: returns flag 1 (step taken), 3 (too much work, no step),
 * 4 (stiff, no step), 5 (step size too small), 911 (fatal). */
static int rk_step_integrate(or_rk* R)
{
    int n = R->neq;
    int ier = RK_OK;
    double hmin = 0;
    if (R->at_t_start) {
        R->f(R->ctx, R->t, R->y, R->yp);
        R->f_count++;
        vmax_abs(n, R->y, R->thresh, R->weights);
        /* phase 1: h_start == 0 always on this path */
        R->phase2 = 1;
        R->h = fabs(R->h);
        double ypnorm = 0.0;
        int any = 0;
        double mx = 0.0;
        for (int q = 0; q < n; ++q) {
            if (R->y[q] == 0.0) continue;
            double v = fabs(R->yp[q]) / R->weights[q];
            mx = any ? fmax(mx, v) : v;
            any = 1;
        }
        ypnorm = fmax(0.0, any ? mx : -DBL_MAX);
        double tau = or_root5(R->tol);
        if (R->h * ypnorm > tau) R->h = tau / ypnorm;
        hmin = fmax(R->sqtiny, R->toosml * fmax(fabs(R->t_start), fabs(R->t_end)));
        R->h = R->dir * fmax(R->h, hmin);
    } else if (R->at_t_end) {
        return RK_FATAL;
    }
    int phase3 = 1;
    int failed = 0;
    for (;;) {                                            /* take_step */
        R->h = copysign(fabs(R->h), R->dir);
        R->at_t_end = R->dir * ((R->t + R->h) - R->t_end) >= 0.0;
        if (R->at_t_end) R->h = R->t_end - R->t;
        else if (R->dir * ((R->t + 2.0 * R->h) - R->t_end) >= 0.0) R->h = (R->t_end - R->t) / 2.0;
        hmin = fmax(R->sqtiny, R->toosml * fmax(fabs(R->t), fabs(R->t + R->h)));
        if (fabs(R->h) < hmin) { ier = 5; break; }
        if (R->chkeff) {
            R->hit_t_end_count++;
            if (R->hit_t_end_count >= 100 && R->hit_t_end_count >= R->step_count / 3) {
                ier = 2; R->hit_t_end_count = 0; break;
            }
        }
        if (!failed) {
            int toomch = R->f_count > 5000;
            if (toomch) {
                ier = 3;
                R->full_f_count += R->f_count;
                R->f_count = 0;
            }
            if (rk_stiff(R, toomch)) ier = 4;
            if (ier != RK_OK) break;
        }
        double htry = R->h;
        double err = rk_step(R, R->t, &htry, hmin);
        R->h = htry;
        double alpha;
        if (err > R->tol) {
            if (R->at_t_start) { phase3 = 0; alpha = R->rs1; }
            else {
                R->bad_step_count++;
                R->stiff_bad_step_count++;
                if (failed) alpha = R->rs1;
                else { alpha = R->safety * or_root5(R->tol / err); alpha = fmax(alpha, R->rs1); }
            }
            R->h = alpha * R->h; failed = 1;
            continue;
        }
        double beta = or_root5(err / R->tol);
        if (!R->at_t_start) {
            double t1 = or_root5(err) / R->h;
            double t2 = or_root5(R->errold) / R->h_old;
            if (t1 < t2 * 100.0 && t2 < t1 * 100.0) beta = beta * (t1 / t2);
        }
        alpha = R->rs3;
        if (R->safety < beta * alpha) alpha = R->safety / beta;
        if (R->at_t_start) {
            R->phase2 = 0;
            phase3 = phase3 && !R->at_t_end && (alpha > R->rs2);
            if (phase3) { R->h = alpha * R->h; continue; }
        }
        alpha = fmin(alpha, R->rs);
        if (failed) alpha = fmin(alpha, 1.0);
        alpha = fmax(alpha, R->rs1);
        R->h_old = R->h; R->h = alpha * R->h;
        if (R->at_t_start) R->h_average = R->h_old;
        else R->h_average = 0.9 * R->h_average + 0.1 * R->h_old;
        R->at_t_start = 0; R->errold = err; R->t_old = R->t;
        if (R->at_t_end) R->t = R->t_end; else R->t = R->t + R->h_old;
        R->step_count++;
        /* advance: y_old <- y, y <- y_new, yp_old <- yp, yp <- stage 8 */
        double* tmp = R->y_old; R->y_old = R->y; R->y = R->y_new; R->y_new = tmp;
        tmp = R->yp_old; R->yp_old = R->yp; R->yp = R->stg[8]; R->stg[8] = tmp;
        if (R->renorm) rk_renorm(R, R->y);
        break;
    }
    if (ier < RK_FATAL) {
        R->at_t_end = R->t == R->t_end;
        R->chkeff = R->at_t_end;
        for (int q = 0; q < n; ++q) R->ymax[q] = fmax(fabs(R->y[q]), R->ymax[q]);
        if (ier == RK_OK) R->intrp_ready = 0;
    }
    R->last_step_flag = ier;
    return ier;
}

/* INTERPOLATE (task 'R'): value of the 6th-degree interpolant at t_want */
static void rk_interpolate(or_rk* R, double t_want, double* y_want)
{
    const bs45_tab* T = &R->T;
    int n = R->neq;
    if (!R->intrp_ready) {
        /* extra stages 9, 10, 11 from the data of the last step */
        for (int i = 9; i <= 11; ++i) {
            double* yt = R->ytemp;
            for (int q = 0; q < n; ++q) yt[q] = T->a[i][1] * R->yp_old[q];
            for (int j = 2; j <= i - 1; ++j) {
                const double* s = (j == 8) ? R->yp : R->stg[j];
                for (int q = 0; q < n; ++q) yt[q] = yt[q] + T->a[i][j] * s[q];
            }
            for (int q = 0; q < n; ++q) yt[q] = R->y_old[q] + R->h_old * yt[q];
            R->f(R->ctx, R->t_old + T->c[i] * R->h_old, yt, R->stg[i]);
            R->f_count++;
        }
        double (*r)[7] = (double (*)[7])T->r;
        const double *k1 = R->yp_old, *k3 = R->stg[3], *k4 = R->stg[4], *k5 = R->stg[5], *k6 = R->stg[6],
                     *k7 = R->stg[7], *k8 = R->yp, *k9 = R->stg[9], *k10 = R->stg[10], *k11 = R->stg[11];
        for (int q = 0; q < n; ++q) {
            double p5 = r[5][6] * k5[q] + ((r[10][6] * k10[q] + r[8][6] * k8[q]) + (r[7][6] * k7[q] + r[6][6] * k6[q]))
                      + ((r[4][6] * k4[q] + r[9][6] * k9[q]) + (r[3][6] * k3[q] + r[11][6] * k11[q]) + r[1][6] * k1[q]);
            double p4 = (r[10][5] * k10[q] + r[9][5] * k9[q]) + ((r[7][5] * k7[q] + r[6][5] * k6[q]) + r[5][5] * k5[q])
                      + ((r[4][5] * k4[q] + r[8][5] * k8[q]) + (r[3][5] * k3[q] + r[11][5] * k11[q]) + r[1][5] * k1[q]);
            double p3 = ((r[4][4] * k4[q] + r[8][4] * k8[q]) + (r[7][4] * k7[q] + r[6][4] * k6[q]) + r[5][4] * k5[q])
                      + ((r[10][4] * k10[q] + r[9][4] * k9[q]) + (r[3][4] * k3[q] + r[11][4] * k11[q]) + r[1][4] * k1[q]);
            double p2 = r[5][3] * k5[q] + r[6][3] * k6[q]
                      + ((r[3][3] * k3[q] + r[9][3] * k9[q]) + (r[10][3] * k10[q] + r[8][3] * k8[q]) + r[1][3] * k1[q])
                      + ((r[4][3] * k4[q] + r[11][3] * k11[q]) + r[7][3] * k7[q]);
            double p1 = r[5][2] * k5[q] + ((r[6][2] * k6[q] + r[8][2] * k8[q]) + r[1][2] * k1[q])
                      + ((r[3][2] * k3[q] + r[9][2] * k9[q]) + r[10][2] * k10[q])
                      + ((r[4][2] * k4[q] + r[11][2] * k11[q]) + r[7][2] * k7[q]);
            R->p[5][q] = R->h_old * p5; R->p[4][q] = R->h_old * p4; R->p[3][q] = R->h_old * p3;
            R->p[2][q] = R->h_old * p2; R->p[1][q] = R->h_old * p1;
        }
        R->intrp_ready = 1;
    }
    double sigma = (t_want - R->t) / R->h_old;
    for (int q = 0; q < n; ++q) {
        double v = R->p[5][q] * sigma;
        v = (v + R->p[4][q]) * sigma;
        v = (v + R->p[3][q]) * sigma;
        v = (v + R->p[2][q]) * sigma;
        v = (v + R->p[1][q]) * sigma;
        y_want[q] = (v + R->h_old * R->yp[q]) * sigma + R->y[q];
    }
}

/* RANGE_INTEGRATE: returns the step flag that ended the call (1 normal). */
static int rk_range_integrate(or_rk* R, double t_want, double* t_got, double* y_got)
{
    if (R->at_t_start) {
        R->range_t_end = R->t_end;
        R->tlast = R->t_start;
        *t_got = R->t_start;
        R->h = fmin(fabs(R->h), fabs(t_want - R->t_start));
        double hmin = fmax(R->sqtiny, R->toosml * fmax(fabs(R->t_start), fabs(R->t_end)));
        R->h = fmax(R->h, hmin);
    } else if (R->tlast == R->range_t_end) {
        return RK_FATAL;
    }
    if (R->dir * (t_want - R->tlast) <= 0.0) return RK_FATAL;
    if (R->dir * (t_want - R->range_t_end) > 0.0) return RK_FATAL;
    int flag = RK_OK;
    for (;;) {
        if (R->dir * (R->t - t_want) >= 0.0) {
            rk_interpolate(R, t_want, y_got);
            *t_got = t_want;
            break;
        }
        flag = rk_step_integrate(R);
        if (flag == RK_OK) continue;
        if (flag >= RK_FATAL) return flag;
        *t_got = R->t;
        memcpy(y_got, R->y, sizeof(double) * (size_t)R->neq);
        break;
    }
    R->tlast = *t_got;
    return flag;
}

typedef struct {
    long f_evals;        /* total RHS evaluations */
    long steps;          /* accepted steps */
    long bad_steps;      /* rejected steps after the first */
    long n_flag3, n_flag4;
    long n_out;          /* stored output samples */
    int status;          /* 0 ok, <0 setup error, 911 fatal, 5 step too small */
    int converged_at;    /* output index where the t_conv criterion stopped the run, or -1 */
} or_stats;

/* MagTense_ODE_RKSuite: output-time driver.  y_out is [nt][neq]; flags_out[k]
 * records the flag of the range_integrate call that produced sample k. */
static int cmp_dbl(const void* a, const void* b)
{
    double x = *(const double*)a, y = *(const double*)b;
    return (x > y) - (x < y);
}

int or_solve_generic(or_rhs_fn f, void* ctx, int neq, int ncell, int renorm,
                     const double* t, int nt, const double* y0, double tol, double thres_value,
                     const double* t_conv, int nt_conv, double conv_tol,
                     double* t_out, double* y_out, int* flags_out, or_stats* st)
{
    memset(st, 0, sizeof(*st));
    st->converged_at = -1;
    double* thresh = (double*)malloc(sizeof(double) * neq);
    for (int q = 0; q < neq; ++q) thresh[q] = thres_value;
    or_rk R;
    int rc = rk_setup(&R, f, ctx, neq, t[0], y0, t[nt - 1], tol, thresh);
    free(thresh);
    if (rc != 0) { st->status = rc; rk_free(&R); return rc; }
    R.renorm = renorm; R.ncell = ncell;
    /* unique (first occurrence) then ascending sort */
    int ncomb = nt + nt_conv;
    double* comb = (double*)malloc(sizeof(double) * ncomb);
    int k = 0;
    for (int i = 0; i < ncomb; ++i) {
        double v = (i < nt) ? t[i] : t_conv[i - nt];
        /* simple_unique compares against its zero-initialised output array, so a
           0.0 after the first position always counts as a duplicate */
        int dup = (v == 0.0);
        for (int q = 0; q < k; ++q) if (comb[q] == v) { dup = 1; break; }
        if (i == 0 || !dup) comb[k++] = v;
    }
    qsort(comb, k, sizeof(double), cmp_dbl);
    double* y_last = (double*)malloc(sizeof(double) * neq);
    double* y_step = (double*)malloc(sizeof(double) * neq);
    memcpy(y_last, y0, sizeof(double) * neq);
    t_out[0] = t[0];
    memcpy(y_out, y0, sizeof(double) * neq);
    if (flags_out) flags_out[0] = 0;
    int ko = 1;
    int status = 0;
    for (int i = 1; i < k; ++i) {
        double t_step;
        int flag = rk_range_integrate(&R, comb[i], &t_step, y_step);
        if (flag >= RK_FATAL) { status = flag; break; }
        if (flag == 3) st->n_flag3++;
        if (flag == 4) st->n_flag4++;
        if (flag == 5 || flag == 2) { status = flag; }
        int in_conv = 0, in_t = 0;
        for (int q = 0; q < nt_conv; ++q) if (t_conv[q] == comb[i]) { in_conv = 1; break; }
        if (in_conv) {
            double ce = 0.0;
            for (int q = 0; q < neq; ++q) ce = fmax(ce, fabs(y_step[q] - y_last[q]));
            if (ce < conv_tol) {
                if (ko < nt) {
                    memcpy(y_out + (size_t)ko * neq, y_step, sizeof(double) * neq);
                    t_out[ko] = t_step;
                    if (flags_out) flags_out[ko] = flag;
                }
                st->converged_at = ko;
                break;
            }
            memcpy(y_last, y_step, sizeof(double) * neq);
        }
        for (int q = 0; q < nt; ++q) if (t[q] == comb[i]) { in_t = 1; break; }
        if (in_t && ko < nt) {
            memcpy(y_out + (size_t)ko * neq, y_step, sizeof(double) * neq);
            t_out[ko] = t_step;
            if (flags_out) flags_out[ko] = flag;
            ko++;
        }
        if (status) break;
    }
    st->n_out = ko;
    st->f_evals = R.full_f_count + R.f_count;
    st->steps = R.step_count;
    st->bad_steps = R.bad_step_count;
    st->status = status;
    free(comb); free(y_last); free(y_step);
    rk_free(&R);
    return status;
}

static void rhs_adapter(void* ctx, double t, const double* y, double* f) { or_rhs((or_problem*)ctx, t, y, f); }

int or_solve(or_problem* p, const double* t, int nt, const double* y0, double tol, double thres,
             const double* t_conv, int nt_conv, double conv_tol,
             double* t_out, double* y_out, int* flags_out, or_stats* st)
{
    return or_solve_generic(rhs_adapter, p, 3 * p->n, p->n, p->renorm, t, nt, y0, tol, thres,
                            t_conv, nt_conv, conv_tol, t_out, y_out, flags_out, st);
}

/* Linear test problem y' = lam * y (used to check the integrator alone). */
typedef struct { int n; const double* lam; } or_linear_ctx;
static void linear_rhs(void* c, double t, const double* y, double* f)
{
    (void)t;
    const or_linear_ctx* L = (const or_linear_ctx*)c;
    for (int i = 0; i < L->n; ++i) f[i] = L->lam[i] * y[i];
}
int or_solve_linear(int neq, const double* lam, const double* t, int nt, const double* y0, double tol,
                    double thres, double* t_out, double* y_out, int* flags_out, or_stats* st)
{
    or_linear_ctx L = {neq, lam};
    double tc = 0.0;
    return or_solve_generic(linear_rhs, &L, neq, neq, 0, t, nt, y0, tol, thres, &tc, 1, 1e-4,
                            t_out, y_out, flags_out, st);
}

int or_stats_size(void) { return (int)sizeof(or_stats); }

/* Demag field (the reference's internal H = -Ms K m) at a subset of receivers,
 * given their tensor rows K[c][r][j] (as written by or_assemble with the same
 * row list).  mode 0: FP32 rows and FP32 product (reference order); mode 1: FP64. */
void or_demag_rows(const float* K32, const double* K64, int nrows, int n, const double* m,
                   const double* Ms_rows, int mode, double* Hout /* [3][nrows] */)
{
    static const int blk[3][3] = {{0, 1, 2}, {1, 3, 4}, {2, 4, 5}};
    float* ms = (float*)malloc(sizeof(float) * 3 * (size_t)n);
    for (int i = 0; i < 3 * n; ++i) ms[i] = (float)m[i];
#pragma omp parallel for schedule(static)
    for (int r = 0; r < nrows; ++r) {
        for (int a = 0; a < 3; ++a) {
            if (mode == 0) {
                float acc = 0.0f;
                for (int b = 0; b < 3; ++b) {
                    const float* row = K32 + ((size_t)blk[a][b] * nrows + r) * (size_t)n;
                    const float* xb = ms + (size_t)b * n;
                    for (int j = 0; j < n; ++j) { float tmp = -xb[j]; acc = acc + tmp * row[j]; }
                }
                float hm = acc * (float)Ms_rows[r];
                Hout[(size_t)a * nrows + r] = (double)hm;
            } else {
                double acc = 0.0;
                for (int b = 0; b < 3; ++b) {
                    const double* row = K64 + ((size_t)blk[a][b] * nrows + r) * (size_t)n;
                    const double* xb = m + (size_t)b * n;
                    for (int j = 0; j < n; ++j) acc = acc + (-xb[j]) * row[j];
                }
                Hout[(size_t)a * nrows + r] = acc * (double)(float)Ms_rows[r];
            }
        }
    }
    free(ms);
}

/* ------------------------------------------------------------------ */
/* thresholded-sparse demag                                            */
/* ------------------------------------------------------------------ */
/* FindThresholdFraction (DemagAuxFunctions.f90:353-428) as ApplyThresholdDense
 * (:20-122) calls it: on the positive entries of the six blocks (K32[c][i][j],
 * masks K > 0 at :45-50), bisection in single precision between the smallest and
 * the largest of them; a step counts the positive entries <= f_middle, moves the
 * upper end when that count exceeds frac * (their number) and the lower end
 * otherwise, and stops when the count lies within (frac -+ 0.01) * number, the
 * literal 0.01 being a double in the 8-byte-real build; at most 1000 steps;
 * frac >= 1 returns huge(). */
float or_threshold_fraction(const float* K32, int n, float frac)
{
    if (frac >= 1.0f) return FLT_MAX;
    const size_t tot = (size_t)6 * n * n;
    long long n_pos = 0;
    float f_small = FLT_MAX, f_large = 0.0f;
    for (size_t e = 0; e < tot; ++e) {
        const float v = K32[e];
        if (v > 0.0f) {
            n_pos++;
            if (v < f_small) f_small = v;
            if (v > f_large) f_large = v;
        }
    }
    if (n_pos == 0) return 0.0f;
    float f_middle = f_small;
    for (int k_do = 1;; ++k_do) {
        f_middle = (f_large - f_small) / 2.0f + f_small;
        long long count_middle = 0;
#pragma omp parallel for reduction(+ : count_middle) schedule(static)
        for (long long e = 0; e < (long long)tot; ++e) {
            const float v = K32[e];
            if (v > 0.0f && v <= f_middle) count_middle++;
        }
        if ((float)count_middle > frac * (float)n_pos) f_large = f_middle;
        else f_small = f_middle;
        const double c = (double)count_middle, np = (double)n_pos;
        if (c >= ((double)frac - 0.01) * np && c <= ((double)frac + 0.01) * np) break;
        if (k_do > 1000) break;
    }
    return f_middle;
}

/* Keep only the entries with |K| > thr (ConvertDenseToSparse_s, util_micromag.f90:98)
 * in the FP32 product of mode 0: the dropped entries are zeroed in the column copy,
 * which leaves every remaining term and its order unchanged.  Returns the kept
 * entries of the six blocks. */
long long or_problem_set_threshold(or_problem* p, float thr)
{
    if (!p->KT32) return -1;
    const size_t tot = (size_t)6 * p->n * p->n;
    long long kept = 0;
    for (size_t e = 0; e < tot; ++e) {
        if (fabsf(p->KT32[e]) > thr) kept++;
        else p->KT32[e] = 0.0f;
    }
    return kept;
}
