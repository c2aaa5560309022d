// Boundary-element (DPCM / IEFPCM) model on the device.
//
// Reference: src/bem/bem_module.f90 (create_tesserae :420-491,
// construct_constant_matrix_bem :678-782, construct_dynamic_field_rhs_bem
// :788-873, construct_dynamic_matrix_bem :881-933,
// new_gmres_diagonal_shift_bem :977-997) and
// src/bem/accurate_green_function.f90 (polar Gauss-Lobatto diagonal integrals,
// 28-point Strang-Fix near off-diagonals, near-element selection, the -2 pi
// closure of the diagonal).
//
// The Green-function derivative D (n x n) is stored transposed, d_T[j][i] =
// D(i,j): the few-column and tiled FP64 contractions compute X^T d_T = (D X)^T,
// which is the operator's D x for every column; the tensor-core split
// transposes it back when it is built.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "plx_internal.h"

namespace plx {

namespace {

constexpr double kDiagParam = 1.0694;
constexpr double kTwoPi = 6.283185307179586476925286766559;
constexpr double kFourPi = 12.566370614359172953850573533118;

// Strang & Fix 28-point rule on the unit triangle (barycentric x, y, weight);
// the rule of accurate_green_function.f90:138-238.
__constant__ double c_sf[28][3] = {
    {0.3333333333333333, 0.3333333333333333, 0.08797730116222190},
    {0.9480217181434233, 0.02598914092828833, 0.008744311553736190},
    {0.02598914092828833, 0.9480217181434233, 0.008744311553736190},
    {0.02598914092828833, 0.02598914092828833, 0.008744311553736190},
    {0.8114249947041546, 0.09428750264792270, 0.03808157199393533},
    {0.09428750264792270, 0.8114249947041546, 0.03808157199393533},
    {0.09428750264792270, 0.09428750264792270, 0.03808157199393533},
    {0.01072644996557060, 0.4946367750172147, 0.01885544805613125},
    {0.4946367750172147, 0.01072644996557060, 0.01885544805613125},
    {0.4946367750172147, 0.4946367750172147, 0.01885544805613125},
    {0.5853132347709715, 0.2073433826145142, 0.07215969754474100},
    {0.2073433826145142, 0.5853132347709715, 0.07215969754474100},
    {0.2073433826145142, 0.2073433826145142, 0.07215969754474100},
    {0.1221843885990187, 0.4389078057004907, 0.06932913870553720},
    {0.4389078057004907, 0.1221843885990187, 0.06932913870553720},
    {0.4389078057004907, 0.4389078057004907, 0.06932913870553720},
    {0.6779376548825902, 0.04484167758913055, 0.04105631542928860},
    {0.6779376548825902, 0.27722066752827925, 0.04105631542928860},
    {0.04484167758913055, 0.6779376548825902, 0.04105631542928860},
    {0.04484167758913055, 0.27722066752827925, 0.04105631542928860},
    {0.27722066752827925, 0.6779376548825902, 0.04105631542928860},
    {0.27722066752827925, 0.04484167758913055, 0.04105631542928860},
    {0.8588702812826364, 0.0, 0.007362383783300573},
    {0.8588702812826364, 0.1411297187173636, 0.007362383783300573},
    {0.0, 0.8588702812826364, 0.007362383783300573},
    {0.0, 0.1411297187173636, 0.007362383783300573},
    {0.1411297187173636, 0.8588702812826364, 0.007362383783300573},
    {0.1411297187173636, 0.0, 0.007362383783300573}};

// Tessera geometry: centroid, area, normal, tangents, circumradius (bohr).
// tri: [n][3 vertices][3].  Outputs: pos [4][n] (x, y, z, area),
// frame [9][n] (normal, tangent 1, tangent 2), rad [n].
__global__ void tess_kernel(int n, double nfac, const double *__restrict__ tri, double *__restrict__ pos,
                            double *__restrict__ frame, double *__restrict__ rad) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double *v = tri + 9LL * i;
    double c[3], a[3], b[3], cr[3];
    for (int k = 0; k < 3; ++k) {
        c[k] = (v[k] + v[3 + k] + v[6 + k]) / 3.0;
        a[k] = v[3 + k] - v[k];
        b[k] = v[6 + k] - v[k];
    }
    cr[0] = a[1] * b[2] - a[2] * b[1];
    cr[1] = a[2] * b[0] - a[0] * b[2];
    cr[2] = a[0] * b[1] - a[1] * b[0];
    double na = sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
    double nc = sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
    double nrm[3], t1[3], t2[3];
    for (int k = 0; k < 3; ++k) {
        nrm[k] = nfac * cr[k] / nc;
        t1[k] = -a[k] / na;
    }
    t2[0] = nrm[1] * t1[2] - nrm[2] * t1[1];
    t2[1] = nrm[2] * t1[0] - nrm[0] * t1[2];
    t2[2] = nrm[0] * t1[1] - nrm[1] * t1[0];
    for (int k = 0; k < 3; ++k) {
        pos[(int64_t)k * n + i] = c[k];
        frame[(int64_t)k * n + i] = nrm[k];
        frame[(int64_t)(3 + k) * n + i] = t1[k];
        frame[(int64_t)(6 + k) * n + i] = t2[k];
    }
    pos[3LL * n + i] = nc / 2.0;
    double r = 0.0;
    for (int p = 0; p < 3; ++p) {
        double dx = c[0] - v[3 * p], dy = c[1] - v[3 * p + 1], dz = c[2] - v[3 * p + 2];
        r = fmax(r, sqrt(dx * dx + dy * dy + dz * dz));
    }
    rad[i] = r;
}

// Accurate diagonal before the closure: g_i = n (sum_n) + t1 (sum_t1) + t2 (sum_t2)
// over the polar rule around the centroid; gvec [3][n], dpre [n] = -(g . n).
// rule: [np][3] (barycentric x, y, weight); dmax4 = 1e-4 of the largest
// centroid-to-point distance (replaces distances below 1e-4 in the tangential sums).
__global__ void bem_diag_kernel(int n, int np, const double *__restrict__ rule, const double *__restrict__ tri,
                                const double *__restrict__ pos, const double *__restrict__ frame, double dmax4,
                                double *__restrict__ gvec, double *__restrict__ dpre) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double *v = tri + 9LL * i;
    double c[3] = {pos[i], pos[n + i], pos[2LL * n + i]};
    double a = pos[3LL * n + i];
    double fr[9];
    for (int k = 0; k < 9; ++k) fr[k] = frame[(int64_t)k * n + i];
    double sn = 0.0, s1 = 0.0, s2 = 0.0;
    for (int p = 0; p < np; ++p) {
        double x = rule[3 * p], y = rule[3 * p + 1], w = rule[3 * p + 2], z = 1.0 - x - y;
        double vec[3];
        for (int k = 0; k < 3; ++k) vec[k] = c[k] - ((x * v[k] + y * v[3 + k]) + z * v[6 + k]);
        double d = sqrt(vec[0] * vec[0] + vec[1] * vec[1] + vec[2] * vec[2]);
        double d3 = d * d * d;
        sn -= w * a * (vec[0] * fr[0] + vec[1] * fr[1] + vec[2] * fr[2]) / d3;
        if (d < 1.0e-4) d = dmax4;
        d3 = d * d * d;
        s1 -= w * a * (vec[0] * fr[3] + vec[1] * fr[4] + vec[2] * fr[5]) / d3;
        s2 -= w * a * (vec[0] * fr[6] + vec[1] * fr[7] + vec[2] * fr[8]) / d3;
    }
    double g[3];
    for (int k = 0; k < 3; ++k) {
        g[k] = fr[k] * sn + fr[3 + k] * s1 + fr[6 + k] * s2;
        gvec[(int64_t)k * n + i] = g[k];
    }
    dpre[i] = -(g[0] * fr[0] + g[1] * fr[1] + g[2] * fr[2]);
}

// Largest distance from a centroid to its polar-rule points (for dmax4).
__global__ void bem_polar_dmax(int n, int np, const double *__restrict__ rule, const double *__restrict__ tri,
                               const double *__restrict__ pos, unsigned long long *__restrict__ dmax_bits) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double *v = tri + 9LL * i;
    double c[3] = {pos[i], pos[n + i], pos[2LL * n + i]};
    double m = 0.0;
    for (int p = 0; p < np; ++p) {
        double x = rule[3 * p], y = rule[3 * p + 1], z = 1.0 - x - y;
        double s = 0.0;
        for (int k = 0; k < 3; ++k) {
            double d = c[k] - ((x * v[k] + y * v[3 + k]) + z * v[6 + k]);
            s += d * d;
        }
        m = fmax(m, sqrt(s));
    }
    // non-negative doubles order like their bit patterns
    atomicMax(dmax_bits, (unsigned long long)__double_as_longlong(m));
}

// d_T[j][i] = D(i, j).  One thread per (i, j).
__global__ void bem_matrix_kernel(int n, int accurate, double sphere_r, const double *__restrict__ tri,
                                  const double *__restrict__ pos, const double *__restrict__ frame,
                                  const double *__restrict__ rad, const double *__restrict__ dpre,
                                  double *__restrict__ Dt) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int j = blockIdx.y;
    if (i >= n) return;
    double xi = pos[i], yi = pos[n + i], zi = pos[2LL * n + i];
    double nx = frame[i], ny = frame[n + i], nz = frame[2LL * n + i];
    double aj = pos[3LL * n + j];
    double dx = xi - pos[j], dy = yi - pos[n + j], dz = zi - pos[2LL * n + j];
    double r = sqrt(dx * dx + dy * dy + dz * dz);
    double d;
    bool near = false;
    if (accurate) {
        // selection_of_refined_elements: |c_i - c_j| (from the expanded form) - radius_j < 0
        double ni = xi * xi + yi * yi + zi * zi;
        double nj = pos[j] * pos[j] + pos[n + j] * pos[n + j] + pos[2LL * n + j] * pos[2LL * n + j];
        double pr = 2.0 * (xi * pos[j] + yi * pos[n + j] + zi * pos[2LL * n + j]);
        double t = ni + nj - pr;
        if (t < 1.0e-10) t = 0.0;
        near = sqrt(t) - rad[j] < 0.0;
    }
    if (i == j) {
        d = accurate ? dpre[i] : kDiagParam * sqrt(kFourPi * aj) / (2.0 * sphere_r);
    } else if (near) {
        const double *v = tri + 9LL * j;
        double ox = 0.0, oy = 0.0, oz = 0.0;
        for (int p = 0; p < 28; ++p) {
            double x = c_sf[p][0], y = c_sf[p][1], w = c_sf[p][2], z = 1.0 - x - y;
            double tx = xi - ((x * v[0] + y * v[3]) + z * v[6]);
            double ty = yi - ((x * v[1] + y * v[4]) + z * v[7]);
            double tz = zi - ((x * v[2] + y * v[5]) + z * v[8]);
            double nn = sqrt(tx * tx + ty * ty + tz * tz);
            double n3 = nn * nn * nn;
            ox -= w * aj * tx / n3;
            oy -= w * aj * ty / n3;
            oz -= w * aj * tz / n3;
        }
        d = -(ox * nx + oy * ny + oz * nz);
    } else {
        d = aj * (dx * nx + dy * ny + dz * nz) / (r * r * r);
    }
    Dt[(int64_t)j * n + i] = d;
}

// Closure of the accurate diagonal (final_refinement_green_function):
// colsum_i = sum_r D(r, i) a_r / a_i (= sum over row i of d_T), then
// g_i += n_i (-2 pi + colsum_i), D_ii = -(g_i . n_i).  One warp per i.
__global__ void bem_closure_kernel(int n, const double *__restrict__ pos, const double *__restrict__ frame,
                                   double *__restrict__ gvec, double *__restrict__ Dt) {
    int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    if (i >= n) return;
    const double *row = Dt + (int64_t)i * n;
    double ai = pos[3LL * n + i];
    double s = 0.0;
    for (int r = lane; r < n; r += 32) s += row[r] / ai * pos[3LL * n + r];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) {
        double g[3], nr[3];
        for (int k = 0; k < 3; ++k) {
            nr[k] = frame[(int64_t)k * n + i];
            g[k] = nr[k] * (-kTwoPi + s) + gvec[(int64_t)k * n + i];
            gvec[(int64_t)k * n + i] = g[k];
        }
        Dt[(int64_t)i * n + i] = -(g[0] * nr[0] + g[1] * nr[1] + g[2] * nr[2]);
    }
}

// S A^-1 of IEFPCM: M(i,j) = 1/r_ij, M(i,i) = 1.0694 sqrt(4 pi a_i) / a_i (symmetric).
__global__ void bem_sainv_kernel(int n, const double *__restrict__ pos, double *__restrict__ M) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int j = blockIdx.y;
    if (i >= n) return;
    double v;
    if (i == j) {
        double a = pos[3LL * n + i];
        v = kDiagParam * sqrt(kFourPi * a) * (1.0 / a);
    } else {
        double dx = pos[i] - pos[j], dy = pos[n + i] - pos[n + j], dz = pos[2LL * n + i] - pos[2LL * n + j];
        double r = sqrt(dx * dx + dy * dy + dz * dz);
        v = pos[3LL * n + j] / r * (1.0 / pos[3LL * n + j]);
    }
    M[(int64_t)j * n + i] = v;
}

// y = S + z(w) x for every column (the BEM GMRES operator: D x + shift).
__global__ void bem_rows(int n, int count, const int32_t *__restrict__ freq, const Cplx *__restrict__ zf,
                         const double *__restrict__ S, const double *__restrict__ X, double *__restrict__ Y) {
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    int c = blockIdx.y;
    if (r >= n || c >= count) return;
    Cplx z = zf[freq[c]];
    const double *s = S + (int64_t)c * 2 * n, *x = X + (int64_t)c * 2 * n;
    double xr = x[r], xi = x[n + r];
    Y[(int64_t)c * 2 * n + r] = s[r] + z.re * xr - z.im * xi;
    Y[(int64_t)c * 2 * n + n + r] = s[n + r] + z.re * xi + z.im * xr;
}

// Right-hand sides: DPCM b = -E0 n_p; IEFPCM v = -E0 r_p (the potential; the
// caller then forms -(2 pi I + D_before_closure) v).
__global__ void bem_rhs_kernel(int n, int count, int ief, const int32_t *__restrict__ pol, double e0,
                               const double *__restrict__ pos, const double *__restrict__ frame,
                               double *__restrict__ B) {
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    int c = blockIdx.y;
    if (r >= n || c >= count) return;
    int p = pol[c];
    double v = ief ? -e0 * pos[(int64_t)p * n + r] : -e0 * frame[(int64_t)p * n + r];
    B[(int64_t)c * 2 * n + r] = v;
    B[(int64_t)c * 2 * n + n + r] = 0.0;
}

// b = D_after v + (dpre_ii - D_after,ii - 2 pi) v_i, i.e. (D_before - 2 pi I) v.
__global__ void bem_ief_fix(int n, int count, const double *__restrict__ dpre, const double *__restrict__ Dt,
                            const double *__restrict__ V, double *__restrict__ B) {
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    int c = blockIdx.y;
    if (r >= n || c >= count) return;
    double corr = dpre[r] - Dt[(int64_t)r * n + r] - kTwoPi;
    for (int part = 0; part < 2; ++part) {
        int64_t k = (int64_t)c * 2 * n + (int64_t)part * n + r;
        B[k] += corr * V[k];
    }
}

// Column-major A(w) for the direct solve: DPCM D + z I; IEFPCM -(DM + z M).
__global__ void bem_assemble(int n, int ief, Cplx z, const double *__restrict__ Dt, const double *__restrict__ DM,
                             const double *__restrict__ M, double2 *__restrict__ A) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int j = blockIdx.y;
    if (i >= n) return;
    int64_t k = (int64_t)j * n + i;
    double re, im;
    if (!ief) {
        re = Dt[k] + (i == j ? z.re : 0.0);
        im = i == j ? z.im : 0.0;
    } else {
        re = -(DM[k] + z.re * M[k]);
        im = -(z.im * M[k]);
    }
    A[k] = make_double2(re, im);
}

// 1 / (D_ii + z(w)) for every column (Jacobi preconditioner of the refined solves).
__global__ void bem_diag_inverse_kernel(int n, int count, const int32_t *__restrict__ freq,
                                        const Cplx *__restrict__ zf, const double *__restrict__ Dt,
                                        double *__restrict__ P) {
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    int c = blockIdx.y;
    if (r >= n || c >= count) return;
    Cplx z = zf[freq[c]];
    double re = Dt[(int64_t)r * n + r] + z.re, im = z.im;
    double m = re * re + im * im;
    P[(int64_t)c * 2 * n + r] = m > 0.0 ? re / m : 1.0;
    P[(int64_t)c * 2 * n + n + r] = m > 0.0 ? -im / m : 0.0;
}

// Legendre-Gauss-Lobatto nodes and weights, the reference's Newton iteration
// on the Legendre-Vandermonde matrix (accurate_green_function.f90:361-434).
void lgl(int npol, std::vector<double> &x, std::vector<double> &w) {
    const double pi = 3.14159265358979323846;
    x.assign(npol, 0.0);
    w.assign(npol, 0.0);
    std::vector<double> xold(npol, 2.0), P((size_t)npol * npol, 0.0);
    for (int i = 0; i < npol; ++i) x[i] = std::cos(pi * i / (npol - 1));
    auto maxdiff = [&]() {
        double m = 0.0;
        for (int i = 0; i < npol; ++i) m = std::max(m, std::fabs(x[i] - xold[i]));
        return m;
    };
    double check = maxdiff();
    while (check > 2.2204e-16) {
        check = maxdiff();
        xold = x;
        for (int i = 0; i < npol; ++i) {
            P[i] = 1.0;
            P[i + npol] = x[i];
            for (int j = 2; j < npol; ++j)
                P[i + (size_t)j * npol] = ((2.0 * j - 1.0) * x[i] * P[i + (size_t)(j - 1) * npol] -
                                           (j - 1.0) * P[i + (size_t)(j - 2) * npol]) /
                                          j;
        }
        for (int i = 0; i < npol; ++i) {
            double pn = P[i + (size_t)(npol - 1) * npol], pm = P[i + (size_t)(npol - 2) * npol];
            x[i] = xold[i] - (x[i] * pn - pm) / (npol * pn);
        }
    }
    for (int i = 0; i < npol; ++i) {
        double pn = P[i + (size_t)(npol - 1) * npol];
        w[i] = 2.0 / (npol * (npol - 1.0) * pn * pn);
    }
}

// The 144-point polar rule of tesserae_integration_polar_coordinates
// (accurate_green_function.f90:245-356), as (x, y, weight) rows.
std::vector<double> polar_rule(int npol1 = 8, int npol2 = 6) {
    const double pi = 3.14159265358979323846;
    std::vector<double> p1, w1, p2, w2;
    lgl(npol1, p1, w1);
    lgl(npol2, p2, w2);
    const int nt = npol1 * npol2;
    std::vector<double> tphi(nt), trho(nt), tw(nt);
    for (int j = 0; j < npol2; ++j)
        for (int i = 0; i < npol1; ++i) {
            tphi[i + npol1 * j] = pi * (270.0 + 60.0 * p2[j]) / 180.0;
            trho[i + npol1 * j] = 0.5 * (p1[i] + 1.0 + 1.0e-06);
            tw[i + npol1 * j] = w1[i] * w2[j];
        }
    const double phi0 = (120.0 / 180.0) * pi;
    std::vector<double> rule((size_t)3 * nt * 3);
    double wsum = 0.0;
    for (int k = 0; k < 3; ++k)
        for (int t = 0; t < nt; ++t) {
            double s = std::fabs(2.0 * std::sin(tphi[t]));
            double tx = std::cos(tphi[t] + k * phi0) * trho[t] * 1.0 / s;
            double ty = std::sin(tphi[t] + k * phi0) * trho[t] * 1.0 / s;
            double wt = tw[t] * trho[t] * std::pow(std::fabs(1.0 / (2.0 * std::sin(tphi[t]))), 2.0);
            size_t e = (size_t)(t + k * nt);
            rule[3 * e] = (1.0 - std::sqrt(3.0) * tx - ty) / 3.0;
            rule[3 * e + 1] = (1.0 + std::sqrt(3.0) * tx - ty) / 3.0;
            rule[3 * e + 2] = wt;
            wsum += wt;
        }
    for (int e = 0; e < 3 * nt; ++e) rule[3 * e + 2] /= wsum;
    return rule;
}

}  // namespace

void build_bem(plx_geom *g, const double *tri_host, double normal_factor, double sphere_r, int accurate) {
    plx_ctx *ctx = g->ctx;
    cudaStream_t st = ctx->stream;
    const int n = g->n_var;
    DevArray<double> tri, rad;
    tri.alloc(ctx, 9LL * n);
    rad.alloc(ctx, n);
    PLX_CHECK_CUDA(cudaMemcpyAsync(tri.p, tri_host, 9LL * n * 8, cudaMemcpyHostToDevice, st));
    g->d_pos.alloc(ctx, 4LL * n);
    g->d_frame.alloc(ctx, 9LL * n);
    g->d_dpre.alloc(ctx, n);
    tess_kernel<<<n_blocks(n, 128), 128, 0, st>>>(n, normal_factor, tri.p, g->d_pos.p, g->d_frame.p, rad.p);
    ctx->launches++;
    DevArray<double> gvec;
    gvec.alloc(ctx, 3LL * n);
    if (accurate) {
        std::vector<double> rule = polar_rule();
        const int np = (int)(rule.size() / 3);
        DevArray<double> d_rule;
        DevArray<unsigned long long> dmax;
        d_rule.alloc(ctx, rule.size());
        dmax.alloc(ctx, 1);
        PLX_CHECK_CUDA(cudaMemcpyAsync(d_rule.p, rule.data(), rule.size() * 8, cudaMemcpyHostToDevice, st));
        PLX_CHECK_CUDA(cudaMemsetAsync(dmax.p, 0, 8, st));
        bem_polar_dmax<<<n_blocks(n, 128), 128, 0, st>>>(n, np, d_rule.p, tri.p, g->d_pos.p, dmax.p);
        unsigned long long bits = 0;
        PLX_CHECK_CUDA(cudaMemcpyAsync(&bits, dmax.p, 8, cudaMemcpyDeviceToHost, st));
        PLX_CHECK_CUDA(cudaStreamSynchronize(st));
        double dm;
        std::memcpy(&dm, &bits, 8);
        bem_diag_kernel<<<n_blocks(n, 128), 128, 0, st>>>(n, np, d_rule.p, tri.p, g->d_pos.p, g->d_frame.p,
                                                         dm * 1.0e-4, gvec.p, g->d_dpre.p);
        ctx->launches += 2;
    }
    g->d_T.alloc(ctx, (size_t)n * n);
    dim3 grid(n_blocks(n, 128), n);
    bem_matrix_kernel<<<grid, 128, 0, st>>>(n, accurate, sphere_r, tri.p, g->d_pos.p, g->d_frame.p, rad.p,
                                            g->d_dpre.p, g->d_T.p);
    ctx->launches++;
    if (!accurate) {
        // the diagonal is the same before and after (no closure)
        PLX_CHECK_CUDA(cudaMemcpy2DAsync(g->d_dpre.p, 8, g->d_T.p, (size_t)(n + 1) * 8, 8, n,
                                         cudaMemcpyDeviceToDevice, st));
    } else {
        bem_closure_kernel<<<n_blocks((int64_t)n * 32, 256), 256, 0, st>>>(n, g->d_pos.p, g->d_frame.p, gvec.p,
                                                                           g->d_T.p);
        ctx->launches++;
    }
    g->has_T = true;
    g->t_symmetric = false;
    PLX_CHECK_CUDA(cudaGetLastError());
    PLX_CHECK_CUDA(cudaStreamSynchronize(st));
}

void build_bem_ief(plx_geom *g) {
    if (g->d_M.p) return;
    plx_ctx *ctx = g->ctx;
    cudaStream_t st = ctx->stream;
    const int n = g->n_var;
    g->d_M.alloc(ctx, (size_t)n * n);
    g->d_DM.alloc(ctx, (size_t)n * n);
    bem_sainv_kernel<<<dim3(n_blocks(n, 128), n), 128, 0, st>>>(n, g->d_pos.p, g->d_M.p);
    ctx->launches++;
    // DM = D M (column-major: d_T row-major is D column-major)
    bem_dgemm(g, g->d_T.p, g->d_M.p, g->d_DM.p);
    PLX_CHECK_CUDA(cudaGetLastError());
}

void bem_apply_rows(plx_geom *g, const OpBatch &b, const double *S, const double *X, double *Y) {
    bem_rows<<<dim3(n_blocks(g->n_var, 256), b.count), 256, 0, g->ctx->stream>>>(g->n_var, b.count, b.d_freq,
                                                                                 g->d_dq.p, S, X, Y);
    g->ctx->launches++;
    PLX_CHECK_CUDA(cudaGetLastError());
}

void bem_diagonal_inverse(plx_geom *g, const OpBatch &b, double *Pinv) {
    bem_diag_inverse_kernel<<<dim3(n_blocks(g->n_var, 256), b.count), 256, 0, g->ctx->stream>>>(
        g->n_var, b.count, b.d_freq, g->d_dq.p, g->d_T.p, Pinv);
    g->ctx->launches++;
    PLX_CHECK_CUDA(cudaGetLastError());
}

void bem_rhs(plx_geom *g, const OpBatch &b, const int32_t *d_pol, double *Bout) {
    plx_ctx *ctx = g->ctx;
    cudaStream_t st = ctx->stream;
    const int n = g->n_var;
    const bool ief = g->model == PLX_BEM_IEF;
    dim3 grid(n_blocks(n, 256), b.count);
    if (!ief) {
        bem_rhs_kernel<<<grid, 256, 0, st>>>(n, b.count, 0, d_pol, g->e0, g->d_pos.p, g->d_frame.p, Bout);
        ctx->launches++;
        PLX_CHECK_CUDA(cudaGetLastError());
        return;
    }
    DevArray<double> V;
    V.alloc(ctx, (size_t)b.count * 2 * n);
    bem_rhs_kernel<<<grid, 256, 0, st>>>(n, b.count, 1, d_pol, g->e0, g->d_pos.p, g->d_frame.p, V.p);
    contract_t(g, b.count, V.p, Bout, Contraction::FP64);
    bem_ief_fix<<<grid, 256, 0, st>>>(n, b.count, g->d_dpre.p, g->d_T.p, V.p, Bout);
    ctx->launches += 2;
    PLX_CHECK_CUDA(cudaGetLastError());
    PLX_CHECK_CUDA(cudaStreamSynchronize(st));
}

void bem_assemble_matrix(plx_geom *g, int i_freq, double2 *A) {
    const int n = g->n_var;
    const bool ief = g->model == PLX_BEM_IEF;
    if (ief) build_bem_ief(g);
    Cplx z = g->bem_z[i_freq];
    bem_assemble<<<dim3(n_blocks(n, 128), n), 128, 0, g->ctx->stream>>>(n, ief, z, g->d_T.p, g->d_DM.p, g->d_M.p,
                                                                       A);
    g->ctx->launches++;
    PLX_CHECK_CUDA(cudaGetLastError());
}

}  // namespace plx
