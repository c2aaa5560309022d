// Induced field and plasmon density at points: the analysis step of the
// reference (calculate_induced_field_at_point_{wfq,wfqfmu} and
// calculate_density_at_point_{wfq,wfqfmu}, src/wfq/wfq_module.f90:590-650,
// src/wfq/wfqfmu_module.f90:975-1040, with the kernels
// calculate_induced_field_q / _mu and calculate_density_q / _mu of
// src/matrix/matrix_module.f90:1140-1322).  For d = r_atom - r_point (bohr):
//   E  = E0 e_pol - sum_i q_i d f(r, Rq_i) / r^3                  (r > 0.1)
//      + sum_i [(-3 d d^T / r^5 + I / r^3) fD1 + fD2 d d^T / r^2] mu_i  (r > 0.1)
//   rho = sum_i q_i exp(-r^2/Rq^2) / (pi^3/2 Rq^3)
//       - sum_i 2 exp(-r^2/Rmu^2) / (pi^3/2 Rmu^5) (mu_i . d)
// One thread per point; the atoms (position, widths, charge, dipole) are
// staged through shared memory in tiles.
#include <vector>

#include "pair_tiles.cuh"
#include "plx_internal.h"

namespace plx {

namespace {

constexpr int kPts = 128;
constexpr int kProfPoints = 7;   // plx_profile_read category of the point kernels
constexpr double kPi32 = 5.5683279968317078453;   // pi^(3/2)

__global__ void __launch_bounds__(kPts) field_points(int N, int nv, int fmu, int pol, double e0, int P,
                                                     const double *__restrict__ pos, const double *__restrict__ par,
                                                     const double2 *__restrict__ x, const double *__restrict__ pts,
                                                     double2 *__restrict__ field, double2 *__restrict__ dens) {
    __shared__ double sa[kPts][5];          // x, y, z, Rq, Rmu
    __shared__ double2 sq[kPts], sm[kPts][3];
    const int p = blockIdx.x * kPts + threadIdx.x;
    const bool live = p < P;
    const double px = live ? pts[p] : 0.0, py = live ? pts[P + p] : 0.0, pz = live ? pts[2LL * P + p] : 0.0;
    double er[3] = {0.0, 0.0, 0.0}, ei[3] = {0.0, 0.0, 0.0};
    double dr = 0.0, di = 0.0;
    for (int a0 = 0; a0 < N; a0 += kPts) {
        const int a = a0 + threadIdx.x;
        __syncthreads();
        if (a < N) {
            sa[threadIdx.x][0] = pos[a];
            sa[threadIdx.x][1] = pos[N + a];
            sa[threadIdx.x][2] = pos[2LL * N + a];
            sa[threadIdx.x][3] = par[a];
            sa[threadIdx.x][4] = par[N + a];
            sq[threadIdx.x] = x[a];
            if (fmu)
                for (int k = 0; k < 3; ++k) sm[threadIdx.x][k] = x[N + 3LL * a + k];
        }
        __syncthreads();
        if (!live) continue;
        const int an = min(kPts, N - a0);
        for (int t = 0; t < an; ++t) {
            const double d[3] = {sa[t][0] - px, sa[t][1] - py, sa[t][2] - pz};
            const double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
            const double r = sqrt(r2);
            const double Rq = sa[t][3];
            const double2 q = sq[t];
            const double gq = exp(-r2 / (Rq * Rq)) / (kPi32 * Rq * Rq * Rq);
            dr += gq * q.x;
            di += gq * q.y;
            const bool far = r > 1.0e-1;
            const double ir3 = far ? 1.0 / (r * r2) : 0.0;
            if (far) {
                const double f = erf(r / Rq) - (2.0 / (PLX_SQRT_PI * Rq)) * r * exp(-r2 / (Rq * Rq));
                for (int k = 0; k < 3; ++k) {
                    er[k] -= f * d[k] * q.x * ir3;
                    ei[k] -= f * d[k] * q.y * ir3;
                }
            }
            if (fmu) {
                const double Rm = sa[t][4];
                const double em = exp(-r2 / (Rm * Rm));
                const double2 m0 = sm[t][0], m1 = sm[t][1], m2 = sm[t][2];
                const double gm = 2.0 * em / (kPi32 * Rm * Rm * Rm) / (Rm * Rm);
                dr -= gm * (m0.x * d[0] + m1.x * d[1] + m2.x * d[2]);
                di -= gm * (m0.y * d[0] + m1.y * d[1] + m2.y * d[2]);
                if (far) {
                    const double fD1 = erf(r / Rm) - ((2.0 * r) / (PLX_SQRT_PI * Rm)) * em;
                    const double fD2 = (4.0 / (PLX_SQRT_PI * Rm * Rm * Rm)) * em;
                    const double ir2 = 1.0 / r2, ir5 = ir3 * ir2;
                    for (int aa = 0; aa < 3; ++aa) {
                        double tr = 0.0, ti = 0.0;
                        const double2 mb[3] = {m0, m1, m2};
                        for (int b = 0; b < 3; ++b) {
                            const double T = (-3.0 * d[aa] * d[b] * ir5 + (aa == b ? ir3 : 0.0)) * fD1 +
                                              fD2 * d[aa] * d[b] * ir2;
                            tr += T * mb[b].x;
                            ti += T * mb[b].y;
                        }
                        er[aa] += tr;
                        ei[aa] += ti;
                    }
                }
            }
        }
    }
    if (!live) return;
    er[pol] += e0;
    if (field)
        for (int k = 0; k < 3; ++k) field[3LL * p + k] = make_double2(er[k], ei[k]);
    if (dens) dens[p] = make_double2(dr, di);
}

// BEM field at points (calculate_induced_field_at_point_bem,
// src/bem/bem_module.f90:1152-1222, with calculate_induced_field_q_bem,
// src/matrix/matrix_module.f90:1444-1464): the point's first nearest tessera l
// decides inside / outside -- outside when |p - com| > |c_l - com| + 0.5 A,
// com the mean of the centres; inside, the field is zero; outside,
// E = E0 e_pol - sum_i q_i d_i / |d_i|^3 over |d_i| > 0.1 bohr, d_i = c_i - p.
// One thread per point; the centres and charges are read through the cache.
__global__ void __launch_bounds__(kPts) bem_field_points(int n, int P, int pol, double e0, double margin,
                                                         double cx, double cy, double cz,
                                                         const double *__restrict__ c /*[3][n]*/,
                                                         const double2 *__restrict__ q,
                                                         const double *__restrict__ pts /*[3][P]*/,
                                                         double2 *__restrict__ field) {
    const int p = blockIdx.x * kPts + threadIdx.x;
    if (p >= P) return;
    const double px = pts[p], py = pts[P + p], pz = pts[2 * P + p];
    double lowest = 1.0e6;
    int l = 0;
    for (int i = 0; i < n; ++i) {
        const double dx = c[i] - px, dy = c[n + i] - py, dz = c[2 * n + i] - pz;
        const double r = sqrt(dx * dx + dy * dy + dz * dz);
        if (lowest > r) {
            lowest = r;
            l = i;
        }
    }
    const double ex = c[l] - cx, ey = c[n + l] - cy, ez = c[2 * n + l] - cz;
    const double gx = px - cx, gy = py - cy, gz = pz - cz;
    double er[3] = {0.0, 0.0, 0.0}, ei[3] = {0.0, 0.0, 0.0};
    if (sqrt(gx * gx + gy * gy + gz * gz) > sqrt(ex * ex + ey * ey + ez * ez) + margin) {
        er[pol] = e0;
        for (int i = 0; i < n; ++i) {
            const double d[3] = {c[i] - px, c[n + i] - py, c[2 * n + i] - pz};
            const double r = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
            if (r > 1.0e-1) {
                const double r3 = r * (r * r);
                const double2 qi = q[i];
                for (int k = 0; k < 3; ++k) {
                    er[k] -= d[k] * qi.x / r3;
                    ei[k] -= d[k] * qi.y / r3;
                }
            }
        }
    }
    for (int k = 0; k < 3; ++k) field[3LL * p + k] = make_double2(er[k], ei[k]);
}

}  // namespace

void bem_field_at_points(plx_ctx *ctx, int n, const double *centres, const double *q, double e0, int pol, int P,
                         const double *points, double *field_out) {
    if (n < 1 || P < 0 || !centres || !q || !points || !field_out)
        throw Error(PLX_ERR_ARG, "BEM field at points: empty surface or null array");
    if (pol < 0 || pol > 2) throw Error(PLX_ERR_ARG, "polarisation index must be 0, 1 or 2");
    if (P == 0) return;
    std::vector<double> c(3 * (size_t)n), pts(3 * (size_t)P);
    double com[3] = {0.0, 0.0, 0.0};
    for (int i = 0; i < n; ++i)
        for (int k = 0; k < 3; ++k) {
            c[(size_t)k * n + i] = centres[3 * (size_t)i + k];
            com[k] += centres[3 * (size_t)i + k] / n;
        }
    for (int i = 0; i < P; ++i)
        for (int k = 0; k < 3; ++k) pts[(size_t)k * P + i] = points[3 * (size_t)i + k];
    cudaStream_t st = ctx->stream;
    DevArray<double> d_c, d_q, d_p, d_f;
    d_c.alloc(ctx, c.size());
    d_q.alloc(ctx, 2 * (size_t)n);
    d_p.alloc(ctx, pts.size());
    d_f.alloc(ctx, 6 * (size_t)P);
    PLX_CHECK_CUDA(cudaMemcpyAsync(d_c.p, c.data(), c.size() * 8, cudaMemcpyHostToDevice, st));
    PLX_CHECK_CUDA(cudaMemcpyAsync(d_q.p, q, 2 * (size_t)n * 8, cudaMemcpyHostToDevice, st));
    PLX_CHECK_CUDA(cudaMemcpyAsync(d_p.p, pts.data(), pts.size() * 8, cudaMemcpyHostToDevice, st));
    const double margin = 0.5 * 1.8897261254578281;   // 0.5 Angstrom in bohr
    prof_begin(ctx);
    bem_field_points<<<n_blocks(P, kPts), kPts, 0, st>>>(n, P, pol, e0, margin, com[0], com[1], com[2], d_c.p,
                                                         reinterpret_cast<const double2 *>(d_q.p), d_p.p,
                                                         reinterpret_cast<double2 *>(d_f.p));
    ctx->launches++;
    PLX_CHECK_CUDA(cudaGetLastError());
    prof_end(ctx, kProfPoints, 0.0, 8.0 * (5.0 * n + 9.0 * P));
    PLX_CHECK_CUDA(cudaMemcpyAsync(field_out, d_f.p, 6 * (size_t)P * 8, cudaMemcpyDeviceToHost, st));
    PLX_CHECK_CUDA(cudaStreamSynchronize(st));
}

void field_at_points(plx_geom *g, int pol, const double *d_x, int P, const double *d_pts, double *d_field,
                     double *d_dens) {
    plx_ctx *ctx = g->ctx;
    prof_begin(ctx);
    field_points<<<n_blocks(P, kPts), kPts, 0, ctx->stream>>>(
        g->n_atoms, g->n_var, g->model == PLX_WFQFMU, pol, g->e0, P, g->d_pos.p, g->d_par.p,
        reinterpret_cast<const double2 *>(d_x), d_pts, reinterpret_cast<double2 *>(d_field),
        reinterpret_cast<double2 *>(d_dens));
    ctx->launches++;
    PLX_CHECK_CUDA(cudaGetLastError());
    // atoms (positions, widths, the solution) once, points in, field and density out
    prof_end(ctx, kProfPoints, 0.0, 8.0 * (5.0 * g->n_atoms + 2.0 * g->n_var + 3.0 * P + 6.0 * P + 2.0 * P));
}

}  // namespace plx
