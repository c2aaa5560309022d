// Gaussian-damped interaction tiles of the wFQ / wFQFMu kernel, evaluated for
// one ordered atom pair (i, j), i != j, in FP64.
//
// Follows construct_static_t_qq / t_qmu / t_muq / t_mumu
// (src/matrix/matrix_module.f90:58-345) and the on-the-fly products
// product_q_block_x / product_mu_block_x (matrix_module.f90:727-1001):
//   T_qq(i,j)      = erf(r/R_qq) / r,                R_qq = sqrt(Rq_i^2 + Rq_j^2)
//   T_qmu(i,j_k)   = d_k / r^3 * f(r, R_qm),          R_qm = sqrt(Rq_i^2 + Rmu_j^2)
//   T_muq(i_k,j)   = T_qmu(j, i_k) = -d_k / r^3 * f(r, R_mq), R_mq = sqrt(Rq_j^2 + Rmu_i^2)
//   T_mumu(i_a,j_b)= (-3 d_a d_b / r^5 + delta_ab / r^3) fD1 + fD2 d_a d_b / r^2,
//                    R_mm = sqrt(Rmu_i^2 + Rmu_j^2)
// with d = r_i - r_j, f(r,R) = erf(r/R) - 2r/(sqrt(pi) R) exp(-r^2/R^2) (= fD1),
// fD2 = 4 / (sqrt(pi) R^3) exp(-r^2/R^2).  The diagonal (i == j) is eta_i for
// T_qq and zero for the dipole blocks of the w-models.
#pragma once

#define PLX_SQRT_PI 1.7724538509055160273

struct PairTile {
    double qq;
    double qm[3];   // T_qmu(i, j_k)
    double mq[3];   // T_muq(i_k, j)
    double mm[6];   // T_mumu(i_a, j_b): xx, xy, xz, yy, yz, zz
};

__device__ __forceinline__ double plx_fdamp(double r, double R, double *e_out) {
    double invR = 1.0 / R;
    double e = exp(-(r * r) * (invR * invR));
    *e_out = e;
    return erf(r * invR) - ((2.0 * r) * invR / PLX_SQRT_PI) * e;
}

// Full tile for wFQFMu.  rq_i, rm_i: widths of atom i; rq_j, rm_j: of atom j.
__device__ __forceinline__ void plx_pair_tile(double dx, double dy, double dz, double rq_i,
                                              double rm_i, double rq_j, double rm_j,
                                              PairTile &t) {
    double r2 = dx * dx + dy * dy + dz * dz;
    double r = sqrt(r2);
    double ir = 1.0 / r;
    double ir2 = ir * ir;
    double ir3 = ir2 * ir;
    double ir5 = ir3 * ir2;
    double Rqq = sqrt(rq_i * rq_i + rq_j * rq_j);
    t.qq = erf(r / Rqq) * ir;
    double e;
    double f1 = plx_fdamp(r, sqrt(rq_i * rq_i + rm_j * rm_j), &e) * ir3;
    double f2 = plx_fdamp(r, sqrt(rq_j * rq_j + rm_i * rm_i), &e) * ir3;
    t.qm[0] = dx * f1;
    t.qm[1] = dy * f1;
    t.qm[2] = dz * f1;
    t.mq[0] = -dx * f2;
    t.mq[1] = -dy * f2;
    t.mq[2] = -dz * f2;
    double Rmm = sqrt(rm_i * rm_i + rm_j * rm_j);
    double em;
    double fD1 = plx_fdamp(r, Rmm, &em);
    double fD2 = (4.0 / (PLX_SQRT_PI * Rmm * Rmm * Rmm)) * em;
    double a = -3.0 * ir5 * fD1 + fD2 * ir2;
    double dd = ir3 * fD1;
    t.mm[0] = a * dx * dx + dd;
    t.mm[1] = a * dx * dy;
    t.mm[2] = a * dx * dz;
    t.mm[3] = a * dy * dy + dd;
    t.mm[4] = a * dy * dz;
    t.mm[5] = a * dz * dz + dd;
}

// Charge-charge element only (wFQ).
__device__ __forceinline__ double plx_pair_qq(double dx, double dy, double dz, double rq_i,
                                              double rq_j) {
    double r = sqrt(dx * dx + dy * dy + dz * dz);
    return erf(r / sqrt(rq_i * rq_i + rq_j * rq_j)) / r;
}

// One entry T[r][k] of the dense interaction matrix (rows/columns q_i -> i,
// mu_i,a -> N + 3 i + a), evaluated alone with the formulas of plx_pair_tile /
// plx_pair_qq: the building block of tiles generated in place (no stored T).
// pos [4][N] (x, y, z), par [4][N] (r_q, r_mu, eta, a_ij).
__device__ __forceinline__ double plx_t_element(int N, bool fmu, const double *__restrict__ pos,
                                                const double *__restrict__ par, int64_t r, int64_t k) {
    const int i = r < N ? (int)r : (int)((r - N) / 3), a = r < N ? -1 : (int)((r - N) % 3);
    const int j = k < N ? (int)k : (int)((k - N) / 3), b = k < N ? -1 : (int)((k - N) % 3);
    if (i == j) return (a < 0 && b < 0) ? par[2 * N + i] : 0.0;
    const double d[3] = {pos[i] - pos[j], pos[N + i] - pos[N + j], pos[2 * N + i] - pos[2 * N + j]};
    const double rq_i = par[i], rq_j = par[j];
    if (!fmu) return plx_pair_qq(d[0], d[1], d[2], rq_i, rq_j);
    const double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
    const double rr = sqrt(r2);
    const double ir = 1.0 / rr, ir2 = ir * ir, ir3 = ir2 * ir, ir5 = ir3 * ir2;
    const double rm_i = par[N + i], rm_j = par[N + j];
    double e;
    if (a < 0 && b < 0) return erf(rr / sqrt(rq_i * rq_i + rq_j * rq_j)) * ir;
    if (a < 0) return d[b] * (plx_fdamp(rr, sqrt(rq_i * rq_i + rm_j * rm_j), &e) * ir3);
    if (b < 0) return -d[a] * (plx_fdamp(rr, sqrt(rq_j * rq_j + rm_i * rm_i), &e) * ir3);
    const double Rmm = sqrt(rm_i * rm_i + rm_j * rm_j);
    const double fD1 = plx_fdamp(rr, Rmm, &e);
    const double fD2 = (4.0 / (PLX_SQRT_PI * Rmm * Rmm * Rmm)) * e;
    const double c = -3.0 * ir5 * fD1 + fD2 * ir2;
    return c * d[a] * d[b] + (a == b ? ir3 * fD1 : 0.0);
}

// Drude/Fermi conductance K_ij = (1 - 1/(1 + exp(-d (r/(s r0) - 1)))) A_i / r
// (construct_K_minus_P_matrix and fermi_function, matrix_module.f90:393-426,
// 694-715), evaluated in the same order as the reference so that pairs whose
// Fermi factor rounds to one give exactly zero, as in the reference.
__device__ __forceinline__ double plx_conductance(double r, double d, double s, double r0,
                                                  double a_i) {
    double f = 1.0 / (1.0 + exp(-d * ((r / (s * r0)) - 1.0)));
    return (1.0 - f) * a_i / r;
}
