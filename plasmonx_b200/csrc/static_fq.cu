// Static FQ / FQFMu solves and the principal-axis rotation.
//
// The static force fields of the reference, whose types the w-models extend:
//   * the static matrix, built on the device element by element (column-major,
//     n_var x n_var): the charge block T_qq with the Coulomb, Ohno or Gaussian
//     kernel (construct_static_t_qq, src/matrix/matrix_module.f90:58-115), one
//     charge-constraint row and column per molecule (add_lagrangian_blocks,
//     :351-382) and, for FQFMu, T_qmu, its transpose and T_mumu with 1/alpha on
//     the diagonal blocks (:120-345); layout of construct_static_matrix_fq
//     (src/forcefield/fq_module.f90:179-207) and construct_static_matrix_fqfmu
//     (src/forcefield/fqfmu_module.f90:81-132);
//   * right-hand sides: -chi per atom for the ground state
//     (construct_ground_state_rhs_fq, fq_module.f90:212-242), or the three
//     static-field columns (construct_static_field_rhs_q / _mu,
//     src/rhs/rhs_module.f90:43-127);
//   * the solve: the reference factors with dsysv (Bunch-Kaufman on the upper
//     triangle, real_inversion, src/solvers/algorithm_module.f90:469-504); the
//     matrix built here is exactly symmetric, and the library factors it with
//     cuSOLVER's pivoted LU (dgetrf / dgetrs), the same solution to rounding;
//   * the ground-state energy -1/2 x.b (calculate_energy_fq, fq_module.f90:358-374)
//     and the FQ static polarizability
//     R^T J^-1 R - (L^T J^-1 R)^T (L^T J^-1 L)^-1 (L^T J^-1 R), J the charge
//     block and L the constraint columns (calculate_static_polar_fq,
//     fq_module.f90:379-595; the reference forms J^-1 and (L^T J^-1 L)^-1
//     explicitly, here both are applied through their LU factors).
// The principal-axis rotation (rotate_principal_axis,
// src/target/target_module.f90:684-835) runs on the host: it is O(N) with a
// 3 x 3 eigenproblem, done before the geometry reaches the device.
#include <cublas_v2.h>
#include <cusolverDn.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "plx_internal.h"

namespace plx {
cusolverDnHandle_t solver_handle(plx_ctx *ctx);
cublasHandle_t blas_handle(plx_ctx *ctx);
}  // namespace plx

using namespace plx;

namespace {

constexpr double kSqrtPi = 1.7724538509055160273;
// plx_profile_read categories of the static solve
constexpr int kProfStaticAssembly = 5;   // static matrix and right-hand sides
constexpr int kProfStaticFactor = 6;     // dense LU factorisations and solves

struct StaticDims {
    int n;        // atoms (charges)
    int n_mol;    // molecules (constraint rows)
    int n_fq;     // n + n_mol
    int n_var;    // n_fq (FQ) or 4 n + n_mol (FQFMu)
    int fmu;      // FQFMu
    int kernel;   // plx_charge_kernel
    int n_types;
};

// per-type parameters, [5][n_types]: chi, eta, alpha, r_q, r_mu
enum { P_CHI = 0, P_ETA = 1, P_ALPHA = 2, P_RQ = 3, P_RMU = 4 };

__device__ __forceinline__ double tpar(const double *par, int nt, int which, int t) { return par[which * nt + t]; }

// erf(d/R) - 2 d / (sqrt(pi) R) exp(-d^2/R^2): the screening of a Gaussian
// charge-dipole and dipole-dipole pair (matrix_module.f90:155-166, :301-307)
__device__ __forceinline__ double screen(double d, double R) {
    return erf(d / R) - ((2.0 * d) / (kSqrtPi * R)) * exp(-(d * d) / (R * R));
}

__device__ double t_qq(const StaticDims &s, const double *pos, const int32_t *type, const double *par, int i, int j) {
    const double dx = pos[i] - pos[j], dy = pos[s.n + i] - pos[s.n + j], dz = pos[2 * s.n + i] - pos[2 * s.n + j];
    const double d = sqrt(dx * dx + dy * dy + dz * dz);
    const int ti = type[i], tj = type[j];
    const double ei = tpar(par, s.n_types, P_ETA, ti), ej = tpar(par, s.n_types, P_ETA, tj);
    if (s.kernel == PLX_KERNEL_OHNO) {
        const double ea = 0.5 * (ei + ej);
        return ea / sqrt(1.0 + (ea * ea) * (d * d));
    }
    if (i == j) return (ei + ej) / 2.0;
    if (s.kernel == PLX_KERNEL_COULOMB) return 1.0 / d;
    const double ri = tpar(par, s.n_types, P_RQ, ti), rj = tpar(par, s.n_types, P_RQ, tj);
    return erf(d / sqrt(ri * ri + rj * rj)) / d;
}

// T_qmu(i, 3 j + k): charge i, dipole component k of atom j (zero for i == j)
__device__ double t_qmu(const StaticDims &s, const double *pos, const int32_t *type, const double *par, int i, int j,
                        int k) {
    if (i == j) return 0.0;
    const double dx = pos[i] - pos[j], dy = pos[s.n + i] - pos[s.n + j], dz = pos[2 * s.n + i] - pos[2 * s.n + j];
    const double d = sqrt(dx * dx + dy * dy + dz * dz);
    const double rq = tpar(par, s.n_types, P_RQ, type[i]), rm = tpar(par, s.n_types, P_RMU, type[j]);
    const double rk = k == 0 ? dx : (k == 1 ? dy : dz);
    return rk / (d * d * d) * screen(d, sqrt(rq * rq + rm * rm));
}

// T_mumu(3 i + a, 3 j + b)
__device__ double t_mumu(const StaticDims &s, const double *pos, const int32_t *type, const double *par, int i, int a,
                         int j, int b) {
    if (i == j) return a == b ? 1.0 / tpar(par, s.n_types, P_ALPHA, type[i]) : 0.0;
    const double r[3] = {pos[i] - pos[j], pos[s.n + i] - pos[s.n + j], pos[2 * s.n + i] - pos[2 * s.n + j]};
    const double d = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
    const double d2 = d * d, d3 = d2 * d, d5 = d3 * d2;
    const double mi = tpar(par, s.n_types, P_RMU, type[i]), mj = tpar(par, s.n_types, P_RMU, type[j]);
    const double R = sqrt(mi * mi + mj * mj);
    const double fd1 = screen(d, R);
    const double fd2 = (4.0 / (kSqrtPi * (R * R * R))) * exp(-d2 / (R * R));
    const double rab = r[a] * r[b];
    return ((-3.0 * rab) / d5 + (a == b ? 1.0 / d3 : 0.0)) * fd1 + fd2 * rab / d2;
}

// One element A(r, c) per thread, rows fastest (coalesced column-major stores).
__global__ void static_matrix_kernel(StaticDims s, const double *__restrict__ pos, const int32_t *__restrict__ type,
                                     const double *__restrict__ par, const int32_t *__restrict__ mol_lo,
                                     const int32_t *__restrict__ mol_hi, double *__restrict__ A) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= s.n_var) return;
    for (int c = blockIdx.y; c < s.n_var; c += gridDim.y) {
        double v = 0.0;
        if (r < s.n && c < s.n) {
            v = t_qq(s, pos, type, par, r, c);
        } else if (r < s.n && c < s.n_fq) {
            v = (r >= mol_lo[c - s.n] && r < mol_hi[c - s.n]) ? 1.0 : 0.0;
        } else if (r < s.n_fq && c < s.n) {
            v = (c >= mol_lo[r - s.n] && c < mol_hi[r - s.n]) ? 1.0 : 0.0;
        } else if (s.fmu) {
            if (r < s.n && c >= s.n_fq) {
                v = t_qmu(s, pos, type, par, r, (c - s.n_fq) / 3, (c - s.n_fq) % 3);
            } else if (r >= s.n_fq && c < s.n) {
                v = t_qmu(s, pos, type, par, c, (r - s.n_fq) / 3, (r - s.n_fq) % 3);
            } else if (r >= s.n_fq && c >= s.n_fq) {
                v = t_mumu(s, pos, type, par, (r - s.n_fq) / 3, (r - s.n_fq) % 3, (c - s.n_fq) / 3, (c - s.n_fq) % 3);
            }
        }
        A[(int64_t)c * s.n_var + r] = v;
    }
}

// Right-hand sides, column-major n_var x n_rhs.  Ground state: -chi of the
// atom's type.  Static field: -E0 r_k ("field") or -E0 |r_k - min r_k|
// ("potential") for the charges; for the dipoles of FQFMu the reference writes
// E0 on the k-th component of column k when E0 is zero (|E0| <= 1e-14) and 1
// otherwise (rhs_module.f90:96-127).
__global__ void static_rhs_kernel(StaticDims s, int field, int potential, double e0, double x0, double y0, double z0,
                                  const double *__restrict__ pos, const int32_t *__restrict__ type,
                                  const double *__restrict__ par, double *__restrict__ B) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= s.n_var) return;
    if (!field) {
        B[r] = r < s.n ? -tpar(par, s.n_types, P_CHI, type[r]) : 0.0;
        return;
    }
    const double mins[3] = {x0, y0, z0};
    const double vmu = fabs(e0) <= 1.0e-14 ? e0 : 1.0;
    for (int k = 0; k < 3; ++k) {
        double v = 0.0;
        if (r < s.n) {
            const double c = pos[k * s.n + r];
            v = potential ? -e0 * fabs(c - mins[k]) : -e0 * c;
        } else if (s.fmu && r >= s.n_fq && (r - s.n_fq) % 3 == k) {
            v = vmu;
        }
        B[(int64_t)k * s.n_var + r] = v;
    }
}

void check_info(plx_ctx *ctx, const DevArray<int32_t> &info, const char *what) {
    int h = 0;
    PLX_CHECK_CUDA(cudaMemcpyAsync(&h, info.p, 4, cudaMemcpyDeviceToHost, ctx->stream));
    PLX_CHECK_CUDA(cudaStreamSynchronize(ctx->stream));
    if (h != 0) throw Error(PLX_ERR_SINGULAR, std::string("info = ") + std::to_string(h) + " in " + what);
}

// A (n x n, column-major, overwritten by its LU factors) X = B (n x nrhs)
void lu_solve(plx_ctx *ctx, int n, double *A, int nrhs, double *B, const char *what) {
    cusolverDnHandle_t h = solver_handle(ctx);
    int lwork = 0;
    if (cusolverDnDgetrf_bufferSize(h, n, n, A, n, &lwork) != CUSOLVER_STATUS_SUCCESS)
        throw Error(PLX_ERR_CUDA, "cusolverDnDgetrf_bufferSize failed");
    DevArray<double> work;
    DevArray<int32_t> ipiv, info;
    work.alloc(ctx, std::max(lwork, 1));
    ipiv.alloc(ctx, n);
    info.alloc(ctx, 1);
    if (cusolverDnDgetrf(h, n, n, A, n, work.p, ipiv.p, info.p) != CUSOLVER_STATUS_SUCCESS)
        throw Error(PLX_ERR_CUDA, "cusolverDnDgetrf failed");
    check_info(ctx, info, what);
    if (cusolverDnDgetrs(h, CUBLAS_OP_N, n, nrhs, A, n, ipiv.p, B, n, info.p) != CUSOLVER_STATUS_SUCCESS)
        throw Error(PLX_ERR_CUDA, "cusolverDnDgetrs failed");
    check_info(ctx, info, what);
}

// C (m x k) = A^T B with A (n x m, lda) and B (n x k, ldb), column-major
void gemm_tn(plx_ctx *ctx, int m, int k, int n, const double *A, int lda, const double *B, int ldb, double *C) {
    const double one = 1.0, zero = 0.0;
    if (cublasDgemm(blas_handle(ctx), CUBLAS_OP_T, CUBLAS_OP_N, m, k, n, &one, A, lda, B, ldb, &zero, C, m) !=
        CUBLAS_STATUS_SUCCESS)
        throw Error(PLX_ERR_CUDA, "cublasDgemm failed");
}

}  // namespace

namespace plx {

int64_t static_n_var(const plx_static_desc *d) {
    if (!d || d->n_atoms < 1 || d->n_mol < 1) return -1;
    return d->forcefield == PLX_STATIC_FQFMU ? 4 * (int64_t)d->n_atoms + d->n_mol : (int64_t)d->n_atoms + d->n_mol;
}

void static_solve(plx_ctx *ctx, const plx_static_desc *d, int what, double *variables, double *energy,
                  double *polar) {
    if (!d || !d->coord || !d->atom_type || !d->atoms_per_molecule || !d->eta || !d->chi)
        throw Error(PLX_ERR_ARG, "static description with a null array");
    if (d->forcefield != PLX_STATIC_FQ && d->forcefield != PLX_STATIC_FQFMU)
        throw Error(PLX_ERR_ARG, "forcefield must be PLX_STATIC_FQ or PLX_STATIC_FQFMU");
    if (d->kernel < PLX_KERNEL_COULOMB || d->kernel > PLX_KERNEL_GAUSSIAN)
        throw Error(PLX_ERR_ARG, "unknown charge kernel");
    if (what != PLX_GROUND_STATE && what != PLX_STATIC_FIELD) throw Error(PLX_ERR_ARG, "unknown static solve");
    const bool fmu = d->forcefield == PLX_STATIC_FQFMU;
    if (fmu && (!d->alpha || !d->r_q || !d->r_mu)) throw Error(PLX_ERR_ARG, "FQFMu needs alpha, r_q and r_mu");
    if (d->kernel == PLX_KERNEL_GAUSSIAN && !d->r_q) throw Error(PLX_ERR_ARG, "the Gaussian kernel needs r_q");
    if (polar && (what != PLX_STATIC_FIELD || fmu))
        throw Error(PLX_ERR_UNSUPPORTED, fmu ? "Static Polar for FQFMu not yet implemented (as in the reference)"
                                             : "the static polarizability needs a static-field solve");
    if (energy && what != PLX_GROUND_STATE) throw Error(PLX_ERR_ARG, "the energy is a ground-state quantity");
    const int64_t nv64 = static_n_var(d);
    if (nv64 < 1 || d->n_types < 1) throw Error(PLX_ERR_ARG, "n_atoms, n_mol and n_types must be positive");
    if (nv64 > (1 << 30)) throw Error(PLX_ERR_ARG, "static problem too large");
    StaticDims s{d->n_atoms, d->n_mol, d->n_atoms + d->n_mol, (int)nv64, fmu ? 1 : 0, d->kernel, d->n_types};
    const int n = s.n, nt = s.n_types, nv = s.n_var, m = s.n_mol;
    for (int i = 0; i < n; ++i)
        if (d->atom_type[i] < 0 || d->atom_type[i] >= nt) throw Error(PLX_ERR_ARG, "atom type out of range");

    // constraint rows of molecule k, as add_lagrangian_blocks indexes them:
    // molecule 1 is atoms 1..apm(1), molecule k > 1 atoms apm(k-1)(k-1)+1 ..
    // apm(k-1)(k-1)+apm(k) (exact for molecules of equal size)
    std::vector<int32_t> lo(m), hi(m);
    for (int k = 0; k < m; ++k) {
        const int64_t a = d->atoms_per_molecule[k];
        if (a < 1) throw Error(PLX_ERR_ARG, "a molecule without atoms");
        const int64_t l = k == 0 ? 0 : (int64_t)d->atoms_per_molecule[k - 1] * k;
        if (l + a > n)
            throw Error(PLX_ERR_ARG, "molecule " + std::to_string(k + 1) +
                                         ": the constraint rows of the reference's indexing run past the atoms");
        lo[k] = (int32_t)l;
        hi[k] = (int32_t)(l + a);
    }
    std::vector<double> pos(3 * (size_t)n), par(5 * (size_t)nt, 0.0);
    double mins[3] = {0.0, 0.0, 0.0};
    for (int i = 0; i < n; ++i)
        for (int k = 0; k < 3; ++k) {
            const double c = d->coord[3 * (size_t)i + k];
            pos[(size_t)k * n + i] = c;
            if (i == 0 || c < mins[k]) mins[k] = c;
        }
    for (int t = 0; t < nt; ++t) {
        par[P_CHI * nt + t] = d->chi[t];
        par[P_ETA * nt + t] = d->eta[t];
        if (d->alpha) par[P_ALPHA * nt + t] = d->alpha[t];
        if (d->r_q) par[P_RQ * nt + t] = d->r_q[t];
        if (d->r_mu) par[P_RMU * nt + t] = d->r_mu[t];
    }
    cudaStream_t st = ctx->stream;
    DevArray<double> d_pos, d_par, A, B, B0;
    DevArray<int32_t> d_type, d_lo, d_hi;
    d_pos.alloc(ctx, pos.size());
    d_par.alloc(ctx, par.size());
    d_type.alloc(ctx, n);
    d_lo.alloc(ctx, m);
    d_hi.alloc(ctx, m);
    PLX_CHECK_CUDA(cudaMemcpyAsync(d_pos.p, pos.data(), pos.size() * 8, cudaMemcpyHostToDevice, st));
    PLX_CHECK_CUDA(cudaMemcpyAsync(d_par.p, par.data(), par.size() * 8, cudaMemcpyHostToDevice, st));
    PLX_CHECK_CUDA(cudaMemcpyAsync(d_type.p, d->atom_type, (size_t)n * 4, cudaMemcpyHostToDevice, st));
    PLX_CHECK_CUDA(cudaMemcpyAsync(d_lo.p, lo.data(), (size_t)m * 4, cudaMemcpyHostToDevice, st));
    PLX_CHECK_CUDA(cudaMemcpyAsync(d_hi.p, hi.data(), (size_t)m * 4, cudaMemcpyHostToDevice, st));

    const int nrhs = what == PLX_STATIC_FIELD ? 3 : 1;
    A.alloc(ctx, (size_t)nv * nv);
    B.alloc(ctx, (size_t)nv * nrhs);
    const int rows = n_blocks(nv, 128);
    prof_begin(ctx);
    static_matrix_kernel<<<dim3(rows, std::min(nv, 65535)), 128, 0, st>>>(s, d_pos.p, d_type.p, d_par.p, d_lo.p,
                                                                          d_hi.p, A.p);
    static_rhs_kernel<<<rows, 128, 0, st>>>(s, what == PLX_STATIC_FIELD, d->rhs_potential, d->e0, mins[0], mins[1],
                                            mins[2], d_pos.p, d_type.p, d_par.p, B.p);
    ctx->launches += 2;
    PLX_CHECK_CUDA(cudaGetLastError());
    prof_end(ctx, kProfStaticAssembly, 0.0, 8.0 * ((double)nv * nv + (double)nv * nrhs));

    // the polarizability works on the charge block J and the constraint
    // columns L, copied out before A is factored in place
    DevArray<double> J, L, X;
    if (polar) {
        J.alloc(ctx, (size_t)n * n);
        L.alloc(ctx, (size_t)n * m);
        X.alloc(ctx, (size_t)n * (3 + m));
        PLX_CHECK_CUDA(cudaMemcpy2DAsync(J.p, (size_t)n * 8, A.p, (size_t)nv * 8, (size_t)n * 8, n,
                                         cudaMemcpyDeviceToDevice, st));
        PLX_CHECK_CUDA(cudaMemcpy2DAsync(L.p, (size_t)n * 8, A.p + (size_t)n * nv, (size_t)nv * 8, (size_t)n * 8, m,
                                         cudaMemcpyDeviceToDevice, st));
        PLX_CHECK_CUDA(cudaMemcpyAsync(X.p, d_pos.p, (size_t)3 * n * 8, cudaMemcpyDeviceToDevice, st));
        PLX_CHECK_CUDA(cudaMemcpyAsync(X.p + (size_t)3 * n, L.p, (size_t)n * m * 8, cudaMemcpyDeviceToDevice, st));
    }
    if (energy) {
        B0.alloc(ctx, (size_t)nv);
        PLX_CHECK_CUDA(cudaMemcpyAsync(B0.p, B.p, (size_t)nv * 8, cudaMemcpyDeviceToDevice, st));
    }
    const double dn = nv;
    prof_begin(ctx);
    lu_solve(ctx, nv, A.p, nrhs, B.p, "DSYSV in real inversion");
    prof_end(ctx, kProfStaticFactor, 2.0 / 3.0 * dn * dn * dn + 2.0 * dn * dn * nrhs, 8.0 * dn * dn);
    A.release();
    if (energy) {
        double dot = 0.0;
        if (cublasDdot(blas_handle(ctx), nv, B.p, 1, B0.p, 1, &dot) != CUBLAS_STATUS_SUCCESS)
            throw Error(PLX_ERR_CUDA, "cublasDdot failed");
        *energy = -0.5 * dot;
    }
    if (variables) {
        PLX_CHECK_CUDA(cudaMemcpyAsync(variables, B.p, (size_t)nv * nrhs * 8, cudaMemcpyDeviceToHost, st));
    }
    if (polar) {
        // X = J^-1 [R | L]
        prof_begin(ctx);
        lu_solve(ctx, n, J.p, 3 + m, X.p, "dgetrf in FQ calculate_static_polar");
        prof_end(ctx, kProfStaticFactor, 2.0 / 3.0 * n * (double)n * n + 2.0 * n * (double)n * (3 + m),
                 8.0 * n * (double)n);
        J.release();
        DevArray<double> P, J11, J1R, Y;
        P.alloc(ctx, 18);
        J11.alloc(ctx, (size_t)m * m);
        J1R.alloc(ctx, (size_t)m * 3);
        Y.alloc(ctx, (size_t)m * 3);
        const double *XR = X.p, *XL = X.p + (size_t)3 * n;
        gemm_tn(ctx, 3, 3, n, d_pos.p, n, XR, n, P.p);      // R^T J^-1 R
        gemm_tn(ctx, m, m, n, L.p, n, XL, n, J11.p);        // L^T J^-1 L
        gemm_tn(ctx, m, 3, n, L.p, n, XR, n, J1R.p);        // L^T J^-1 R
        PLX_CHECK_CUDA(cudaMemcpyAsync(Y.p, J1R.p, (size_t)m * 3 * 8, cudaMemcpyDeviceToDevice, st));
        lu_solve(ctx, m, J11.p, 3, Y.p, "dgetrf @2 in FQ calculate_static_polar");
        gemm_tn(ctx, 3, 3, m, J1R.p, m, Y.p, m, P.p + 9);  // (L^T J^-1 R)^T (L^T J^-1 L)^-1 (L^T J^-1 R)
        double h[18];
        PLX_CHECK_CUDA(cudaMemcpyAsync(h, P.p, sizeof(h), cudaMemcpyDeviceToHost, st));
        PLX_CHECK_CUDA(cudaStreamSynchronize(st));
        for (int k = 0; k < 9; ++k) polar[k] = h[k] - h[9 + k];
    }
    PLX_CHECK_CUDA(cudaStreamSynchronize(st));
}

// ---------------------------------------------------------------------------
// principal axes (host)
// ---------------------------------------------------------------------------

// standard atomic masses of the elements the reference knows (mass_atom,
// src/target/target_module.f90:233-289); 0 for the others
static double atomic_mass(int z) {
    switch (z) {
        case 1: return 1.00794;
        case 2: return 4.00260;
        case 3: return 6.941;
        case 4: return 9.01218;
        case 5: return 10.81;
        case 6: return 12.0107;
        case 7: return 14.0067;
        case 8: return 15.9990;
        case 9: return 18.998403;
        case 10: return 20.179;
        case 11: return 22.989770;
        case 12: return 24.305;
        case 13: return 26.98154;
        case 14: return 28.0855;
        case 15: return 30.97376;
        case 16: return 32.06;
        case 17: return 35.453;
        case 18: return 39.948;
        case 29: return 63.546;
        case 47: return 107.8682;
        case 79: return 196.9665;
        default: return 0.0;
    }
}

// Eigen-decomposition of a symmetric 3 x 3 matrix by the cyclic Jacobi method
// (rotations that annihilate one off-diagonal entry at a time, Golub & Van
// Loan, Matrix Computations, sec. 8.5): a is destroyed, w receives the
// eigenvalues in ascending order and v (column-major) the eigenvectors.
static void jacobi3(double a[3][3], double w[3], double v[9]) {
    double V[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
    for (int sweep = 0; sweep < 64; ++sweep) {
        const double off = a[0][1] * a[0][1] + a[0][2] * a[0][2] + a[1][2] * a[1][2];
        const double diag = a[0][0] * a[0][0] + a[1][1] * a[1][1] + a[2][2] * a[2][2];
        if (off == 0.0 || off <= 1e-36 * diag) break;
        for (int p = 0; p < 2; ++p)
            for (int q = p + 1; q < 3; ++q) {
                if (a[p][q] == 0.0) continue;
                // rotation angle from cot(2 theta) = (a_qq - a_pp) / (2 a_pq)
                const double theta = (a[q][q] - a[p][p]) / (2.0 * a[p][q]);
                const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
                const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
                for (int k = 0; k < 3; ++k) {  // A <- A J
                    const double akp = a[k][p], akq = a[k][q];
                    a[k][p] = c * akp - s * akq;
                    a[k][q] = s * akp + c * akq;
                }
                for (int k = 0; k < 3; ++k) {  // A <- J^T A
                    const double apk = a[p][k], aqk = a[q][k];
                    a[p][k] = c * apk - s * aqk;
                    a[q][k] = s * apk + c * aqk;
                }
                for (int k = 0; k < 3; ++k) {  // V <- V J
                    const double vkp = V[k][p], vkq = V[k][q];
                    V[k][p] = c * vkp - s * vkq;
                    V[k][q] = s * vkp + c * vkq;
                }
            }
    }
    int order[3] = {0, 1, 2};
    std::sort(order, order + 3, [&](int x, int y) { return a[x][x] < a[y][y]; });
    for (int c = 0; c < 3; ++c) {
        const int o = order[c];
        w[c] = a[o][o];
        // LAPACK leaves the sign to the implementation; the last nonzero
        // component is made positive
        double sgn = 1.0;
        for (int k = 2; k >= 0; --k)
            if (V[k][o] != 0.0) {
                sgn = V[k][o] < 0 ? -1.0 : 1.0;
                break;
            }
        for (int k = 0; k < 3; ++k) v[3 * c + k] = sgn * V[k][o];
    }
}

void principal_axes(int n, const int32_t *z, double *coord, double *eigenvalues, double *axes) {
    if (n < 1 || !z || !coord) throw Error(PLX_ERR_ARG, "principal axes of an empty geometry");
    std::vector<double> mass(n);
    double total = 0.0;
    for (int i = 0; i < n; ++i) {
        mass[i] = atomic_mass(z[i]);
        if (mass[i] == 0.0) throw Error(PLX_ERR_ARG, "Atomic number not recognized for atomic mass");
        total += mass[i];
    }
    double com[3] = {0.0, 0.0, 0.0};
    for (int i = 0; i < n; ++i)
        for (int k = 0; k < 3; ++k) com[k] += mass[i] * coord[3 * (size_t)i + k] / total;
    double I[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    for (int i = 0; i < n; ++i) {
        double *c = coord + 3 * (size_t)i;
        for (int k = 0; k < 3; ++k) c[k] -= com[k];
        const double m = mass[i], x = c[0], y = c[1], zz = c[2];
        I[0][0] += m * (y * y + zz * zz);
        I[1][1] += m * (x * x + zz * zz);
        I[2][2] += m * (y * y + x * x);
        I[0][1] -= m * (x * y);
        I[0][2] -= m * (x * zz);
        I[1][2] -= m * (y * zz);
    }
    I[1][0] = I[0][1];
    I[2][0] = I[0][2];
    I[2][1] = I[1][2];
    double w[3], v[9];
    jacobi3(I, w, v);
    for (int i = 0; i < n; ++i) {  // r' = V^T r
        double *c = coord + 3 * (size_t)i;
        const double r[3] = {c[0], c[1], c[2]};
        for (int k = 0; k < 3; ++k) c[k] = v[3 * k] * r[0] + v[3 * k + 1] * r[1] + v[3 * k + 2] * r[2];
    }
    if (eigenvalues)
        for (int k = 0; k < 3; ++k) eigenvalues[k] = w[k];
    if (axes)
        for (int k = 0; k < 9; ++k) axes[k] = v[k];
}

}  // namespace plx
