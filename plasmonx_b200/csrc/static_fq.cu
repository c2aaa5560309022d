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
//   * the solve: the reference factors the full symmetric indefinite system
//     with dsysv (Bunch-Kaufman on the upper triangle, real_inversion,
//     src/solvers/algorithm_module.f90:469-504).  Here, by default, the charge
//     constraints are eliminated on a null-space basis (Householder reflectors
//     per molecule) and the remaining symmetric positive definite system is
//     factored by Cholesky (cuSOLVER dpotrf): the same solution to rounding
//     with, for water, 1/16 of the LU's flops.  When the constraint blocks
//     overlap (ragged molecules under the reference's indexing) or Cholesky
//     breaks down, or when asked, the full system is factored by pivoted LU
//     (dgetrf / dgetrs).  On request the reduced system is factored in single
//     precision and refined in double (mixed_cholesky); measured on B200 it
//     does not beat the double-precision factor at these sizes.  Also on
//     request, the reduced system is factored by the hand-written blocked
//     Cholesky of cholesky.cu (correct, but measured far slower than dpotrf:
//     96 ms against 5 ms at 6,000 unknowns);
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

// Z[:, j] = K Y[:, j] for nrhs <= 3 columns (K N x N column-major), in
// kGemvChunks column chunks (partials Zp[chunk][j][r], then summed in chunk
// order): one thread per row and chunk, K read once (coalesced), Y broadcast.
constexpr int kGemvChunks = 16;
__global__ void dense_gemv_part(int N, int nrhs, const double *__restrict__ K, const double *__restrict__ Y,
                                double *__restrict__ Zp) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= N) return;
    const int per = (N + kGemvChunks - 1) / kGemvChunks;
    const int c0 = blockIdx.y * per, c1 = min(N, c0 + per);
    double acc[3] = {0.0, 0.0, 0.0};
    for (int c = c0; c < c1; ++c) {
        const double k = K[(int64_t)c * N + r];
        for (int j = 0; j < nrhs; ++j) acc[j] = fma(k, Y[c + (int64_t)N * j], acc[j]);
    }
    for (int j = 0; j < nrhs; ++j) Zp[((int64_t)blockIdx.y * nrhs + j) * N + r] = acc[j];
}

__global__ void dense_gemv_sum(int N, int nrhs, const double *__restrict__ Zp, double *__restrict__ Z) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (int64_t)N * nrhs) return;
    double s = 0.0;
    for (int q = 0; q < kGemvChunks; ++q) s += Zp[(int64_t)q * nrhs * N + e];
    Z[e] = s;
}

// C[i + m j] = sum_p A[p + lda i] B[p + ldb j], one block per output (fixed order).
__global__ void small_gemm_tn(int m, int n, const double *__restrict__ A, int lda, const double *__restrict__ B,
                              int ldb, double *__restrict__ C) {
    const int i = blockIdx.x % m, j = blockIdx.x / m;
    double s = 0.0;
    for (int p = threadIdx.x; p < n; p += blockDim.x) s += A[p + (int64_t)lda * i] * B[p + (int64_t)ldb * j];
    __shared__ double red[32];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
        C[blockIdx.x] = t;
    }
}

// C (m x k) = A^T B with A (n x m, lda) and B (n x k, ldb), column-major
void gemm_tn(plx_ctx *ctx, int m, int k, int n, const double *A, int lda, const double *B, int ldb, double *C) {
    if (m * k <= 64) {
        // a few outputs (the 3 x 3 polarizability): block reductions
        small_gemm_tn<<<m * k, 256, 0, ctx->stream>>>(m, n, A, lda, B, ldb, C);
        ctx->launches++;
        PLX_CHECK_CUDA(cudaGetLastError());
        return;
    }
    const double one = 1.0, zero = 0.0;
    if (cublasDgemm(blas_handle(ctx), CUBLAS_OP_T, CUBLAS_OP_N, m, k, n, &one, A, lda, B, ldb, &zero, C, m) !=
        CUBLAS_STATUS_SUCCESS)
        throw Error(PLX_ERR_CUDA, "cublasDgemm failed");
}

// ---------------------------------------------------------------------------
// constraint elimination
//
// Molecule k constrains the charges of its atom rows [lo_k, hi_k) to sum to
// zero.  With the Householder reflector H_k = I - beta v v^T, v = 1 + sqrt(a) e_0
// (a = hi_k - lo_k, beta = 1 / (a + sqrt(a))), H_k 1 = -sqrt(a) e_0: in the
// reflected basis the constraint fixes the first coordinate of the block to zero
// and leaves the other a - 1 free.  With H the block-diagonal product of the
// H_k (disjoint blocks), the constrained solve becomes an unconstrained one on
// H K H with the first row and column of every block removed, symmetric positive
// definite when K (the matrix without the constraint rows) is, and factored by
// Cholesky: for water (a = 3) 2/3 of the charge unknowns remain and the
// constraint rows disappear.  The multipliers follow from the removed rows:
// lambda_k = ((H b)_f - (H K H y)_f) / (-sqrt(a)), f = lo_k.
// ---------------------------------------------------------------------------

// X <- H X on the charge rows, X column-major with leading dimension ld;
// one thread per (block, column), blocks fastest (neighbouring threads touch
// neighbouring rows of one column)
__global__ void reflect_rows(int m, int ncols, int64_t ld, const int32_t *__restrict__ lo,
                             const int32_t *__restrict__ hi, double *__restrict__ X) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= (int64_t)m * ncols) return;
    const int k = (int)(t % m);
    double *col = X + (t / m) * ld;
    const int l = lo[k], h = hi[k];
    const double a = h - l, sa = sqrt(a), beta = 1.0 / (a + sa);
    double w = (1.0 + sa) * col[l];
    for (int i = l + 1; i < h; ++i) w += col[i];
    const double bw = beta * w;
    col[l] -= bw * (1.0 + sa);
    for (int i = l + 1; i < h; ++i) col[i] -= bw;
}

// X <- X H on the charge columns; one thread per (row, block), rows fastest
__global__ void reflect_cols(int nrows, int m, int64_t ld, const int32_t *__restrict__ lo,
                             const int32_t *__restrict__ hi, double *__restrict__ X) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= (int64_t)nrows * m) return;
    const int r = (int)(t % nrows), k = (int)(t / nrows);
    const int l = lo[k], h = hi[k];
    const double a = h - l, sa = sqrt(a), beta = 1.0 / (a + sa);
    double w = (1.0 + sa) * X[l * ld + r];
    for (int j = l + 1; j < h; ++j) w += X[j * ld + r];
    const double bw = beta * w;
    X[l * ld + r] -= bw * (1.0 + sa);
    for (int j = l + 1; j < h; ++j) X[j * ld + r] -= bw;
}

// Kr(p, q) = K(keep_p, keep_q), q < ncols (ncols = nr: the matrix; or right-hand sides)
__global__ void gather_kept(int nr, int ncols, int64_t ld, const int32_t *__restrict__ keep,
                            const double *__restrict__ K, double *__restrict__ Kr, int gather_cols) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= nr) return;
    const int64_t src_row = keep[p];
    for (int q = blockIdx.y; q < ncols; q += gridDim.y) {
        const int64_t src_col = gather_cols ? keep[q] : q;
        Kr[(int64_t)q * nr + p] = K[src_col * ld + src_row];
    }
}

// Y(keep_p, c) = Yr(p, c); the removed rows stay zero
__global__ void scatter_kept(int nr, int ncols, int64_t ld, const int32_t *__restrict__ keep,
                             const double *__restrict__ Yr, double *__restrict__ Y) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= nr) return;
    for (int c = blockIdx.y; c < ncols; c += gridDim.y) Y[(int64_t)c * ld + keep[p]] = Yr[(int64_t)c * nr + p];
}

// multipliers lambda_k of column c, written into the reference-ordered
// variables V (n_var x ncols): V(n + k, c)
__global__ void multipliers(int m, int ncols, int64_t ld, int n, int64_t nv, const int32_t *__restrict__ lo,
                            const int32_t *__restrict__ hi, const double *__restrict__ Bt,
                            const double *__restrict__ Z, double *__restrict__ V) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= (int64_t)m * ncols) return;
    const int k = (int)(t % m), c = (int)(t / m);
    const int64_t f = (int64_t)c * ld + lo[k];
    V[(int64_t)c * nv + n + k] = (Bt[f] - Z[f]) / (-sqrt((double)(hi[k] - lo[k])));
}

// ---------------------------------------------------------------------------
// mixed-precision Cholesky with FP64 iterative refinement (the published
// algorithm of LAPACK's dsposv: factor in single precision, correct in double
// until ||r||_inf < ||x||_inf ||A||_inf eps sqrt(n) for every column, at most
// 30 corrections; otherwise the caller factors in double precision)
// ---------------------------------------------------------------------------

__global__ void to_float(int64_t n, const double *__restrict__ a, float *__restrict__ b) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        b[i] = (float)a[i];
}

__global__ void add_float(int64_t n, const float *__restrict__ d, double *__restrict__ y) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        y[i] += (double)d[i];
}

// out[c] = max_i |A(i, c)|, one block per column
__global__ void col_max_abs(int rows, const double *__restrict__ A, double *__restrict__ out) {
    __shared__ double red[256];
    const double *a = A + (int64_t)blockIdx.x * rows;
    double m = 0.0;
    for (int i = threadIdx.x; i < rows; i += blockDim.x) m = fmax(m, fabs(a[i]));
    red[threadIdx.x] = m;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + w]);
        __syncthreads();
    }
    if (threadIdx.x == 0) out[blockIdx.x] = red[0];
}

// out[c] = sum_i |A(i, c)| (column sums; the row sums of a symmetric matrix)
__global__ void col_sum_abs(int rows, const double *__restrict__ A, double *__restrict__ out) {
    __shared__ double red[256];
    const double *a = A + (int64_t)blockIdx.x * rows;
    double t = 0.0;
    for (int i = threadIdx.x; i < rows; i += blockDim.x) t += fabs(a[i]);
    red[threadIdx.x] = t;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[blockIdx.x] = red[0];
}

// K (n x n, FP64, kept) X = B (n x ncols, right-hand sides in, solutions out);
// false when the single-precision factor fails or the corrections stall
bool mixed_cholesky(plx_ctx *ctx, int n, int ncols, const double *K, double *B, int *iterations) {
    cudaStream_t st = ctx->stream;
    cusolverDnHandle_t h = solver_handle(ctx);
    const int64_t nn = (int64_t)n * n, nb = (int64_t)n * ncols;
    DevArray<float> Kf, Rf, fwork;
    DevArray<double> X, R, B0, norms, colsum;
    DevArray<int32_t> info;
    Kf.alloc(ctx, nn);
    Rf.alloc(ctx, nb);
    X.alloc(ctx, nb);
    R.alloc(ctx, nb);
    B0.alloc(ctx, nb);
    norms.alloc(ctx, 2 * (size_t)ncols);
    colsum.alloc(ctx, n);
    info.alloc(ctx, 1);
    const int grid = (int)std::min<int64_t>(n_blocks(nn, 256), 148 * 16);
    to_float<<<grid, 256, 0, st>>>(nn, K, Kf.p);
    col_sum_abs<<<n, 256, 0, st>>>(n, K, colsum.p);
    ctx->launches += 2;
    PLX_CHECK_CUDA(cudaGetLastError());
    int lwork = 0;
    if (cusolverDnSpotrf_bufferSize(h, CUBLAS_FILL_MODE_LOWER, n, Kf.p, n, &lwork) != CUSOLVER_STATUS_SUCCESS)
        throw Error(PLX_ERR_CUDA, "cusolverDnSpotrf_bufferSize failed");
    fwork.alloc(ctx, std::max(lwork, 1));
    if (cusolverDnSpotrf(h, CUBLAS_FILL_MODE_LOWER, n, Kf.p, n, fwork.p, lwork, info.p) != CUSOLVER_STATUS_SUCCESS)
        throw Error(PLX_ERR_CUDA, "cusolverDnSpotrf failed");
    int hinfo = 0;
    std::vector<double> cs(n);
    PLX_CHECK_CUDA(cudaMemcpyAsync(&hinfo, info.p, 4, cudaMemcpyDeviceToHost, st));
    PLX_CHECK_CUDA(cudaMemcpyAsync(cs.data(), colsum.p, (size_t)n * 8, cudaMemcpyDeviceToHost, st));
    PLX_CHECK_CUDA(cudaStreamSynchronize(st));
    if (hinfo != 0) return false;
    const double anrm = *std::max_element(cs.begin(), cs.end());
    const double cte = anrm * std::ldexp(1.0, -53) * std::sqrt((double)n);
    PLX_CHECK_CUDA(cudaMemcpyAsync(B0.p, B, nb * 8, cudaMemcpyDeviceToDevice, st));
    PLX_CHECK_CUDA(cudaMemsetAsync(X.p, 0, nb * 8, st));
    PLX_CHECK_CUDA(cudaMemcpyAsync(R.p, B, nb * 8, cudaMemcpyDeviceToDevice, st));
    const double one = 1.0, minus = -1.0;
    std::vector<double> hn(2 * (size_t)ncols);
    const int gb = (int)std::min<int64_t>(n_blocks(nb, 256), 148 * 8);
    for (int it = 0; it <= 30; ++it) {
        // correction d = K^-1 r in single precision; x += d; r = b - K x
        to_float<<<gb, 256, 0, st>>>(nb, R.p, Rf.p);
        ctx->launches++;
        if (cusolverDnSpotrs(h, CUBLAS_FILL_MODE_LOWER, n, ncols, Kf.p, n, Rf.p, n, info.p) != CUSOLVER_STATUS_SUCCESS)
            throw Error(PLX_ERR_CUDA, "cusolverDnSpotrs failed");
        add_float<<<gb, 256, 0, st>>>(nb, Rf.p, X.p);
        ctx->launches++;
        PLX_CHECK_CUDA(cudaMemcpyAsync(R.p, B0.p, nb * 8, cudaMemcpyDeviceToDevice, st));
        if (cublasDgemm(blas_handle(ctx), CUBLAS_OP_N, CUBLAS_OP_N, n, ncols, n, &minus, K, n, X.p, n, &one, R.p, n) !=
            CUBLAS_STATUS_SUCCESS)
            throw Error(PLX_ERR_CUDA, "cublasDgemm failed");
        col_max_abs<<<ncols, 256, 0, st>>>(n, R.p, norms.p);
        col_max_abs<<<ncols, 256, 0, st>>>(n, X.p, norms.p + ncols);
        ctx->launches += 2;
        PLX_CHECK_CUDA(cudaGetLastError());
        PLX_CHECK_CUDA(cudaMemcpyAsync(hn.data(), norms.p, hn.size() * 8, cudaMemcpyDeviceToHost, st));
        PLX_CHECK_CUDA(cudaStreamSynchronize(st));
        bool done = true;
        for (int c = 0; c < ncols; ++c) {
            if (!std::isfinite(hn[c]) || !std::isfinite(hn[ncols + c])) return false;
            if (!(hn[c] < hn[ncols + c] * cte) && hn[c] != 0.0) done = false;
        }
        if (done) {
            PLX_CHECK_CUDA(cudaMemcpyAsync(B, X.p, nb * 8, cudaMemcpyDeviceToDevice, st));
            PLX_CHECK_CUDA(cudaStreamSynchronize(st));
            *iterations = it + 1;
            return true;
        }
    }
    return false;
}

// blocks disjoint and inside the charge rows: the elimination applies
bool blocks_disjoint(const std::vector<int32_t> &lo, const std::vector<int32_t> &hi) {
    std::vector<int> order(lo.size());
    for (size_t k = 0; k < order.size(); ++k) order[k] = (int)k;
    std::sort(order.begin(), order.end(), [&](int x, int y) { return lo[x] < lo[y]; });
    for (size_t i = 1; i < order.size(); ++i)
        if (hi[order[i - 1]] > lo[order[i]]) return false;
    return true;
}

}  // namespace

namespace plx {

bool finish_eliminated(plx_ctx *ctx, const StaticDims &s, int N, int nr, int nrhs, const int32_t *d_keep,
                       const int32_t *d_lo, const int32_t *d_hi, const double *K, const double *B, const double *Bt,
                       const double *Br, const double *Rr, double *variables, double *energy, double *polar);

// The constrained solve by elimination (see reflect_rows); false when the
// matrix without the constraint rows is not positive definite (Cholesky
// breaks down), and the caller then factors the full system by LU.
bool solve_eliminated(plx_ctx *ctx, const StaticDims &s, int what, int mode, int potential, double e0, const double *mins,
                      const double *d_pos, const int32_t *d_type, const double *d_par,
                      const std::vector<int32_t> &lo, const std::vector<int32_t> &hi, const int32_t *d_lo,
                      const int32_t *d_hi, double *variables, double *energy, double *polar) {
    cudaStream_t st = ctx->stream;
    const int n = s.n, m = s.n_mol;
    const int N = s.fmu ? 4 * n : n;          // unknowns without the constraint rows
    const int nrhs = what == PLX_STATIC_FIELD ? 3 : 1;
    const int ncols = nrhs + (polar ? 3 : 0);  // the polarizability adds R as right-hand sides
    StaticDims sk = s;
    sk.n_mol = 0;
    sk.n_fq = n;
    sk.n_var = N;
    std::vector<int32_t> keep;
    keep.reserve(N);
    {
        std::vector<char> removed(N, 0);
        for (int k = 0; k < m; ++k) removed[lo[k]] = 1;
        for (int i = 0; i < N; ++i)
            if (!removed[i]) keep.push_back(i);
    }
    const int nr = (int)keep.size();
    DevArray<double> K, Kr, B, Bt, Br, Rr, work;
    DevArray<int32_t> d_keep, info;
    K.alloc(ctx, (size_t)N * N);
    Kr.alloc(ctx, (size_t)nr * nr);
    B.alloc(ctx, (size_t)N * ncols);
    Bt.alloc(ctx, (size_t)N * ncols);
    Br.alloc(ctx, (size_t)nr * ncols);
    d_keep.alloc(ctx, nr);
    PLX_CHECK_CUDA(cudaMemcpyAsync(d_keep.p, keep.data(), (size_t)nr * 4, cudaMemcpyHostToDevice, st));

    prof_begin(ctx);
    const int rows = n_blocks(N, 128);
    static_matrix_kernel<<<dim3(rows, std::min(N, 65535)), 128, 0, st>>>(sk, d_pos, d_type, d_par, d_lo, d_hi, K.p);
    static_rhs_kernel<<<rows, 128, 0, st>>>(sk, what == PLX_STATIC_FIELD, potential, e0, mins[0], mins[1], mins[2],
                                            d_pos, d_type, d_par, B.p);
    ctx->launches += 2;
    PLX_CHECK_CUDA(cudaGetLastError());
    if (polar) {
        // R (n x 3) as three more right-hand sides (FQ: N = n)
        PLX_CHECK_CUDA(cudaMemcpyAsync(B.p + (size_t)nrhs * N, d_pos, (size_t)3 * n * 8, cudaMemcpyDeviceToDevice,
                                       st));
    }
    PLX_CHECK_CUDA(cudaMemcpyAsync(Bt.p, B.p, (size_t)N * ncols * 8, cudaMemcpyDeviceToDevice, st));
    // K <- H K H, B <- H B; then the kept rows and columns
    reflect_rows<<<n_blocks((int64_t)m * N, 128), 128, 0, st>>>(m, N, N, d_lo, d_hi, K.p);
    reflect_cols<<<n_blocks((int64_t)N * m, 128), 128, 0, st>>>(N, m, N, d_lo, d_hi, K.p);
    reflect_rows<<<n_blocks((int64_t)m * ncols, 128), 128, 0, st>>>(m, ncols, N, d_lo, d_hi, Bt.p);
    gather_kept<<<dim3(n_blocks(nr, 128), std::min(nr, 65535)), 128, 0, st>>>(nr, nr, N, d_keep.p, K.p, Kr.p, 1);
    gather_kept<<<dim3(n_blocks(nr, 128), ncols), 128, 0, st>>>(nr, ncols, N, d_keep.p, Bt.p, Br.p, 0);
    ctx->launches += 5;
    PLX_CHECK_CUDA(cudaGetLastError());
    prof_end(ctx, kProfStaticAssembly, 0.0, 8.0 * ((double)N * N + (double)nr * nr + 2.0 * N * ncols));
    if (polar) {
        Rr.alloc(ctx, (size_t)nr * 3);
        PLX_CHECK_CUDA(cudaMemcpyAsync(Rr.p, Br.p + (size_t)nrhs * nr, (size_t)nr * 3 * 8, cudaMemcpyDeviceToDevice,
                                       st));
    }

    const double dr = nr;
    if (mode == 2) {
        // single-precision Cholesky refined in double; Kr stays intact for the
        // double-precision factorisation if the refinement gives up
        prof_begin(ctx);
        int iters = 0;
        const bool ok = mixed_cholesky(ctx, nr, ncols, Kr.p, Br.p, &iters);
        prof_end(ctx, kProfStaticFactor, ok ? dr * dr * dr / 3.0 + iters * 4.0 * dr * dr * ncols : 0.0,
                 ok ? 4.0 * dr * dr : 0.0);
        if (ok) return finish_eliminated(ctx, s, N, nr, nrhs, d_keep.p, d_lo, d_hi, K.p, B.p, Bt.p, Br.p,
                                         Rr.p, variables, energy, polar);
    }
    prof_begin(ctx);
    if (mode == 3) {
        // the hand-written blocked Cholesky (cholesky.cu)
        if (cholesky_factor(ctx, nr, Kr.p) != 0) {
            prof_end(ctx, kProfStaticFactor, 0.0, 0.0);
            return false;  // not positive definite: the caller factors the full system
        }
        cholesky_solve(ctx, nr, Kr.p, ncols, Br.p);
    } else {
        cusolverDnHandle_t h = solver_handle(ctx);
        DevArray<double> work;
        DevArray<int32_t> info;
        int lwork = 0;
        if (cusolverDnDpotrf_bufferSize(h, CUBLAS_FILL_MODE_LOWER, nr, Kr.p, nr, &lwork) != CUSOLVER_STATUS_SUCCESS)
            throw Error(PLX_ERR_CUDA, "cusolverDnDpotrf_bufferSize failed");
        work.alloc(ctx, std::max(lwork, 1));
        info.alloc(ctx, 1);
        if (cusolverDnDpotrf(h, CUBLAS_FILL_MODE_LOWER, nr, Kr.p, nr, work.p, lwork, info.p) != CUSOLVER_STATUS_SUCCESS)
            throw Error(PLX_ERR_CUDA, "cusolverDnDpotrf failed");
        int hinfo = 0;
        PLX_CHECK_CUDA(cudaMemcpyAsync(&hinfo, info.p, 4, cudaMemcpyDeviceToHost, st));
        PLX_CHECK_CUDA(cudaStreamSynchronize(st));
        if (hinfo != 0) {
            prof_end(ctx, kProfStaticFactor, 0.0, 0.0);
            return false;  // not positive definite: the caller factors the full system
        }
        if (cusolverDnDpotrs(h, CUBLAS_FILL_MODE_LOWER, nr, ncols, Kr.p, nr, Br.p, nr, info.p) != CUSOLVER_STATUS_SUCCESS)
            throw Error(PLX_ERR_CUDA, "cusolverDnDpotrs failed");
        check_info(ctx, info, "DPOTRS of the reduced static matrix");
    }
    prof_end(ctx, kProfStaticFactor, dr * dr * dr / 3.0 + 2.0 * dr * dr * ncols, 8.0 * dr * dr);
    return finish_eliminated(ctx, s, N, nr, nrhs, d_keep.p, d_lo, d_hi, K.p, B.p, Bt.p, Br.p, Rr.p, variables,
                             energy, polar);
}

// Back to the original basis after the reduced solve (Br holds the reduced
// solutions, and R^T-side columns for the polarizability after the first nrhs):
// y with the removed rows zero, the multipliers from the removed rows, x = H y,
// the variables in the reference's order, the energy and the polarizability.
bool finish_eliminated(plx_ctx *ctx, const StaticDims &s, int N, int nr, int nrhs, const int32_t *d_keep,
                       const int32_t *d_lo, const int32_t *d_hi, const double *K, const double *B, const double *Bt,
                       const double *Br, const double *Rr, double *variables, double *energy, double *polar) {
    cudaStream_t st = ctx->stream;
    const int n = s.n, m = s.n_mol, nv = s.n_var;
    DevArray<double> Y, Z, V, P;
    Y.alloc(ctx, (size_t)N * nrhs);
    Z.alloc(ctx, (size_t)N * nrhs);
    V.alloc(ctx, (size_t)nv * nrhs);
    PLX_CHECK_CUDA(cudaMemsetAsync(Y.p, 0, (size_t)N * nrhs * 8, st));
    scatter_kept<<<dim3(n_blocks(nr, 128), nrhs), 128, 0, st>>>(nr, nrhs, N, d_keep, Br, Y.p);
    if (nrhs > 3) throw Error(PLX_ERR_ARG, "at most three static right-hand sides");
    {
        DevArray<double> Zp;                                               // Z = (H K H) y
        Zp.alloc(ctx, (size_t)kGemvChunks * nrhs * N);
        dense_gemv_part<<<dim3(n_blocks(N, 128), kGemvChunks), 128, 0, st>>>(N, nrhs, K, Y.p, Zp.p);
        dense_gemv_sum<<<n_blocks((int64_t)N * nrhs, 256), 256, 0, st>>>(N, nrhs, Zp.p, Z.p);
        ctx->launches += 2;
    }
    multipliers<<<n_blocks((int64_t)m * nrhs, 128), 128, 0, st>>>(m, nrhs, N, n, nv, d_lo, d_hi, Bt, Z.p, V.p);
    reflect_rows<<<n_blocks((int64_t)m * nrhs, 128), 128, 0, st>>>(m, nrhs, N, d_lo, d_hi, Y.p);
    ctx->launches += 3;
    PLX_CHECK_CUDA(cudaGetLastError());
    // reference order: charges, multipliers, dipoles
    PLX_CHECK_CUDA(cudaMemcpy2DAsync(V.p, (size_t)nv * 8, Y.p, (size_t)N * 8, (size_t)n * 8, nrhs,
                                     cudaMemcpyDeviceToDevice, st));
    if (N > n)
        PLX_CHECK_CUDA(cudaMemcpy2DAsync(V.p + n + m, (size_t)nv * 8, Y.p + n, (size_t)N * 8, (size_t)(N - n) * 8,
                                         nrhs, cudaMemcpyDeviceToDevice, st));
    if (energy) {
        // the constraint rows' right-hand side is zero: y . b over the N rows
        DevArray<double> dd;
        dd.alloc(ctx, 1);
        small_gemm_tn<<<1, 256, 0, st>>>(1, N, Y.p, N, B, N, dd.p);
        ctx->launches++;
        double dot = 0.0;
        PLX_CHECK_CUDA(cudaMemcpyAsync(&dot, dd.p, 8, cudaMemcpyDeviceToHost, st));
        PLX_CHECK_CUDA(cudaStreamSynchronize(st));
        *energy = -0.5 * dot;
    }
    if (variables)
        PLX_CHECK_CUDA(cudaMemcpyAsync(variables, V.p, (size_t)nv * nrhs * 8, cudaMemcpyDeviceToHost, st));
    if (polar) {
        // R^T Z (Z^T J Z)^-1 Z^T R: the reference's
        // R^T J^-1 R - (L^T J^-1 R)^T (L^T J^-1 L)^-1 (L^T J^-1 R) for disjoint constraints
        P.alloc(ctx, 9);
        gemm_tn(ctx, 3, 3, nr, Rr, nr, Br + (size_t)nrhs * nr, nr, P.p);
        PLX_CHECK_CUDA(cudaMemcpyAsync(polar, P.p, 9 * 8, cudaMemcpyDeviceToHost, st));
    }
    PLX_CHECK_CUDA(cudaStreamSynchronize(st));
    return true;
}

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
    if (d->factorization < 0 || d->factorization > 3) throw Error(PLX_ERR_ARG, "unknown static factorization");
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
    if (d->factorization != 1 && blocks_disjoint(lo, hi) &&
        solve_eliminated(ctx, s, what, d->factorization, d->rhs_potential, d->e0, mins, d_pos.p, d_type.p, d_par.p, lo, hi, d_lo.p,
                         d_hi.p, variables, energy, polar))
        return;
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
