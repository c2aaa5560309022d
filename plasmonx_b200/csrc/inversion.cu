// Direct inversion mode and the polarizability reduction.
//
// complex_inversion (algorithm_module.f90:510-541) factors the dynamic matrix
// A(w) (construct_dynamic_matrix_{wfq,wfqfmu}, wfq_module.f90:214-254,
// wfqfmu_module.f90:436-538) with zgetrf and solves with zgetrs.  Here A(w) is
// assembled on the device from the stored T, the conductance CSR and the
// frequency diagonal, written row-major (which cuSOLVER sees as A^T in
// column-major order), factored with cusolverDnZgetrf and solved with
// cusolverDnZgetrs(op = T).
#include <cublas_v2.h>
#include <cusolverDn.h>

#include <algorithm>

#include "plx_internal.h"

namespace plx {

namespace {

// Row i of A(w) (row-major, complex interleaved), all columns.
// Charge rows: sum_e c_e (T[j_e][col] - T[i][col]); dipole rows: T[r][col];
// plus the diagonal D(w).
__global__ void assemble_rows(int N, int nt, int nv, int f, int hetero, const int32_t *__restrict__ type,
                              const int32_t *__restrict__ rowptr, const int32_t *__restrict__ colidx,
                              const double *__restrict__ kval, const double *__restrict__ ktval,
                              const Cplx *__restrict__ wratio, const Cplx *__restrict__ dq,
                              const double *__restrict__ frac, const Cplx *__restrict__ inv_alpha,
                              const double *__restrict__ T, double2 *__restrict__ A) {
    int r = blockIdx.y;
    int col = blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= nv) return;
    double re = 0.0, im = 0.0;
    Cplx d = {0.0, 0.0};
    if (r < N) {
        int ti = type[r];
        double tic = T[(int64_t)r * nv + col];
        for (int e = rowptr[r]; e < rowptr[r + 1]; ++e) {
            int j = colidx[e];
            double diff = T[(int64_t)j * nv + col] - tic;
            if (!hetero) {
                re += kval[e] * diff;
            } else {
                Cplx w = wratio[ti + nt * type[j] + (int64_t)nt * nt * f];
                double kt = ktval[e];
                re += 0.5 * (kval[e] + w.re * kt) * diff;
                im += 0.5 * (w.im * kt) * diff;
            }
        }
        d = dq[ti + nt * f];
    } else {
        re = T[(int64_t)r * nv + col];
        int i = (r - N) / 3;
        for (int t = 0; t < nt; ++t) {
            double fr = frac[t + (int64_t)nt * i];
            Cplx a = inv_alpha[t + nt * f];
            d.re += fr * a.re;
            d.im += fr * a.im;
        }
    }
    if (col == r) {
        re += d.re;
        im += d.im;
    }
    A[(int64_t)r * nv + col] = make_double2(re, im);
}

__global__ void split_to_interleaved(int n, int count, const double *__restrict__ S,
                                     double2 *__restrict__ Z) {
    int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (int64_t)n * count) return;
    int c = (int)(idx / n), r = (int)(idx % n);
    Z[idx] = make_double2(S[(int64_t)c * 2 * n + r], S[(int64_t)c * 2 * n + n + r]);
}

__global__ void interleaved_to_split(int n, int count, const double2 *__restrict__ Z,
                                     double *__restrict__ S) {
    int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (int64_t)n * count) return;
    int c = (int)(idx / n), r = (int)(idx % n);
    S[(int64_t)c * 2 * n + r] = Z[idx].x;
    S[(int64_t)c * 2 * n + n + r] = Z[idx].y;
}

// alpha(a, pol_c) = sum_i w_i q_i r_ia / E0 (+ sum_i mu_ia / E0), one block per
// (column, a); w_i = 1, or the tessera area for DPCM (calculate_dynamic_polar_bem,
// bem_module.f90:1051-1142).
__global__ void polar_kernel(int N, int nv, int fmu, int area_weight, double e0, const double *__restrict__ pos,
                             const double *__restrict__ X, Cplx *__restrict__ out) {
    int c = blockIdx.y, a = blockIdx.x;
    const double *xr = X + (int64_t)c * 2 * nv, *xi = xr + nv;
    double sr = 0.0, si = 0.0;
    for (int i = threadIdx.x; i < N; i += blockDim.x) {
        double p = pos[(int64_t)a * N + i];
        if (area_weight) {
            double w = pos[3LL * N + i];
            sr += w * xr[i] * p / e0;
            si += w * xi[i] * p / e0;
            continue;
        }
        sr += xr[i] * p / e0;
        si += xi[i] * p / e0;
        if (fmu) {
            sr += xr[N + 3 * i + a] / e0;
            si += xi[N + 3 * i + a] / e0;
        }
    }
    __shared__ double ra[32], rb[32];
    for (int o = 16; o > 0; o >>= 1) {
        sr += __shfl_xor_sync(0xffffffffu, sr, o);
        si += __shfl_xor_sync(0xffffffffu, si, o);
    }
    int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) {
        ra[w] = sr;
        rb[w] = si;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double tr = 0.0, ti = 0.0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) {
            tr += ra[k];
            ti += rb[k];
        }
        out[(int64_t)c * 3 + a] = {tr, ti};
    }
}

struct SolverHandle {
    cusolverDnHandle_t h = nullptr;
};

struct BlasHandle {
    cublasHandle_t h = nullptr;
};

}  // namespace

// One cuSOLVER / cuBLAS handle per host thread, bound to the context's stream
// at every use (contexts are used by one thread at a time).
cusolverDnHandle_t solver_handle(plx_ctx *ctx) {
    static thread_local SolverHandle sh;
    if (!sh.h) {
        if (cusolverDnCreate(&sh.h) != CUSOLVER_STATUS_SUCCESS)
            throw Error(PLX_ERR_CUDA, "cusolverDnCreate failed");
    }
    cusolverDnSetStream(sh.h, ctx->stream);
    return sh.h;
}

cublasHandle_t blas_handle(plx_ctx *ctx) {
    static thread_local BlasHandle bh;
    if (!bh.h && cublasCreate(&bh.h) != CUBLAS_STATUS_SUCCESS) throw Error(PLX_ERR_CUDA, "cublasCreate failed");
    cublasSetStream(bh.h, ctx->stream);
    return bh.h;
}

void bem_dgemm(plx_geom *g, const double *A, const double *B, double *C) {
    cublasHandle_t h = blas_handle(g->ctx);
    const int n = g->n_var;
    const double one = 1.0, zero = 0.0;
    if (cublasDgemm(h, CUBLAS_OP_N, CUBLAS_OP_N, n, n, n, &one, A, n, B, n, &zero, C, n) != CUBLAS_STATUS_SUCCESS)
        throw Error(PLX_ERR_CUDA, "cublasDgemm failed");
}

void polar_batch(plx_geom *g, int count, const int32_t * /*d_pol*/, const double *X, Cplx *d_polar) {
    if (count == 0) return;
    polar_kernel<<<dim3(3, count), 256, 0, g->ctx->stream>>>(g->n_atoms, g->n_var, g->model == PLX_WFQFMU,
                                                            g->model == PLX_BEM_DPCM, g->e0, g->d_pos.p, X,
                                                            d_polar);
    g->ctx->launches++;
    PLX_CHECK_CUDA(cudaGetLastError());
}

// d_vars: [count][2][n] split-complex right-hand sides in, solutions out
// (count = number of columns stored; all are solved).
void solve_inversion_cols(plx_geom *g, int i_freq, int count, double *d_vars) {
    if (!g->has_T) throw Error(PLX_ERR_ARG, "geometry was created without the dense T matrix");
    plx_ctx *ctx = g->ctx;
    cudaStream_t st = ctx->stream;
    const int n = g->n_var;
    DevArray<double2> A, B;
    A.alloc(ctx, (size_t)n * n);
    B.alloc(ctx, (size_t)n * std::max(count, 1));
    // atomistic: A row-major (cuSOLVER sees A^T, solve with op T); BEM: column-major (op N)
    const bool colmajor = is_bem(g);
    if (colmajor) {
        bem_assemble_matrix(g, i_freq, A.p);
    } else {
        assemble_rows<<<dim3(n_blocks(n, 128), n), 128, 0, st>>>(
            g->n_atoms, g->n_types, n, i_freq, g->n_types > 1, g->d_type.p, g->d_rowptr.p, g->d_col.p,
            g->d_kval.p, g->d_ktval.p, g->d_wratio.p, g->d_dq.p, g->d_frac.p, g->d_inv_alpha.p, g->d_T.p,
            A.p);
    }
    split_to_interleaved<<<n_blocks((int64_t)n * count, 256), 256, 0, st>>>(n, count, d_vars, B.p);
    ctx->launches += 2;
    PLX_CHECK_CUDA(cudaGetLastError());
    cusolverDnHandle_t h = solver_handle(ctx);
    int lwork = 0;
    if (cusolverDnZgetrf_bufferSize(h, n, n, reinterpret_cast<cuDoubleComplex *>(A.p), n, &lwork) !=
        CUSOLVER_STATUS_SUCCESS)
        throw Error(PLX_ERR_CUDA, "cusolverDnZgetrf_bufferSize failed");
    DevArray<double2> work;
    DevArray<int32_t> ipiv, info;
    work.alloc(ctx, std::max(lwork, 1));
    ipiv.alloc(ctx, n);
    info.alloc(ctx, 1);
    if (cusolverDnZgetrf(h, n, n, reinterpret_cast<cuDoubleComplex *>(A.p), n,
                         reinterpret_cast<cuDoubleComplex *>(work.p), ipiv.p, info.p) != CUSOLVER_STATUS_SUCCESS)
        throw Error(PLX_ERR_CUDA, "cusolverDnZgetrf failed");
    int hinfo = 0;
    PLX_CHECK_CUDA(cudaMemcpyAsync(&hinfo, info.p, 4, cudaMemcpyDeviceToHost, st));
    PLX_CHECK_CUDA(cudaStreamSynchronize(st));
    if (hinfo != 0) throw Error(PLX_ERR_SINGULAR, "INFO.ne.0 in ZGETRF in complex inversion");
    if (count > 0) {
        // atomistic: the buffer holds A^T (row-major A read column-major): solve A x = b
        if (cusolverDnZgetrs(h, colmajor ? CUBLAS_OP_N : CUBLAS_OP_T, n, count, reinterpret_cast<cuDoubleComplex *>(A.p), n, ipiv.p,
                             reinterpret_cast<cuDoubleComplex *>(B.p), n, info.p) != CUSOLVER_STATUS_SUCCESS)
            throw Error(PLX_ERR_CUDA, "cusolverDnZgetrs failed");
        interleaved_to_split<<<n_blocks((int64_t)n * count, 256), 256, 0, st>>>(n, count, B.p, d_vars);
        ctx->launches++;
    }
    PLX_CHECK_CUDA(cudaMemcpyAsync(&hinfo, info.p, 4, cudaMemcpyDeviceToHost, st));
    PLX_CHECK_CUDA(cudaStreamSynchronize(st));
    if (hinfo != 0) throw Error(PLX_ERR_SINGULAR, "INFO.ne.0 in ZGETRS in complex inversion");
}

}  // namespace plx
