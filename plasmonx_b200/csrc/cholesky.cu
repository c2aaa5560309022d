// Dense FP64 Cholesky factorisation and solves for the static solve.
//
// The constraint-eliminated static FQ / FQFMu system is symmetric positive
// definite; the reference solves its full (indefinite) form with dsysv
// (real_inversion, algorithm_module.f90:469-504).  Here the reduced matrix is
// factored A = L L^T by a right-looking blocked algorithm, 64 columns per
// panel, three kernels per panel:
//   chol_diag    the 64 x 64 diagonal block, in shared memory (one CTA)
//   chol_panel   the rows below it: L21 = A21 L11^-T, one warp per row
//   chol_update  the trailing lower triangle: A22 -= L21 L21^T, 64 x 64 tiles,
//                4 x 4 outputs per thread, both operands staged in shared memory
// and solved by forward and backward substitution in 64-row blocks (a
// diagonal-block solve in one CTA, then the rows below updated in parallel).
// Matrices are column-major with leading dimension n (only the lower triangle
// is read and written).  A non-positive pivot is reported as its 1-based
// column (LAPACK's info), and the caller falls back to the LU of the full
// system, as with dpotrf.
#include <algorithm>
#include <cmath>

#include "plx_internal.h"

namespace plx {

namespace {

constexpr int NB = 64;

// Factor the diagonal block A[k0:k0+kb, k0:k0+kb] in place (lower).
__global__ void __launch_bounds__(256) chol_diag(int n, int k0, int kb, double *__restrict__ A, int *__restrict__ info) {
    __shared__ double a[NB][NB + 1];
    for (int e = threadIdx.x; e < kb * kb; e += blockDim.x) {
        const int i = e % kb, j = e / kb;
        a[i][j] = i >= j ? A[(int64_t)(k0 + j) * n + k0 + i] : 0.0;
    }
    __syncthreads();
    __shared__ int bad;
    if (threadIdx.x == 0) bad = 0;
    __syncthreads();
    for (int j = 0; j < kb; ++j) {
        if (threadIdx.x == 0) {
            const double d = a[j][j];
            if (!(d > 0.0) && !bad) {
                bad = 1;
                atomicCAS(info, 0, k0 + j + 1);
            }
            a[j][j] = d > 0.0 ? sqrt(d) : 1.0;
        }
        __syncthreads();
        const double djj = a[j][j];
        for (int i = j + 1 + threadIdx.x; i < kb; i += blockDim.x) a[i][j] /= djj;
        __syncthreads();
        // trailing update of the block: a[i][c] -= a[i][j] a[c][j], j < c <= i
        const int m = kb - j - 1;
        for (int e = threadIdx.x; e < m * m; e += blockDim.x) {
            const int i = j + 1 + e % m, c = j + 1 + e / m;
            if (c <= i) a[i][c] -= a[i][j] * a[c][j];
        }
        __syncthreads();
    }
    for (int e = threadIdx.x; e < kb * kb; e += blockDim.x) {
        const int i = e % kb, j = e / kb;
        if (i >= j) A[(int64_t)(k0 + j) * n + k0 + i] = a[i][j];
    }
}

// Rows below the diagonal block: x L11^T = a for every row (one warp per row;
// lane l holds columns l and l + 32).
__global__ void __launch_bounds__(256) chol_panel(int n, int k0, int kb, double *__restrict__ A) {
    __shared__ double l[NB][NB + 1];
    for (int e = threadIdx.x; e < kb * kb; e += blockDim.x) {
        const int i = e % kb, j = e / kb;
        l[i][j] = i >= j ? A[(int64_t)(k0 + j) * n + k0 + i] : 0.0;
    }
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int row = k0 + kb + blockIdx.x * 8 + warp;
    if (row >= n) return;
    double x0 = lane < kb ? A[(int64_t)(k0 + lane) * n + row] : 0.0;
    double x1 = lane + 32 < kb ? A[(int64_t)(k0 + lane + 32) * n + row] : 0.0;
    for (int j = 0; j < kb; ++j) {
        // x_j is final once the columns before it have been subtracted
        const double xj_raw = __shfl_sync(0xffffffffu, j < 32 ? x0 : x1, j & 31);
        const double xj = xj_raw / l[j][j];
        if (lane == (j & 31)) {
            if (j < 32) x0 = xj;
            else x1 = xj;
        }
        if (lane > j && lane < kb) x0 -= xj * l[lane][j];
        if (lane + 32 > j && lane + 32 < kb) x1 -= xj * l[lane + 32][j];
    }
    if (lane < kb) A[(int64_t)(k0 + lane) * n + row] = x0;
    if (lane + 32 < kb) A[(int64_t)(k0 + lane + 32) * n + row] = x1;
}

// A22 -= L21 L21^T on the lower triangle of the trailing matrix; one CTA per
// 64 x 64 tile (tile row >= tile column), 256 threads with 4 x 4 outputs each.
__global__ void __launch_bounds__(256) chol_update(int n, int k0, int kb, double *__restrict__ A) {
    const int t0 = k0 + kb;
    // lower-triangular tile index -> (ti, tj)
    const int t = blockIdx.x;
    int ti = (int)((sqrt(8.0 * t + 1.0) - 1.0) * 0.5);
    while ((ti + 1) * (ti + 2) / 2 <= t) ++ti;
    while (ti * (ti + 1) / 2 > t) --ti;
    const int tj = t - ti * (ti + 1) / 2;
    const int r0 = t0 + ti * NB, c0 = t0 + tj * NB;
    extern __shared__ double chol_sh[];   // 2 x 64 x 65 doubles (66.5 KB, dynamic)
    double (*Ls)[NB + 1] = reinterpret_cast<double (*)[NB + 1]>(chol_sh);              // rows r0.. of L21
    double (*Lt)[NB + 1] = reinterpret_cast<double (*)[NB + 1]>(chol_sh + NB * (NB + 1));  // rows c0..
    for (int e = threadIdx.x; e < NB * kb; e += blockDim.x) {
        const int r = e % NB, k = e / NB;
        Ls[r][k] = r0 + r < n ? A[(int64_t)(k0 + k) * n + r0 + r] : 0.0;
        Lt[r][k] = c0 + r < n ? A[(int64_t)(k0 + k) * n + c0 + r] : 0.0;
    }
    __syncthreads();
    const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;   // rows ty*4.., cols tx + 16 v
    double acc[4][4];
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) acc[u][v] = 0.0;
    for (int k = 0; k < kb; ++k) {
        double a[4], b[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) a[u] = Ls[ty * 4 + u][k];
#pragma unroll
        for (int v = 0; v < 4; ++v) b[v] = Lt[tx + 16 * v][k];
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
            for (int v = 0; v < 4; ++v) acc[u][v] = fma(a[u], b[v], acc[u][v]);
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        const int r = r0 + ty * 4 + u;
        if (r >= n) continue;
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            const int c = c0 + tx + 16 * v;
            if (c < n && c <= r) A[(int64_t)c * n + r] -= acc[u][v];
        }
    }
}

// Forward (lower = 1: L y = b) or backward (lower = 0: L^T x = y) solve of the
// diagonal block k0.. for every right-hand side (one CTA per column).
__global__ void chol_trsv_block(int n, int k0, int kb, int lower, const double *__restrict__ L, double *__restrict__ B) {
    __shared__ double l[NB][NB + 1];
    __shared__ double x[NB];
    for (int e = threadIdx.x; e < kb * kb; e += blockDim.x) {
        const int i = e % kb, j = e / kb;
        l[i][j] = i >= j ? L[(int64_t)(k0 + j) * n + k0 + i] : 0.0;
    }
    double *b = B + (int64_t)blockIdx.x * n;
    for (int i = threadIdx.x; i < kb; i += blockDim.x) x[i] = b[k0 + i];
    __syncthreads();
    if (threadIdx.x == 0) {
        if (lower) {
            for (int i = 0; i < kb; ++i) {
                double s = x[i];
                for (int j = 0; j < i; ++j) s -= l[i][j] * x[j];
                x[i] = s / l[i][i];
            }
        } else {
            for (int i = kb - 1; i >= 0; --i) {
                double s = x[i];
                for (int j = i + 1; j < kb; ++j) s -= l[j][i] * x[j];
                x[i] = s / l[i][i];
            }
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kb; i += blockDim.x) b[k0 + i] = x[i];
}

// After a block is solved: forward -- rows below it: b_r -= sum_k L[r][k0+k] x_k;
// backward -- rows above it: b_r -= sum_k L[k0+k][r] x_k.  One thread per row.
__global__ void chol_trsv_update(int n, int k0, int kb, int lower, const double *__restrict__ L, double *__restrict__ B) {
    __shared__ double x[NB];
    double *b = B + (int64_t)blockIdx.y * n;
    for (int i = threadIdx.x; i < kb; i += blockDim.x) x[i] = b[k0 + i];
    __syncthreads();
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (lower) {
        const int r = k0 + kb + idx;
        if (r >= n) return;
        double s = 0.0;
        for (int k = 0; k < kb; ++k) s += L[(int64_t)(k0 + k) * n + r] * x[k];
        b[r] -= s;
    } else {
        const int r = idx;
        if (r >= k0) return;
        // L^T row r = L column r: entries L[k0 + k][r], contiguous in k
        double s = 0.0;
        for (int k = 0; k < kb; ++k) s += L[(int64_t)r * n + k0 + k] * x[k];
        b[r] -= s;
    }
}

}  // namespace

// A (n x n, column-major, lower triangle) -> L in place.  Returns 0, or the
// 1-based column of the first non-positive pivot.
int cholesky_factor(plx_ctx *ctx, int n, double *A) {
    cudaStream_t st = ctx->stream;
    constexpr int kUpdateSmem = 2 * NB * (NB + 1) * (int)sizeof(double);
    once_per_device(reinterpret_cast<const void *>(chol_update), ctx->device, [] {
        PLX_CHECK_CUDA(cudaFuncSetAttribute(chol_update, cudaFuncAttributeMaxDynamicSharedMemorySize, kUpdateSmem));
    });
    DevArray<int> info;
    info.alloc(ctx, 1);
    PLX_CHECK_CUDA(cudaMemsetAsync(info.p, 0, sizeof(int), st));
    for (int k0 = 0; k0 < n; k0 += NB) {
        const int kb = std::min(NB, n - k0);
        chol_diag<<<1, 256, 0, st>>>(n, k0, kb, A, info.p);
        const int rest = n - k0 - kb;
        if (rest > 0) {
            chol_panel<<<n_blocks(rest, 8), 256, 0, st>>>(n, k0, kb, A);
            const int tiles = (rest + NB - 1) / NB;
            chol_update<<<tiles * (tiles + 1) / 2, 256, kUpdateSmem, st>>>(n, k0, kb, A);
            ctx->launches += 2;
        }
        ctx->launches++;
    }
    PLX_CHECK_CUDA(cudaGetLastError());
    int h = 0;
    PLX_CHECK_CUDA(cudaMemcpyAsync(&h, info.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    PLX_CHECK_CUDA(cudaStreamSynchronize(st));
    return h;
}

// Solves L L^T X = B for nrhs columns of B (n x nrhs, column-major), in place.
void cholesky_solve(plx_ctx *ctx, int n, const double *L, int nrhs, double *B) {
    cudaStream_t st = ctx->stream;
    for (int k0 = 0; k0 < n; k0 += NB) {
        const int kb = std::min(NB, n - k0);
        chol_trsv_block<<<nrhs, 64, 0, st>>>(n, k0, kb, 1, L, B);
        const int rest = n - k0 - kb;
        if (rest > 0) chol_trsv_update<<<dim3(n_blocks(rest, 128), nrhs), 128, 0, st>>>(n, k0, kb, 1, L, B);
        ctx->launches += rest > 0 ? 2 : 1;
    }
    for (int k0 = ((n - 1) / NB) * NB; k0 >= 0; k0 -= NB) {
        const int kb = std::min(NB, n - k0);
        chol_trsv_block<<<nrhs, 64, 0, st>>>(n, k0, kb, 0, L, B);
        if (k0 > 0) chol_trsv_update<<<dim3(n_blocks(k0, 128), nrhs), 128, 0, st>>>(n, k0, kb, 0, L, B);
        ctx->launches += k0 > 0 ? 2 : 1;
    }
    PLX_CHECK_CUDA(cudaGetLastError());
}

}  // namespace plx
