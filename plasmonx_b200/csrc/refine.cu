// Iterative refinement around a lower-precision inner GMRES.
//
// For every column (frequency x polarisation) independently:
//     x = 0, r = b
//     repeat:  stop if ||r|| < tol                      (FP64, same absolute test
//                                                         as gmres_module.f90:207)
//              d ~= A^{-1} r  by GMRES(inner_m) with the inner contraction
//                             (tensor cores), to ||r - A d|| < inner_rel ||r||
//              x += d ;  r = b - A x                    (FP64 operator)
// The inner solves of all active columns run as one batch (one operator
// application per Arnoldi step for the whole batch); the FP64 residuals of all
// active columns are one FP64 contraction.  Each outer step is also a restart,
// so the Krylov memory is bounded by inner_m whatever the conditioning.
#include <algorithm>
#include <cmath>

#include "plx_internal.h"

namespace plx {

namespace {

__global__ void gather_idx(int n, const int32_t *__restrict__ idx, const double *__restrict__ src,
                           double *__restrict__ dst) {
    int k = blockIdx.y;
    const double *s = src + (int64_t)idx[k] * 2 * n;
    double *d = dst + (int64_t)k * 2 * n;
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < 2LL * n; r += (int64_t)gridDim.x * blockDim.x)
        d[r] = s[r];
}

__global__ void scatter_add(int n, const int32_t *__restrict__ idx, const double *__restrict__ src,
                            double *__restrict__ dst) {
    int k = blockIdx.y;
    const double *s = src + (int64_t)k * 2 * n;
    double *d = dst + (int64_t)idx[k] * 2 * n;
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < 2LL * n; r += (int64_t)gridDim.x * blockDim.x)
        d[r] += s[r];
}

// R[idx[k]] = B[idx[k]] - AX[k]
__global__ void scatter_residual(int n, const int32_t *__restrict__ idx, const double *__restrict__ B,
                                 const double *__restrict__ AX, double *__restrict__ R) {
    int k = blockIdx.y;
    int c = idx[k];
    const double *b = B + (int64_t)c * 2 * n;
    const double *a = AX + (int64_t)k * 2 * n;
    double *r = R + (int64_t)c * 2 * n;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < 2LL * n; t += (int64_t)gridDim.x * blockDim.x)
        r[t] = b[t] - a[t];
}

// ||v_c||_2 for every column, one block per column (fixed summation order).
__global__ void column_norms(int n, const double *__restrict__ V, double *__restrict__ out) {
    int c = blockIdx.x;
    const double *v = V + (int64_t)c * 2 * n;
    double s = 0.0;
    for (int64_t t = threadIdx.x; t < 2LL * n; t += blockDim.x) s += v[t] * v[t];
    __shared__ double red[32];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
        out[c] = sqrt(t);
    }
}

int grid_cols(int n) { return std::min(n_blocks(2LL * n, 256), 512); }

}  // namespace

void solve_refined(plx_geom *g, const RefineRequest &rq, const double *d_B, double *d_X, RefineResult &res) {
    plx_ctx *ctx = g->ctx;
    cudaStream_t st = ctx->stream;
    const int n = g->n_var;
    const int C = (int)rq.freq.size();
    res.status.assign(C, PLX_ERR_NOT_CONVERGED);
    res.inner_steps.assign(C, 0);
    res.outer.assign(C, 0);
    res.residual.assign(C, 0.0);
    if (C == 0) return;
    DevArray<double> R, Ba, Da, AXa, nrm;
    DevArray<int32_t> d_idx, d_fa;
    R.alloc(ctx, (size_t)C * 2 * n);
    Ba.alloc(ctx, (size_t)C * 2 * n);
    Da.alloc(ctx, (size_t)C * 2 * n);
    AXa.alloc(ctx, (size_t)C * 2 * n);
    nrm.alloc(ctx, C);
    d_idx.alloc(ctx, C);
    d_fa.alloc(ctx, C);
    PLX_CHECK_CUDA(cudaMemsetAsync(d_X, 0, (size_t)C * 2 * n * 8, st));
    PLX_CHECK_CUDA(cudaMemcpyAsync(R.p, d_B, (size_t)C * 2 * n * 8, cudaMemcpyDeviceToDevice, st));
    std::vector<double> rn(C);
    std::vector<char> live(C, 1);
    for (int outer = 0;; ++outer) {
        TraceRange trace_("refinement step");
        column_norms<<<C, 256, 0, st>>>(n, R.p, nrm.p);
        ctx->launches++;
        PLX_CHECK_CUDA(cudaMemcpyAsync(rn.data(), nrm.p, C * 8, cudaMemcpyDeviceToHost, st));
        PLX_CHECK_CUDA(cudaStreamSynchronize(st));
        std::vector<int32_t> act;
        for (int c = 0; c < C; ++c) {
            if (!live[c]) continue;
            res.residual[c] = rn[c];
            if (!std::isfinite(rn[c])) {
                res.status[c] = PLX_ERR_NAN;
                live[c] = 0;
            } else if (rn[c] < rq.tol) {
                res.status[c] = PLX_OK;
                live[c] = 0;
            } else {
                act.push_back(c);
            }
        }
        if (act.empty() || outer >= rq.max_outer) break;
        const int na = (int)act.size();
        std::vector<int32_t> fa(na);
        GmresRequest in;
        in.m = rq.inner_m;
        in.contraction = rq.inner_contraction;
        in.inner = true;
        in.jacobi = rq.jacobi;
        // a tensor-core inner solve is accurate to ~1e-6 at best: an FP32 basis costs nothing in accuracy
        in.basis_fp32 = rq.inner_contraction == Contraction::TC3 || rq.inner_contraction == Contraction::TC1;
        // one Gram-Schmidt pass keeps an FP32 basis orthogonal enough up to 64 vectors
        // (measured); longer inner solves re-orthogonalise
        in.single_pass = in.basis_fp32 && rq.single_pass_gs && rq.inner_m <= 64;
        for (int k = 0; k < na; ++k) {
            int c = act[k];
            fa[k] = rq.freq[c];
            in.freq.push_back(rq.freq[c]);
            in.pol.push_back(rq.pol[c]);
            // no point asking the inner solve for more than the outer tolerance
            in.tols.push_back(std::max(rq.inner_rel * rn[c], 0.5 * rq.tol));
        }
        PLX_CHECK_CUDA(cudaMemcpyAsync(d_idx.p, act.data(), na * 4, cudaMemcpyHostToDevice, st));
        PLX_CHECK_CUDA(cudaMemcpyAsync(d_fa.p, fa.data(), na * 4, cudaMemcpyHostToDevice, st));
        gather_idx<<<dim3(grid_cols(n), na), 256, 0, st>>>(n, d_idx.p, R.p, Ba.p);
        ctx->launches++;
        GmresResult ir;
        gmres_batched(g, in, Ba.p, Da.p, ir);
        for (int k = 0; k < na; ++k) {
            res.inner_steps[act[k]] += ir.steps[k];
            res.outer[act[k]] += 1;
        }
        scatter_add<<<dim3(grid_cols(n), na), 256, 0, st>>>(n, d_idx.p, Da.p, d_X);
        gather_idx<<<dim3(grid_cols(n), na), 256, 0, st>>>(n, d_idx.p, d_X, Ba.p);
        ctx->launches += 2;
        // FP64 residual of the active columns
        apply_operator(g, OpBatch{na, d_fa.p}, Ba.p, AXa.p, Da.p, rq.outer_contraction);
        scatter_residual<<<dim3(grid_cols(n), na), 256, 0, st>>>(n, d_idx.p, d_B, AXa.p, R.p);
        ctx->launches++;
        PLX_CHECK_CUDA(cudaGetLastError());
    }
    if (g->d_tc_err.p && tc_error(g) != 0)
        throw Error(PLX_ERR_CUDA, "tensor-core contraction timed out waiting on its pipeline");
}

}  // namespace plx
