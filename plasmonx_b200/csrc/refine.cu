// Iterative refinement around a lower-precision inner GMRES.
//
// For every column (frequency x polarisation) independently:
//     x = 0, r = b
//     repeat:  stop if ||r|| < tol                      (FP64, same absolute test
//                                                         as gmres_module.f90:207)
//              d ~= A^{-1} r  by restarted GMRES(inner_m) with the inner
//                             contraction (tensor cores), to
//                             ||r - A d|| < inner_rel ||r||
//              x += d ;  r = b - A x                    (FP64 operator)
// The inner solves of all active columns run as one batch (one operator
// application per Arnoldi step for the whole batch); the FP64 residuals of all
// active columns are one FP64 contraction.  The Krylov memory is bounded by
// inner_m whatever the conditioning.  A column whose inner cycle uses the whole
// basis without reaching its inner tolerance restarts from its inner residual
// r - A d formed with the inner (tensor-core) contraction -- one cheap product --
// for up to max_cycles cycles before the outer step pays for an FP64 residual:
// the FP64 product, the expensive one, is then spent once per inner_rel of
// progress instead of once per inner_m Arnoldi steps.
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

// out[k] = B[idx[k]] - AX[k] (compact restart right-hand sides)
__global__ void compact_residual(int n, const int32_t *__restrict__ idx, const double *__restrict__ B,
                                 const double *__restrict__ AX, double *__restrict__ out) {
    int k = blockIdx.y;
    const double *b = B + (int64_t)idx[k] * 2 * n;
    const double *a = AX + (int64_t)k * 2 * n;
    double *o = out + (int64_t)k * 2 * n;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < 2LL * n; t += (int64_t)gridDim.x * blockDim.x)
        o[t] = b[t] - a[t];
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
    DevArray<double> R, Ba, Da, AXa, nrm, Dacc, Bc, Wc;
    DevArray<int32_t> d_idx, d_fa, d_sub, d_fsub;
    R.alloc(ctx, (size_t)C * 2 * n);
    Ba.alloc(ctx, (size_t)C * 2 * n);
    Da.alloc(ctx, (size_t)C * 2 * n);
    AXa.alloc(ctx, (size_t)C * 2 * n);
    nrm.alloc(ctx, C);
    d_idx.alloc(ctx, C);
    d_fa.alloc(ctx, C);
    const int max_cycles = std::max(1, rq.max_cycles);
    if (max_cycles > 1) {
        Dacc.alloc(ctx, (size_t)C * 2 * n);
        Bc.alloc(ctx, (size_t)C * 2 * n);
        Wc.alloc(ctx, (size_t)C * 2 * n);
        d_sub.alloc(ctx, C);
        d_fsub.alloc(ctx, C);
    }
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
        std::vector<double> tol_k(na);
        for (int k = 0; k < na; ++k) {
            int c = act[k];
            fa[k] = rq.freq[c];
            in.freq.push_back(rq.freq[c]);
            in.pol.push_back(rq.pol[c]);
            // no point asking the inner solve for more than the outer tolerance
            tol_k[k] = std::max(rq.inner_rel * rn[c], 0.5 * rq.tol);
            in.tols.push_back(tol_k[k]);
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
        if (max_cycles > 1) {
            // restarts: columns whose cycle ended on the full basis continue from their
            // inner residual; cur[] are positions in act of the columns of the last cycle
            PLX_CHECK_CUDA(cudaMemcpyAsync(Dacc.p, Da.p, (size_t)na * 2 * n * 8, cudaMemcpyDeviceToDevice, st));
            std::vector<int32_t> cur(na);
            for (int k = 0; k < na; ++k) cur[k] = k;
            const double *bc = Ba.p;      // right-hand sides of the last cycle, compact over cur
            for (int cyc = 1; cyc < max_cycles; ++cyc) {
                std::vector<int32_t> sub, pos, fsub;
                for (size_t t = 0; t < cur.size(); ++t)
                    if (ir.status[t] == PLX_ERR_NOT_CONVERGED) {
                        sub.push_back((int32_t)t);
                        pos.push_back(cur[t]);
                        fsub.push_back(fa[cur[t]]);
                    }
                if (sub.empty()) break;
                const int ns = (int)sub.size();
                PLX_CHECK_CUDA(cudaMemcpyAsync(d_sub.p, sub.data(), ns * 4, cudaMemcpyHostToDevice, st));
                PLX_CHECK_CUDA(cudaMemcpyAsync(d_fsub.p, fsub.data(), ns * 4, cudaMemcpyHostToDevice, st));
                // Bc = b_cycle[sub] - A d_cycle[sub]   (inner contraction)
                gather_idx<<<dim3(grid_cols(n), ns), 256, 0, st>>>(n, d_sub.p, Da.p, AXa.p);
                ctx->launches++;
                apply_operator(g, OpBatch{ns, d_fsub.p}, AXa.p, Da.p, Wc.p, rq.inner_contraction);
                compact_residual<<<dim3(grid_cols(n), ns), 256, 0, st>>>(n, d_sub.p, bc, Da.p, AXa.p);
                ctx->launches++;
                PLX_CHECK_CUDA(cudaMemcpyAsync(Bc.p, AXa.p, (size_t)ns * 2 * n * 8, cudaMemcpyDeviceToDevice, st));
                bc = Bc.p;
                GmresRequest rin = in;
                rin.freq.clear();
                rin.pol.clear();
                rin.tols.clear();
                for (int t = 0; t < ns; ++t) {
                    rin.freq.push_back(in.freq[pos[t]]);
                    rin.pol.push_back(in.pol[pos[t]]);
                    rin.tols.push_back(tol_k[pos[t]]);
                }
                ir = GmresResult();
                gmres_batched(g, rin, Bc.p, Da.p, ir);
                PLX_CHECK_CUDA(cudaMemcpyAsync(d_sub.p, pos.data(), ns * 4, cudaMemcpyHostToDevice, st));
                scatter_add<<<dim3(grid_cols(n), ns), 256, 0, st>>>(n, d_sub.p, Da.p, Dacc.p);
                ctx->launches++;
                for (int t = 0; t < ns; ++t) res.inner_steps[act[pos[t]]] += ir.steps[t];
                cur = pos;
            }
            PLX_CHECK_CUDA(cudaMemcpyAsync(Da.p, Dacc.p, (size_t)na * 2 * n * 8, cudaMemcpyDeviceToDevice, st));
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
