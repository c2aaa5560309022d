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
//
// The columns live in slots of a RefineState; an OuterStep advances all of a
// state's active columns by one outer step and can hand out its inner
// operator products one Arnoldi step at a time, so that the outer steps of
// several states (several geometries) share one grouped contraction per step
// (refine_group_step).  solve_refined runs the outer steps of one state to the
// end; the continuous-batching entry points (plx_batch_*) run one outer step at
// a time and add or remove columns between steps.
#include <algorithm>
#include <cmath>
#include <memory>

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

// ||v_idx[k]||_2 for every listed slot, one block per slot (fixed summation order).
__global__ void column_norms(int n, const int32_t *__restrict__ idx, const double *__restrict__ V,
                             double *__restrict__ out) {
    int k = blockIdx.x;
    const double *v = V + (int64_t)idx[k] * 2 * n;
    double s = 0.0;
    for (int64_t t = threadIdx.x; t < 2LL * n; t += blockDim.x) s += v[t] * v[t];
    __shared__ double red[32];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
        out[k] = sqrt(t);
    }
}

int grid_cols(int n) { return std::min(n_blocks(2LL * n, 256), 512); }

}  // namespace

// ---------------------------------------------------------------------------
// RefineState: slots of columns
// ---------------------------------------------------------------------------

void RefineState::attach(plx_geom *geom, const RefineRequest &settings, int n_slots, const double *d_B, double *d_X) {
    g = geom;
    rq = settings;
    cap = n_slots;
    B = d_B;
    X = d_X;
    R.alloc(g->ctx, (size_t)cap * 2 * g->n_var);
    scratch(cap);
    slots.assign(cap, Slot());
}

void RefineState::own(plx_geom *geom, const RefineRequest &settings) {
    g = geom;
    rq = settings;
    cap = 0;
    B = nullptr;
    X = nullptr;
}

void RefineState::scratch(int n_cols) {
    plx_ctx *ctx = g->ctx;
    const size_t count = (size_t)n_cols * 2 * g->n_var;
    Ba.alloc(ctx, count);
    Da.alloc(ctx, count);
    AXa.alloc(ctx, count);
    if (rq.max_cycles > 1) {
        Dacc.alloc(ctx, count);
        Bc.alloc(ctx, count);
        Wc.alloc(ctx, count);
        d_sub.alloc(ctx, n_cols);
        d_fsub.alloc(ctx, n_cols);
    }
    nrm.alloc(ctx, n_cols);
    d_idx.alloc(ctx, n_cols);
    d_fa.alloc(ctx, n_cols);
}

int RefineState::grow(int need) {
    // owned storage only (the continuous-batching state): keeps every slot's data
    if (need <= cap) return cap;
    plx_ctx *ctx = g->ctx;
    const int n = g->n_var;
    const int ncap = std::max(need, std::max(16, 2 * cap));
    DevArray<double> nB, nX, nR;
    nB.alloc(ctx, (size_t)ncap * 2 * n);
    nX.alloc(ctx, (size_t)ncap * 2 * n);
    nR.alloc(ctx, (size_t)ncap * 2 * n);
    if (cap > 0) {
        const size_t b = (size_t)cap * 2 * n * 8;
        PLX_CHECK_CUDA(cudaMemcpyAsync(nB.p, ownB.p, b, cudaMemcpyDeviceToDevice, ctx->stream));
        PLX_CHECK_CUDA(cudaMemcpyAsync(nX.p, ownX.p, b, cudaMemcpyDeviceToDevice, ctx->stream));
        PLX_CHECK_CUDA(cudaMemcpyAsync(nR.p, R.p, b, cudaMemcpyDeviceToDevice, ctx->stream));
    }
    std::swap(ownB.p, nB.p);
    std::swap(ownB.n, nB.n);
    std::swap(ownX.p, nX.p);
    std::swap(ownX.n, nX.n);
    std::swap(R.p, nR.p);
    std::swap(R.n, nR.n);
    nB.ctx = nX.ctx = nR.ctx = ctx;
    ownB.ctx = ownX.ctx = R.ctx = ctx;
    B = ownB.p;
    X = ownX.p;
    cap = ncap;
    slots.resize(cap);
    scratch(cap);
    return cap;
}

void RefineState::update_status() {
    plx_ctx *ctx = g->ctx;
    cudaStream_t st = ctx->stream;
    const int n = g->n_var;
    std::vector<int32_t> idx;
    for (int c = 0; c < cap; ++c)
        if (slots[c].state == Slot::ACTIVE) idx.push_back(c);
    if (idx.empty()) return;
    const int k = (int)idx.size();
    PLX_CHECK_CUDA(cudaMemcpyAsync(d_idx.p, idx.data(), k * 4, cudaMemcpyHostToDevice, st));
    column_norms<<<k, 256, 0, st>>>(n, d_idx.p, R.p, nrm.p);
    ctx->launches++;
    std::vector<double> rn(k);
    PLX_CHECK_CUDA(cudaMemcpyAsync(rn.data(), nrm.p, k * 8, cudaMemcpyDeviceToHost, st));
    PLX_CHECK_CUDA(cudaStreamSynchronize(st));
    for (int t = 0; t < k; ++t) {
        Slot &s = slots[idx[t]];
        s.residual = rn[t];
        if (!std::isfinite(rn[t])) {
            s.status = PLX_ERR_NAN;
            s.state = Slot::FINISHED;
        } else if (rn[t] < s.tol) {
            s.status = PLX_OK;
            s.state = Slot::FINISHED;
        } else if (s.outer >= rq.max_outer) {
            s.status = PLX_ERR_NOT_CONVERGED;
            s.state = Slot::FINISHED;
        }
    }
}

// ---------------------------------------------------------------------------
// OuterStep
// ---------------------------------------------------------------------------

OuterStep::OuterStep(RefineState &s) : s_(s) {}
OuterStep::~OuterStep() = default;

bool OuterStep::begin() {
    RefineState &S = s_;
    plx_geom *g = S.g;
    plx_ctx *ctx = g->ctx;
    cudaStream_t st = ctx->stream;
    const int n = g->n_var;
    S.update_status();
    act_.clear();
    for (int c = 0; c < S.cap; ++c)
        if (S.slots[c].state == RefineState::Slot::ACTIVE) act_.push_back(c);
    if (act_.empty()) return false;
    TraceRange trace_("refinement step");
    const int na = (int)act_.size();
    in_ = GmresRequest();
    in_.m = S.rq.inner_m;
    in_.contraction = S.rq.inner_contraction;
    in_.inner = true;
    in_.jacobi = S.rq.jacobi;
    // a tensor-core inner solve is accurate to ~1e-6 at best: an FP32 basis costs nothing in accuracy
    in_.basis_fp32 = S.rq.inner_contraction == Contraction::TC3 || S.rq.inner_contraction == Contraction::TC1;
    // one Gram-Schmidt pass keeps an FP32 basis orthogonal enough up to 64 vectors
    // (measured); longer inner solves re-orthogonalise
    in_.single_pass = in_.basis_fp32 && S.rq.single_pass_gs && S.rq.inner_m <= 64;
    fa_.assign(na, 0);
    tol_k_.assign(na, 0.0);
    for (int k = 0; k < na; ++k) {
        const RefineState::Slot &sl = S.slots[act_[k]];
        fa_[k] = sl.freq;
        in_.freq.push_back(sl.freq);
        in_.pol.push_back(sl.pol);
        // no point asking the inner solve for more than the outer tolerance
        tol_k_[k] = std::max(S.rq.inner_rel * sl.residual, 0.5 * sl.tol);
        in_.tols.push_back(tol_k_[k]);
    }
    PLX_CHECK_CUDA(cudaMemcpyAsync(S.d_idx.p, act_.data(), na * 4, cudaMemcpyHostToDevice, st));
    PLX_CHECK_CUDA(cudaMemcpyAsync(S.d_fa.p, fa_.data(), na * 4, cudaMemcpyHostToDevice, st));
    gather_idx<<<dim3(grid_cols(n), na), 256, 0, st>>>(n, S.d_idx.p, S.R.p, S.Ba.p);
    ctx->launches++;
    cur_.resize(na);
    for (int k = 0; k < na; ++k) cur_[k] = k;
    cyc_ = 0;
    bc_ = S.Ba.p;
    ir_ = GmresResult();
    run_ = make_gmres(g, in_, S.Ba.p, S.Da.p, ir_);
    done_ = false;
    return true;
}

bool OuterStep::advance(OpInput *need) {
    RefineState &S = s_;
    plx_geom *g = S.g;
    plx_ctx *ctx = g->ctx;
    cudaStream_t st = ctx->stream;
    const int n = g->n_var;
    const int na = (int)act_.size();
    while (!done_) {
        if (run_->wants_product()) {
            *need = run_->pre();
            return true;
        }
        run_->end();
        // a cycle ended: count its steps, keep its correction
        for (size_t t = 0; t < cur_.size(); ++t) S.slots[act_[cur_[t]]].inner_steps += ir_.steps[t];
        if (S.rq.max_cycles > 1) {
            if (cyc_ == 0) {
                PLX_CHECK_CUDA(cudaMemcpyAsync(S.Dacc.p, S.Da.p, (size_t)na * 2 * n * 8, cudaMemcpyDeviceToDevice, st));
            } else {
                PLX_CHECK_CUDA(cudaMemcpyAsync(S.d_sub.p, cur_.data(), cur_.size() * 4, cudaMemcpyHostToDevice, st));
                scatter_add<<<dim3(grid_cols(n), (unsigned)cur_.size()), 256, 0, st>>>(n, S.d_sub.p, S.Da.p,
                                                                                       S.Dacc.p);
                ctx->launches++;
            }
            // restarts: columns whose cycle ended on the full basis continue from
            // their inner residual
            std::vector<int32_t> sub, pos, fsub;
            for (size_t t = 0; t < cur_.size(); ++t)
                if (ir_.status[t] == PLX_ERR_NOT_CONVERGED) {
                    sub.push_back((int32_t)t);
                    pos.push_back(cur_[t]);
                    fsub.push_back(fa_[cur_[t]]);
                }
            if (!sub.empty() && cyc_ + 1 < S.rq.max_cycles) {
                const int ns = (int)sub.size();
                PLX_CHECK_CUDA(cudaMemcpyAsync(S.d_sub.p, sub.data(), ns * 4, cudaMemcpyHostToDevice, st));
                PLX_CHECK_CUDA(cudaMemcpyAsync(S.d_fsub.p, fsub.data(), ns * 4, cudaMemcpyHostToDevice, st));
                // Bc = b_cycle[sub] - A d_cycle[sub]   (inner contraction)
                gather_idx<<<dim3(grid_cols(n), ns), 256, 0, st>>>(n, S.d_sub.p, S.Da.p, S.AXa.p);
                ctx->launches++;
                apply_operator(g, OpBatch{ns, S.d_fsub.p}, S.AXa.p, S.Da.p, S.Wc.p, S.rq.inner_contraction);
                compact_residual<<<dim3(grid_cols(n), ns), 256, 0, st>>>(n, S.d_sub.p, bc_, S.Da.p, S.AXa.p);
                ctx->launches++;
                PLX_CHECK_CUDA(cudaMemcpyAsync(S.Bc.p, S.AXa.p, (size_t)ns * 2 * n * 8, cudaMemcpyDeviceToDevice, st));
                bc_ = S.Bc.p;
                rin_ = in_;
                rin_.freq.clear();
                rin_.pol.clear();
                rin_.tols.clear();
                for (int t = 0; t < ns; ++t) {
                    rin_.freq.push_back(in_.freq[pos[t]]);
                    rin_.pol.push_back(in_.pol[pos[t]]);
                    rin_.tols.push_back(tol_k_[pos[t]]);
                }
                cur_ = pos;
                ++cyc_;
                ir_ = GmresResult();
                run_ = make_gmres(g, rin_, S.Bc.p, S.Da.p, ir_);
                continue;
            }
            PLX_CHECK_CUDA(cudaMemcpyAsync(S.Da.p, S.Dacc.p, (size_t)na * 2 * n * 8, cudaMemcpyDeviceToDevice, st));
        }
        // x += d ; FP64 residual r = b - A x of the active columns
        PLX_CHECK_CUDA(cudaMemcpyAsync(S.d_idx.p, act_.data(), na * 4, cudaMemcpyHostToDevice, st));
        PLX_CHECK_CUDA(cudaMemcpyAsync(S.d_fa.p, fa_.data(), na * 4, cudaMemcpyHostToDevice, st));
        scatter_add<<<dim3(grid_cols(n), na), 256, 0, st>>>(n, S.d_idx.p, S.Da.p, S.X);
        gather_idx<<<dim3(grid_cols(n), na), 256, 0, st>>>(n, S.d_idx.p, S.X, S.Ba.p);
        ctx->launches += 2;
        apply_operator(g, OpBatch{na, S.d_fa.p}, S.Ba.p, S.AXa.p, S.Da.p, S.rq.outer_contraction);
        scatter_residual<<<dim3(grid_cols(n), na), 256, 0, st>>>(n, S.d_idx.p, S.B, S.AXa.p, S.R.p);
        ctx->launches++;
        PLX_CHECK_CUDA(cudaGetLastError());
        for (int c : act_) S.slots[c].outer += 1;
        run_.reset();
        done_ = true;
    }
    return false;
}

void OuterStep::product_done() { run_->post(); }

// ---------------------------------------------------------------------------

void refine_group_step(const std::vector<RefineState *> &states) {
    std::vector<std::unique_ptr<OuterStep>> steps;
    for (RefineState *s : states) {
        auto os = std::make_unique<OuterStep>(*s);
        if (os->begin()) steps.push_back(std::move(os));
    }
    std::vector<OpInput> need;
    std::vector<OuterStep *> who;
    for (;;) {
        need.clear();
        who.clear();
        for (auto &os : steps) {
            OpInput in{};
            if (os->advance(&in)) {
                need.push_back(in);
                who.push_back(os.get());
            }
        }
        if (need.empty()) break;
        apply_operator_group(need);
        for (OuterStep *os : who) os->product_done();
    }
}

void solve_refined(plx_geom *g, const RefineRequest &rq, const double *d_B, double *d_X, RefineResult &res) {
    plx_ctx *ctx = g->ctx;
    const int n = g->n_var;
    const int C = (int)rq.freq.size();
    res.status.assign(C, PLX_ERR_NOT_CONVERGED);
    res.inner_steps.assign(C, 0);
    res.outer.assign(C, 0);
    res.residual.assign(C, 0.0);
    if (C == 0) return;
    RefineState S;
    S.attach(g, rq, C, d_B, d_X);
    for (int c = 0; c < C; ++c) {
        RefineState::Slot &sl = S.slots[c];
        sl.state = RefineState::Slot::ACTIVE;
        sl.freq = rq.freq[c];
        sl.pol = rq.pol[c];
        sl.tol = rq.tol;
    }
    PLX_CHECK_CUDA(cudaMemsetAsync(d_X, 0, (size_t)C * 2 * n * 8, ctx->stream));
    PLX_CHECK_CUDA(cudaMemcpyAsync(S.R.p, d_B, (size_t)C * 2 * n * 8, cudaMemcpyDeviceToDevice, ctx->stream));
    for (;;) {
        OuterStep os(S);
        if (!os.begin()) break;
        OpInput need{};
        while (os.advance(&need)) {
            apply_operator(need.g, need.b, need.X, need.Y, need.work, need.how);
            os.product_done();
        }
    }
    for (int c = 0; c < C; ++c) {
        const RefineState::Slot &sl = S.slots[c];
        res.status[c] = sl.state == RefineState::Slot::FINISHED ? sl.status : PLX_ERR_NOT_CONVERGED;
        res.inner_steps[c] = sl.inner_steps;
        res.outer[c] = sl.outer;
        res.residual[c] = sl.residual;
    }
    if (g->d_tc_err.p && tc_error(g) != 0)
        throw Error(PLX_ERR_CUDA, "tensor-core contraction timed out waiting on its pipeline");
}

}  // namespace plx
