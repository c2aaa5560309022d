// C ABI of plasmonx_b200 (declared in include/plasmonx_b200.h).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <vector>

#include "plx_internal.h"

using namespace plx;

// ---------------------------------------------------------------------------
// device memory: stream-ordered allocations on the context's stream, charged
// against the context's HBM budget
// ---------------------------------------------------------------------------
void *plx::dev_alloc(plx_ctx *ctx, size_t bytes) {
    if (ctx->budget && ctx->in_use + bytes > ctx->budget)
        throw Error(PLX_ERR_BUDGET, "device allocation of " + std::to_string(bytes) +
                                        " bytes exceeds the HBM budget (" + std::to_string(ctx->in_use) +
                                        " of " + std::to_string(ctx->budget) + " in use)");
    void *p = nullptr;
    cudaError_t e = cudaMallocAsync(&p, bytes, ctx->stream);
    if (e == cudaErrorMemoryAllocation) {
        // the stream-ordered pool keeps freed blocks (release threshold: never), so
        // blocks of other sizes can hold the memory a new size needs: wait for this
        // stream's frees, hand every unused block back to the device, retry once
        cudaGetLastError();
        cudaStreamSynchronize(ctx->stream);
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, ctx->device) == cudaSuccess) cudaMemPoolTrimTo(pool, 0);
        e = cudaMallocAsync(&p, bytes, ctx->stream);
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        throw Error(PLX_ERR_NOMEM, "cudaMallocAsync(" + std::to_string(bytes) + "): " + cudaGetErrorString(e));
    }
    ctx->in_use += bytes;
    return p;
}

void plx::dev_free(plx_ctx *ctx, void *p, size_t bytes) {
    cudaFreeAsync(p, ctx->stream);
    ctx->in_use -= bytes;
}

namespace {

template <typename F>
plx_status guarded(plx_ctx *ctx, F &&f) {
    try {
        f();
        return PLX_OK;
    } catch (const Error &e) {
        if (ctx) ctx->last_error = e.msg;
        return e.code;
    } catch (const std::exception &e) {
        if (ctx) ctx->last_error = e.what();
        return PLX_ERR_ARG;
    }
}

void set_device(plx_ctx *ctx) { PLX_CHECK_CUDA(cudaSetDevice(ctx->device)); }

// host interleaved complex (n) <-> device split [2][n]
void upload_vec(plx_ctx *ctx, const double *h, int64_t n, double *d) {
    std::vector<double> s(2 * n);
    for (int64_t r = 0; r < n; ++r) {
        s[r] = h[2 * r];
        s[n + r] = h[2 * r + 1];
    }
    PLX_CHECK_CUDA(cudaMemcpyAsync(d, s.data(), 2 * n * 8, cudaMemcpyHostToDevice, ctx->stream));
    PLX_CHECK_CUDA(cudaStreamSynchronize(ctx->stream));
}

void download_vec(plx_ctx *ctx, const double *d, int64_t n, double *h) {
    std::vector<double> s(2 * n);
    PLX_CHECK_CUDA(cudaMemcpyAsync(s.data(), d, 2 * n * 8, cudaMemcpyDeviceToHost, ctx->stream));
    PLX_CHECK_CUDA(cudaStreamSynchronize(ctx->stream));
    for (int64_t r = 0; r < n; ++r) {
        h[2 * r] = s[r];
        h[2 * r + 1] = s[n + r];
    }
}

// any(real(b(:,c)) > 1e-15): the reference solves a GMRES column only then
// (complex_gmres_iterative, algorithm_module.f90:568-585).
__global__ void positive_real_flags(int n, int count, const double *__restrict__ B, int *__restrict__ flag) {
    int c = blockIdx.y;
    const double *b = B + (int64_t)c * 2 * n;
    int hit = 0;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x)
        hit |= b[r] > 1.0e-15;
    hit = __syncthreads_or(hit);
    if (threadIdx.x == 0 && hit) flag[c] = 1;
}

__global__ void copy_cols(int n, const int32_t *__restrict__ src_idx, const int32_t *__restrict__ dst_idx,
                          const double *__restrict__ S, double *__restrict__ D) {
    int k = blockIdx.y;
    const double *s = S + (int64_t)src_idx[k] * 2 * n;
    double *d = D + (int64_t)dst_idx[k] * 2 * n;
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < 2LL * n;
         r += (int64_t)gridDim.x * blockDim.x)
        d[r] = s[r];
}

void results_row(const Cplx *P /* 3x3, (a,b) at a+3b */, double w, double *r) {
    const double pi = 4.0 * std::atan(1.0), light = 137.035227;
    r[0] = (P[0].re + P[4].re + P[8].re) / 3;
    r[1] = (P[0].im + P[4].im + P[8].im) / 3;
    r[2] = P[0].re;
    r[3] = P[4].re;
    r[4] = P[8].re;
    r[5] = P[0].im;
    r[6] = P[4].im;
    r[7] = P[8].im;
    double m_iso = r[0] * r[0] + r[1] * r[1];
    double mx = r[2] * r[2] + r[5] * r[5], my = r[3] * r[3] + r[6] * r[6], mz = r[4] * r[4] + r[7] * r[7];
    r[8] = 4.0 * pi * w * r[1] / light;
    r[9] = 4.0 * pi * w * r[5] / light;
    r[10] = 4.0 * pi * w * r[6] / light;
    r[11] = 4.0 * pi * w * r[7] / light;
    double c4 = 3.0 * std::pow(light, 4);
    double w4 = 8.0 * pi * std::pow(w, 4);
    r[12] = w4 * m_iso / c4;
    r[13] = w4 * mx / c4;
    r[14] = w4 * my / c4;
    r[15] = w4 * mz / c4;
    r[16] = r[8] + r[12];
    r[17] = r[9] + r[13];
    r[18] = r[10] + r[14];
    r[19] = r[11] + r[15];
}

}  // namespace

extern "C" {

plx_ctx *plx_ctx_create(int32_t device, uint64_t hbm_budget_bytes) {
    plx_ctx *ctx = new (std::nothrow) plx_ctx();
    if (!ctx) return nullptr;
    ctx->device = device;
    plx_status s = guarded(ctx, [&] {
        PLX_CHECK_CUDA(cudaSetDevice(device));
        PLX_CHECK_CUDA(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
        PLX_CHECK_CUDA(cudaEventCreate(&ctx->ev0));
        PLX_CHECK_CUDA(cudaEventCreate(&ctx->ev1));
        size_t fr = 0, tot = 0;
        PLX_CHECK_CUDA(cudaMemGetInfo(&fr, &tot));
        ctx->budget = hbm_budget_bytes ? hbm_budget_bytes : (uint64_t)fr;
        // keep freed blocks in the stream-ordered pool for reuse within this process
        cudaMemPool_t pool;
        PLX_CHECK_CUDA(cudaDeviceGetDefaultMemPool(&pool, device));
        uint64_t thr = UINT64_MAX;
        PLX_CHECK_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr));
    });
    if (s != PLX_OK) ctx->budget = 0;
    return ctx;
}

void plx_ctx_destroy(plx_ctx *ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    if (ctx->ev0) cudaEventDestroy(ctx->ev0);
    if (ctx->ev1) cudaEventDestroy(ctx->ev1);
    for (cudaEvent_t e : ctx->prof_events) cudaEventDestroy(e);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    // the pool keeps freed blocks for reuse; a closed context's blocks go back to
    // the device, so that what it held is free for other contexts and processes
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, ctx->device) == cudaSuccess) cudaMemPoolTrimTo(pool, 0);
    delete ctx;
}

const char *plx_last_error(const plx_ctx *ctx) { return ctx ? ctx->last_error.c_str() : "null context"; }

uint64_t plx_ctx_bytes_in_use(const plx_ctx *ctx) { return ctx ? ctx->in_use : 0; }

int64_t plx_ctx_launches(const plx_ctx *ctx) { return ctx ? ctx->launches : -1; }

plx_status plx_geometry_create(plx_ctx *ctx, const plx_geometry_desc *d, int32_t store_t, plx_geom **out) {
    TraceRange trace_("plx_geometry_create");
    if (!ctx || !d || !out) return PLX_ERR_ARG;
    *out = nullptr;
    plx_geom *g = new plx_geom();
    plx_status s = guarded(ctx, [&] {
        if (!ctx->stream) throw Error(PLX_ERR_CUDA, "context has no CUDA stream: " + ctx->last_error);
        set_device(ctx);
        if (d->model != PLX_WFQ && d->model != PLX_WFQFMU) throw Error(PLX_ERR_UNSUPPORTED, "unknown model");
        if (d->n_atoms < 1 || d->n_types < 1) throw Error(PLX_ERR_ARG, "n_atoms and n_types must be positive");
        if (!d->coord || !d->atom_type || !d->neighbours || !d->n_neighbours || !d->eta || !d->r_q ||
            !d->tau || !d->density || !d->a_ij || !d->fermi_d || !d->fermi_s || !d->r0)
            throw Error(PLX_ERR_ARG, "null array in geometry description");
        if (d->model == PLX_WFQFMU && !d->r_mu) throw Error(PLX_ERR_ARG, "r_mu is required for wFQFMu");
        if (d->model == PLX_WFQ && d->n_types > 1)
            throw Error(PLX_ERR_UNSUPPORTED, "heterogeneous wFQ is not provided (the reference builds no "
                                             "charge block for it)");
        const int N = d->n_atoms, nt = d->n_types;
        g->ctx = ctx;
        g->model = d->model;
        g->n_atoms = N;
        g->n_types = nt;
        g->n_var = d->model == PLX_WFQFMU ? 4 * N : N;
        if ((int64_t)g->n_var > INT32_MAX / 2) throw Error(PLX_ERR_ARG, "too many unknowns");
        g->rhs_potential = d->rhs_potential;
        g->e0 = d->e0;
        g->coord.assign(d->coord, d->coord + 3 * N);
        g->atom_type.assign(d->atom_type, d->atom_type + N);
        for (int i = 0; i < N; ++i)
            if (g->atom_type[i] < 0 || g->atom_type[i] >= nt) throw Error(PLX_ERR_ARG, "atom_type out of range");
        auto cp = [&](std::vector<double> &v, const double *p, int cnt) { v.assign(p, p + cnt); };
        cp(g->eta, d->eta, nt);
        cp(g->r_q, d->r_q, nt);
        if (d->r_mu) cp(g->r_mu, d->r_mu, nt);
        else g->r_mu.assign(nt, 1.0);
        cp(g->tau, d->tau, nt);
        cp(g->density, d->density, nt);
        cp(g->a_ij, d->a_ij, nt);
        cp(g->fermi_d, d->fermi_d, nt * nt);
        cp(g->fermi_s, d->fermi_s, nt * nt);
        cp(g->r0, d->r0, nt * nt);
        g->frac.resize((size_t)nt * N);
        for (int i = 0; i < N; ++i)
            for (int t = 0; t < nt; ++t)
                g->frac[t + (size_t)nt * i] = (double)d->neighbours[t + (size_t)nt * i] / (double)d->n_neighbours[i];
        std::vector<double> pos(4 * (size_t)N, 0.0), par(4 * (size_t)N, 0.0);
        for (int i = 0; i < N; ++i) {
            int t = g->atom_type[i];
            for (int k = 0; k < 3; ++k) pos[(size_t)k * N + i] = g->coord[k + 3 * (size_t)i];
            par[i] = g->r_q[t];
            par[N + i] = g->r_mu[t];
            par[2 * (size_t)N + i] = g->eta[t];
            par[3 * (size_t)N + i] = g->a_ij[t];
        }
        cudaStream_t st = ctx->stream;
        g->d_pos.alloc(ctx, 4 * (size_t)N);
        g->d_par.alloc(ctx, 4 * (size_t)N);
        g->d_type.alloc(ctx, N);
        g->d_frac.alloc(ctx, (size_t)nt * N);
        PLX_CHECK_CUDA(cudaMemcpyAsync(g->d_pos.p, pos.data(), pos.size() * 8, cudaMemcpyHostToDevice, st));
        PLX_CHECK_CUDA(cudaMemcpyAsync(g->d_par.p, par.data(), par.size() * 8, cudaMemcpyHostToDevice, st));
        PLX_CHECK_CUDA(cudaMemcpyAsync(g->d_type.p, g->atom_type.data(), N * 4, cudaMemcpyHostToDevice, st));
        PLX_CHECK_CUDA(cudaMemcpyAsync(g->d_frac.p, g->frac.data(), g->frac.size() * 8, cudaMemcpyHostToDevice, st));
        build_conductance(g);
        if (store_t) build_dense_t(g);
    });
    if (s != PLX_OK) {
        delete g;
        return s;
    }
    *out = g;
    return PLX_OK;
}


plx_status plx_bem_create(plx_ctx *ctx, const plx_bem_desc *d, plx_geom **out) {
    TraceRange trace_("plx_bem_create");
    if (!ctx || !d || !out) return PLX_ERR_ARG;
    *out = nullptr;
    plx_geom *g = new plx_geom();
    plx_status s = guarded(ctx, [&] {
        if (!ctx->stream) throw Error(PLX_ERR_CUDA, "context has no CUDA stream: " + ctx->last_error);
        set_device(ctx);
        if (d->variant != PLX_BEM_DPCM && d->variant != PLX_BEM_IEF) throw Error(PLX_ERR_ARG, "unknown BEM variant");
        if (d->n_tess < 1 || !d->triangles) throw Error(PLX_ERR_ARG, "no tesserae");
        if (d->n_tess > 65535) throw Error(PLX_ERR_UNSUPPORTED, "more than 65535 tesserae");
        if (!d->accurate && !(d->sphere_radius > 0.0))
            throw Error(PLX_ERR_ARG, "the approximate Green function needs a positive sphere radius");
        g->ctx = ctx;
        g->model = d->variant;
        g->n_atoms = d->n_tess;
        g->n_var = d->n_tess;
        g->n_types = 1;
        g->e0 = d->e0;
        g->eps_solvent = d->eps_solvent;
        build_bem(g, d->triangles, d->normal_factor, d->sphere_radius, d->accurate);
    });
    if (s != PLX_OK) {
        delete g;
        return s;
    }
    *out = g;
    return PLX_OK;
}

void plx_geometry_destroy(plx_geom *g) {
    if (!g) return;
    if (g->ctx) cudaSetDevice(g->ctx->device);
    delete g;
}

int64_t plx_geometry_n_var(const plx_geom *g) { return g ? g->n_var : 0; }
int64_t plx_geometry_k_nnz(const plx_geom *g) { return g ? g->nnz : 0; }

plx_status plx_set_frequencies(plx_geom *g, int32_t n_freq, const double *omega, const double *alpha_w) {
    if (!g) return PLX_ERR_ARG;
    return guarded(g->ctx, [&] {
        set_device(g->ctx);
        if (n_freq < 1 || !omega) throw Error(PLX_ERR_ARG, "need at least one frequency");
        if (g->open_batches > 0) throw Error(PLX_ERR_ARG, "the geometry's frequencies belong to its open batch");
        if (g->model == PLX_WFQFMU && !alpha_w) throw Error(PLX_ERR_ARG, "alpha_w is required for wFQFMu");
        if (is_bem(g) && !alpha_w) throw Error(PLX_ERR_ARG, "eps(w) (alpha_w) is required for BEM");
        g->n_freq = n_freq;
        g->omega.assign(omega, omega + n_freq);
        g->alpha_w.clear();
        if (alpha_w) {
            g->alpha_w.resize((size_t)g->n_types * n_freq);
            for (size_t e = 0; e < g->alpha_w.size(); ++e) g->alpha_w[e] = {alpha_w[2 * e], alpha_w[2 * e + 1]};
        }
        upload_frequency_tables(g);
    });
}

plx_status plx_matvec(plx_geom *g, int32_t i_freq, int32_t on_the_fly, const double *x, double *y) {
    if (!g || !x || !y) return PLX_ERR_ARG;
    return guarded(g->ctx, [&] {
        set_device(g->ctx);
        if (i_freq < 0 || i_freq >= g->n_freq) throw Error(PLX_ERR_ARG, "frequency index out of range");
        const int n = g->n_var;
        DevArray<double> X, Y, W;
        DevArray<int32_t> F;
        X.alloc(g->ctx, 2 * (size_t)n);
        Y.alloc(g->ctx, 2 * (size_t)n);
        W.alloc(g->ctx, 2 * (size_t)n);
        F.alloc(g->ctx, 1);
        PLX_CHECK_CUDA(cudaMemcpyAsync(F.p, &i_freq, 4, cudaMemcpyHostToDevice, g->ctx->stream));
        upload_vec(g->ctx, x, n, X.p);
        apply_operator(g, OpBatch{1, F.p}, X.p, Y.p, W.p, on_the_fly ? Contraction::FP64_OTF : Contraction::FP64);
        download_vec(g->ctx, Y.p, n, y);
    });
}

plx_status plx_field_at_points(plx_geom *g, int32_t i_pol, const double *x, int32_t n_points, const double *points,
                               double *field_out, double *density_out) {
    if (!g || !x || !points || n_points < 0) return PLX_ERR_ARG;
    return guarded(g->ctx, [&] {
        TraceRange trace_("plx_field_at_points");
        set_device(g->ctx);
        if (is_bem(g)) throw Error(PLX_ERR_UNSUPPORTED, "field at points: atomistic models only");
        if (i_pol < 0 || i_pol > 2) throw Error(PLX_ERR_ARG, "polarisation index must be 0, 1 or 2");
        if (n_points == 0) return;
        cudaStream_t st = g->ctx->stream;
        DevArray<double> X, P, Fd, D;
        X.alloc(g->ctx, 2 * (size_t)g->n_var);
        P.alloc(g->ctx, 3 * (size_t)n_points);
        Fd.alloc(g->ctx, 6 * (size_t)n_points);
        D.alloc(g->ctx, 2 * (size_t)n_points);
        // x stays interleaved complex; points to [3][P]
        std::vector<double> pts(3 * (size_t)n_points);
        for (int64_t i = 0; i < n_points; ++i)
            for (int k = 0; k < 3; ++k) pts[(size_t)k * n_points + i] = points[3 * i + k];
        PLX_CHECK_CUDA(cudaMemcpyAsync(X.p, x, 2 * (size_t)g->n_var * 8, cudaMemcpyHostToDevice, st));
        PLX_CHECK_CUDA(cudaMemcpyAsync(P.p, pts.data(), pts.size() * 8, cudaMemcpyHostToDevice, st));
        field_at_points(g, i_pol, X.p, n_points, P.p, Fd.p, D.p);
        if (field_out)
            PLX_CHECK_CUDA(cudaMemcpyAsync(field_out, Fd.p, 6 * (size_t)n_points * 8, cudaMemcpyDeviceToHost, st));
        if (density_out)
            PLX_CHECK_CUDA(cudaMemcpyAsync(density_out, D.p, 2 * (size_t)n_points * 8, cudaMemcpyDeviceToHost, st));
        PLX_CHECK_CUDA(cudaStreamSynchronize(st));
    });
}

plx_status plx_bem_field_at_points(plx_ctx *ctx, int32_t n_tess, const double *centres, const double *q, double e0,
                                   int32_t i_pol, int32_t n_points, const double *points, double *field_out) {
    if (!ctx) return PLX_ERR_ARG;
    return guarded(ctx, [&] {
        TraceRange trace_("plx_bem_field_at_points");
        set_device(ctx);
        bem_field_at_points(ctx, n_tess, centres, q, e0, i_pol, n_points, points, field_out);
    });
}

plx_status plx_neighbour_counts(plx_ctx *ctx, int32_t n_atoms, int32_t n_types, const double *coord_ang,
                                const int32_t *atom_type, const int32_t *type_z, const double *r0,
                                int32_t *neighbours_out, int32_t *n_neighbours_out) {
    if (!ctx) return PLX_ERR_ARG;
    return guarded(ctx, [&] {
        TraceRange trace_("plx_neighbour_counts");
        set_device(ctx);
        neighbour_counts(ctx, n_atoms, n_types, coord_ang, atom_type, type_z, r0, neighbours_out, n_neighbours_out);
    });
}

int64_t plx_static_n_var(const plx_static_desc *desc) { return static_n_var(desc); }

plx_status plx_static_solve(plx_ctx *ctx, const plx_static_desc *desc, int32_t what, double *variables,
                            double *energy, double *polar) {
    if (!ctx || !desc) return PLX_ERR_ARG;
    return guarded(ctx, [&] {
        TraceRange trace_("plx_static_solve");
        set_device(ctx);
        static_solve(ctx, desc, what, variables, energy, polar);
    });
}

plx_status plx_principal_axes(int32_t n_atoms, const int32_t *atomic_number, double *coord, double *eigenvalues,
                              double *axes) {
    return guarded(nullptr, [&] { principal_axes(n_atoms, atomic_number, coord, eigenvalues, axes); });
}

plx_status plx_rhs(plx_geom *g, int32_t i_freq, int32_t pol_mask, double *b) {
    if (!g || !b) return PLX_ERR_ARG;
    return guarded(g->ctx, [&] {
        set_device(g->ctx);
        if (i_freq < 0 || i_freq >= g->n_freq) throw Error(PLX_ERR_ARG, "frequency index out of range");
        const int n = g->n_var;
        std::memset(b, 0, sizeof(double) * 2 * (size_t)n * 3);
        std::vector<int32_t> pols, fr;
        for (int p = 0; p < 3; ++p)
            if (pol_mask & (1 << p)) {
                pols.push_back(p);
                fr.push_back(i_freq);
            }
        int C = (int)pols.size();
        if (!C) return;
        DevArray<double> B;
        DevArray<int32_t> dP, dF;
        B.alloc(g->ctx, (size_t)C * 2 * n);
        dP.alloc(g->ctx, C);
        dF.alloc(g->ctx, C);
        PLX_CHECK_CUDA(cudaMemcpyAsync(dP.p, pols.data(), C * 4, cudaMemcpyHostToDevice, g->ctx->stream));
        PLX_CHECK_CUDA(cudaMemcpyAsync(dF.p, fr.data(), C * 4, cudaMemcpyHostToDevice, g->ctx->stream));
        rhs_batch(g, OpBatch{C, dF.p}, dP.p, B.p);
        for (int c = 0; c < C; ++c) download_vec(g->ctx, B.p + (size_t)c * 2 * n, n, b + 2 * (size_t)n * pols[c]);
    });
}

plx_status plx_gmres_solver(plx_geom *g, int32_t i_freq, double *x, int32_t on_the_fly, double tol,
                            int32_t max_iter, int32_t restart, int32_t *steps_out, double *trace_out) {
    if (!g || !x) return PLX_ERR_ARG;
    plx_status conv = PLX_OK;
    plx_status s = guarded(g->ctx, [&] {
        TraceRange trace_("plx_gmres_solver");
        set_device(g->ctx);
        if (i_freq < 0 || i_freq >= g->n_freq) throw Error(PLX_ERR_ARG, "frequency index out of range");
        (void)max_iter;   // no restart: the reference errors after the first cycle
        const int n = g->n_var;
        DevArray<double> B, X;
        B.alloc(g->ctx, 2 * (size_t)n);
        X.alloc(g->ctx, 2 * (size_t)n);
        upload_vec(g->ctx, x, n, B.p);
        GmresRequest rq;
        rq.freq = {i_freq};
        rq.pol = {0};
        rq.m = restart;
        rq.tol = tol;
        rq.contraction = on_the_fly ? Contraction::FP64_OTF : Contraction::FP64;
        rq.record_trace = trace_out != nullptr;
        GmresResult res;
        gmres_batched(g, rq, B.p, X.p, res);
        download_vec(g->ctx, X.p, n, x);
        if (steps_out) *steps_out = res.steps[0];
        if (trace_out) std::copy(res.trace.begin(), res.trace.begin() + res.steps[0], trace_out);
        conv = (plx_status)res.status[0];
        if (conv == PLX_ERR_NOT_CONVERGED) g->ctx->last_error = "GMRES not converged and restart GMRES NYI.";
    });
    return s != PLX_OK ? s : conv;
}

plx_status plx_complex_inversion(plx_geom *g, int32_t i_freq, double *variables_w) {
    if (!g || !variables_w) return PLX_ERR_ARG;
    return guarded(g->ctx, [&] {
        TraceRange trace_("plx_complex_inversion");
        set_device(g->ctx);
        if (i_freq < 0 || i_freq >= g->n_freq) throw Error(PLX_ERR_ARG, "frequency index out of range");
        const int n = g->n_var;
        DevArray<double> V;
        V.alloc(g->ctx, 3 * 2 * (size_t)n);
        for (int c = 0; c < 3; ++c) upload_vec(g->ctx, variables_w + 2 * (size_t)n * c, n, V.p + (size_t)c * 2 * n);
        bool done = false;
        if (hessenberg_applies(g, 3)) {
            DevArray<double> Xh;
            Xh.alloc(g->ctx, 3 * 2 * (size_t)n);
            done = hessenberg_solve(g, {i_freq}, 3, V.p, Xh.p);
            if (done)
                PLX_CHECK_CUDA(cudaMemcpyAsync(V.p, Xh.p, 3 * 2 * (size_t)n * 8, cudaMemcpyDeviceToDevice,
                                               g->ctx->stream));
        }
        if (!done) solve_inversion_cols(g, i_freq, 3, V.p);
        for (int c = 0; c < 3; ++c) download_vec(g->ctx, V.p + (size_t)c * 2 * n, n, variables_w + 2 * (size_t)n * c);
    });
}

plx_status plx_solve(plx_geom *g, const plx_solve_desc *desc, double *x_out, double *polar_out,
                     double *results_out, int32_t *status_out, int32_t *steps_out, double *trace_out) {
    if (!g || !desc) return PLX_ERR_ARG;
    plx_status first_bad = PLX_OK;
    plx_status s = guarded(g->ctx, [&] {
        TraceRange trace_("plx_solve");
        plx_ctx *ctx = g->ctx;
        set_device(ctx);
        cudaStream_t st = ctx->stream;
        if (g->n_freq < 1) throw Error(PLX_ERR_ARG, "no frequencies set");
        if (desc->mode < PLX_INVERSION || desc->mode > PLX_GMRES_OTF) throw Error(PLX_ERR_ARG, "bad mode");
        if (desc->precision < PLX_FP64 || desc->precision > PLX_MIXED_BF16)
            throw Error(PLX_ERR_ARG, "bad precision");
        const bool otf = desc->mode == PLX_GMRES_OTF;
        if (otf && is_bem(g))
            throw Error(PLX_ERR_UNSUPPORTED, "BEM on the fly is not provided (the reference's BEM has no "
                                             "on-the-fly product either); use the on-memory mode");
        const bool refined = desc->precision != PLX_FP64 && desc->mode != PLX_INVERSION;
        if (!otf && !g->has_T) throw Error(PLX_ERR_ARG, "this mode needs the stored T (store_t at creation)");
        const int n = g->n_var, F = g->n_freq;
        std::vector<int32_t> pols;
        for (int p = 0; p < 3; ++p)
            if (desc->pol_mask & (1 << p)) pols.push_back(p);
        const int np = (int)pols.size();
        if (!np) throw Error(PLX_ERR_ARG, "empty polarisation mask");
        const int m = std::min(desc->max_krylov, n);
        if (desc->mode != PLX_INVERSION && m < 1) throw Error(PLX_ERR_ARG, "max_krylov must be positive");
        std::vector<Cplx> polar((size_t)F * 9, Cplx{0.0, 0.0});
        std::vector<int32_t> fstat(F, PLX_OK), fsteps((size_t)3 * F, 0);
        if (trace_out && desc->record_trace) std::memset(trace_out, 0, sizeof(double) * (size_t)m * 3 * F);
        if (x_out) std::memset(x_out, 0, sizeof(double) * 2 * (size_t)n * 3 * F);
        int64_t launches0 = ctx->launches;
        PLX_CHECK_CUDA(cudaEventRecord(ctx->ev0, st));
        // frequencies per block
        int fb = desc->freq_block;
        if (fb <= 0) {
            if (desc->mode == PLX_INVERSION) {
                fb = hessenberg_applies(g, np) ? F : 1;
            } else {
                uint64_t avail = ctx->budget > ctx->in_use ? ctx->budget - ctx->in_use : 0;
                // device bytes per complex column: the plain form keeps an FP64 Krylov
                // basis that grows with its (unrestarted) steps, counted up to 512;
                // the refined forms a basis of the inner dimension (FP32 for the mixed
                // forms) plus a dozen FP64 work vectors
                uint64_t per_col;
                if (!refined) {
                    per_col = (uint64_t)16 * n * (std::min(m, 512) + 8);
                } else {
                    const int im = desc->inner_krylov > 0 ? std::min(desc->inner_krylov, n) : std::min(64, n);
                    const uint64_t vb = desc->precision == PLX_FP64_REFINED ? 16 : 8;
                    per_col = vb * n * (uint64_t)(im + 1) + (uint64_t)16 * n * 12;
                }
                fb = (int)std::max<uint64_t>(1, std::min<uint64_t>(avail / 2 / per_col / np, 256 / np));
            }
        }
        fb = std::max(1, std::min(fb, F));
        for (int f0 = 0; f0 < F; f0 += fb) {
            const int nf = std::min(fb, F - f0);
            const int C = nf * np;
            std::vector<int32_t> cf(C), cp(C);
            for (int a = 0; a < nf; ++a)
                for (int b = 0; b < np; ++b) {
                    cf[a * np + b] = f0 + a;
                    cp[a * np + b] = pols[b];
                }
            DevArray<int32_t> dF, dP;
            DevArray<double> B, X;
            dF.alloc(ctx, C);
            dP.alloc(ctx, C);
            B.alloc(ctx, (size_t)C * 2 * n);
            X.alloc(ctx, (size_t)C * 2 * n);
            PLX_CHECK_CUDA(cudaMemcpyAsync(dF.p, cf.data(), C * 4, cudaMemcpyHostToDevice, st));
            PLX_CHECK_CUDA(cudaMemcpyAsync(dP.p, cp.data(), C * 4, cudaMemcpyHostToDevice, st));
            rhs_batch(g, OpBatch{C, dF.p}, dP.p, B.p);
            if (desc->mode == PLX_INVERSION) {
                // scalar-shift models: every frequency of the block in one launch on the
                // geometry's Hessenberg form; a singular factor falls back to the LU
                bool done = false;
                if (hessenberg_applies(g, np)) {
                    std::vector<int32_t> fl(nf);
                    for (int a = 0; a < nf; ++a) fl[a] = f0 + a;
                    done = hessenberg_solve(g, fl, np, B.p, X.p);
                }
                if (!done)
                    PLX_CHECK_CUDA(cudaMemcpyAsync(X.p, B.p, (size_t)C * 2 * n * 8, cudaMemcpyDeviceToDevice, st));
                for (int a = 0; a < nf && !done; ++a) {
                    try {
                        solve_inversion_cols(g, f0 + a, np, X.p + (size_t)a * np * 2 * n);
                    } catch (const Error &e) {
                        if (e.code != PLX_ERR_SINGULAR) throw;
                        fstat[f0 + a] = e.code;
                        ctx->last_error = e.msg;
                    }
                }
            } else {
                DevArray<int> flag;
                flag.alloc(ctx, C);
                PLX_CHECK_CUDA(cudaMemsetAsync(flag.p, 0, C * 4, st));
                positive_real_flags<<<dim3(std::min(n_blocks(n, 256), 64), C), 256, 0, st>>>(n, C, B.p, flag.p);
                ctx->launches++;
                std::vector<int> hf(C);
                PLX_CHECK_CUDA(cudaMemcpyAsync(hf.data(), flag.p, C * 4, cudaMemcpyDeviceToHost, st));
                PLX_CHECK_CUDA(cudaStreamSynchronize(st));
                PLX_CHECK_CUDA(cudaMemcpyAsync(X.p, B.p, (size_t)C * 2 * n * 8, cudaMemcpyDeviceToDevice, st));
                std::vector<int32_t> sel, dst;
                GmresRequest rq;
                for (int c = 0; c < C; ++c)
                    if (hf[c]) {
                        sel.push_back(c);
                        dst.push_back((int32_t)sel.size() - 1);
                        rq.freq.push_back(cf[c]);
                        rq.pol.push_back(cp[c]);
                    }
                const int G = (int)sel.size();
                if (G) {
                    DevArray<int32_t> dsel, ddst;
                    DevArray<double> Bg, Xg;
                    dsel.alloc(ctx, G);
                    ddst.alloc(ctx, G);
                    Bg.alloc(ctx, (size_t)G * 2 * n);
                    Xg.alloc(ctx, (size_t)G * 2 * n);
                    PLX_CHECK_CUDA(cudaMemcpyAsync(dsel.p, sel.data(), G * 4, cudaMemcpyHostToDevice, st));
                    PLX_CHECK_CUDA(cudaMemcpyAsync(ddst.p, dst.data(), G * 4, cudaMemcpyHostToDevice, st));
                    int gr = std::min(n_blocks(2LL * n, 256), 1024);
                    copy_cols<<<dim3(gr, G), 256, 0, st>>>(n, dsel.p, ddst.p, B.p, Bg.p);
                    ctx->launches++;
                    rq.m = m;
                    rq.tol = desc->tol;
                    rq.contraction = otf ? Contraction::FP64_OTF : Contraction::FP64;
                    rq.record_trace = desc->record_trace && trace_out && !refined;
                    GmresResult res;
                    if (refined) {
                        RefineRequest rr;
                        rr.freq = rq.freq;
                        rr.pol = rq.pol;
                        rr.tol = desc->tol;
                        rr.inner_m = desc->inner_krylov > 0 ? std::min(desc->inner_krylov, n) : std::min(64, n);
                        rr.inner_rel = desc->inner_tol > 0 ? desc->inner_tol : 1e-4;
                        rr.max_outer = desc->max_outer > 0 ? desc->max_outer : 60;
                        rr.outer_contraction = otf ? Contraction::FP64_OTF : Contraction::FP64;
                        rr.inner_contraction = desc->precision == PLX_MIXED_BF16X3 ? Contraction::TC3
                                               : desc->precision == PLX_MIXED_BF16 ? Contraction::TC1
                                                                                   : rr.outer_contraction;
                        // tensor-core inner solves restart on their own residual (one cheap
                        // product) up to 8 cycles before an FP64 residual; an FP64 inner solve's
                        // restart product would cost as much as the outer one
                        rr.max_cycles = rr.inner_contraction == rr.outer_contraction ? 1 : 8;
                        RefineResult rres;
                        solve_refined(g, rr, Bg.p, Xg.p, rres);
                        res.status = rres.status;
                        res.steps = rres.inner_steps;
                    } else {
                        gmres_batched(g, rq, Bg.p, Xg.p, res);
                    }
                    copy_cols<<<dim3(gr, G), 256, 0, st>>>(n, ddst.p, dsel.p, Xg.p, X.p);
                    ctx->launches++;
                    for (int k = 0; k < G; ++k) {
                        int f = rq.freq[k], p = rq.pol[k];
                        fsteps[(size_t)3 * f + p] = res.steps[k];
                        if (res.status[k] != PLX_OK && fstat[f] == PLX_OK) fstat[f] = res.status[k];
                        if (rq.record_trace)
                            std::copy(res.trace.begin() + (size_t)k * m, res.trace.begin() + (size_t)(k + 1) * m,
                                      trace_out + ((size_t)3 * f + p) * m);
                    }
                }
            }
            DevArray<Cplx> dpol;
            dpol.alloc(ctx, (size_t)C * 3);
            polar_batch(g, C, dP.p, X.p, dpol.p);
            std::vector<Cplx> hp((size_t)C * 3);
            PLX_CHECK_CUDA(cudaMemcpyAsync(hp.data(), dpol.p, hp.size() * 16, cudaMemcpyDeviceToHost, st));
            if (x_out) {
                std::vector<double> hx((size_t)C * 2 * n);
                PLX_CHECK_CUDA(cudaMemcpyAsync(hx.data(), X.p, hx.size() * 8, cudaMemcpyDeviceToHost, st));
                PLX_CHECK_CUDA(cudaStreamSynchronize(st));
                for (int c = 0; c < C; ++c) {
                    double *dstp = x_out + 2 * (size_t)n * ((size_t)3 * cf[c] + cp[c]);
                    for (int r = 0; r < n; ++r) {
                        dstp[2 * r] = hx[(size_t)c * 2 * n + r];
                        dstp[2 * r + 1] = hx[(size_t)c * 2 * n + n + r];
                    }
                }
            }
            PLX_CHECK_CUDA(cudaStreamSynchronize(st));
            for (int c = 0; c < C; ++c)
                for (int a = 0; a < 3; ++a) polar[(size_t)9 * cf[c] + a + 3 * cp[c]] = hp[(size_t)3 * c + a];
        }
        PLX_CHECK_CUDA(cudaEventRecord(ctx->ev1, st));
        PLX_CHECK_CUDA(cudaEventSynchronize(ctx->ev1));
        float ms = 0.f;
        PLX_CHECK_CUDA(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
        g->last_ms = ms;
        g->last_launches = ctx->launches - launches0;
        for (int f = 0; f < F; ++f) {
            if (polar_out)
                for (int e = 0; e < 9; ++e) {
                    polar_out[2 * (9 * (size_t)f + e)] = polar[9 * (size_t)f + e].re;
                    polar_out[2 * (9 * (size_t)f + e) + 1] = polar[9 * (size_t)f + e].im;
                }
            if (results_out) results_row(&polar[9 * (size_t)f], g->omega[f], results_out + 20 * (size_t)f);
            if (status_out) status_out[f] = fstat[f];
            if (fstat[f] != PLX_OK && first_bad == PLX_OK) {
                first_bad = (plx_status)fstat[f];
                if (first_bad == PLX_ERR_NOT_CONVERGED)
                    ctx->last_error = "GMRES not converged and restart GMRES NYI.";
                else if (first_bad == PLX_ERR_NAN)
                    ctx->last_error = "non-finite residual in GMRES";
            }
        }
        if (steps_out) std::copy(fsteps.begin(), fsteps.end(), steps_out);
    });
    return s != PLX_OK ? s : first_bad;
}

plx_status plx_profile_enable(plx_ctx *ctx, int32_t on) {
    if (!ctx) return PLX_ERR_ARG;
    return guarded(ctx, [&] {
        set_device(ctx);
        PLX_CHECK_CUDA(cudaStreamSynchronize(ctx->stream));
        ctx->profile = on != 0;
        ctx->prof_used = 0;
        for (int c = 0; c < plx_ctx::kProfCategories; ++c) {
            ctx->prof_flops[c] = ctx->prof_bytes[c] = 0.0;
            ctx->prof_launches[c] = 0;
        }
    });
}

plx_status plx_set_wait_limit(plx_ctx *ctx, uint32_t polls) {
    if (!ctx) return PLX_ERR_ARG;
    return guarded(ctx, [&] {
        set_device(ctx);
        PLX_CHECK_CUDA(cudaStreamSynchronize(ctx->stream));
        ctx->wait_limit = polls ? polls : plx_ctx::kDefaultWaitLimit;
    });
}

plx_status plx_profile_read(plx_ctx *ctx, int32_t category, double *ms, int64_t *launches, double *flops,
                            double *bytes) {
    if (!ctx || category < 0 || category >= plx_ctx::kProfCategories) return PLX_ERR_ARG;
    return guarded(ctx, [&] {
        set_device(ctx);
        PLX_CHECK_CUDA(cudaStreamSynchronize(ctx->stream));
        double total = 0.0;
        for (size_t k = 0; k + 1 < ctx->prof_used; k += 2) {
            if (ctx->prof_cat[k / 2] != category) continue;
            float t = 0.f;
            PLX_CHECK_CUDA(cudaEventElapsedTime(&t, ctx->prof_events[k], ctx->prof_events[k + 1]));
            total += t;
        }
        if (ms) *ms = total;
        if (launches) *launches = ctx->prof_launches[category];
        if (flops) *flops = ctx->prof_flops[category];
        if (bytes) *bytes = ctx->prof_bytes[category];
    });
}

plx_status plx_contract(plx_geom *g, int32_t count, const double *X, double *S, int32_t how) {
    if (!g || !X || !S) return PLX_ERR_ARG;
    return guarded(g->ctx, [&] {
        TraceRange trace_("plx_contract");
        set_device(g->ctx);
        if (count < 1 || how < 0 || how > 3) throw Error(PLX_ERR_ARG, "bad column count or contraction kind");
        const int n = g->n_var;
        // [count][n] real columns == [count/2][2][n] split-complex columns; an odd
        // count is padded with one zero column
        const int padded = count + (count & 1);
        DevArray<double> dX, dS;
        dX.alloc(g->ctx, (size_t)padded * n);
        dS.alloc(g->ctx, (size_t)padded * n);
        PLX_CHECK_CUDA(cudaMemsetAsync(dX.p, 0, (size_t)padded * n * 8, g->ctx->stream));
        PLX_CHECK_CUDA(cudaMemcpyAsync(dX.p, X, (size_t)count * n * 8, cudaMemcpyHostToDevice, g->ctx->stream));
        const Contraction kinds[4] = {Contraction::FP64, Contraction::FP64_OTF, Contraction::TC3, Contraction::TC1};
        contract_t(g, padded / 2, dX.p, dS.p, kinds[how]);
        PLX_CHECK_CUDA(cudaMemcpyAsync(S, dS.p, (size_t)count * n * 8, cudaMemcpyDeviceToHost, g->ctx->stream));
        PLX_CHECK_CUDA(cudaStreamSynchronize(g->ctx->stream));
        if (how >= 2 && tc_error(g))
            throw Error(PLX_ERR_CUDA, "tensor-core contraction timed out waiting on its pipeline");
    });
}


}  // extern "C"

// ---------------------------------------------------------------------------
// continuous batching: a refinement solve whose columns come and go between
// outer steps (plx_batch_*)
// ---------------------------------------------------------------------------
struct plx_batch {
    plx_geom *g = nullptr;
    RefineState st;
    struct Request {
        int32_t f0 = 0, n_freq = 0;             // frequency-table range
        std::vector<int32_t> pols;
        std::vector<int32_t> slots;             // freq-major, pol-minor
    };
    std::map<int64_t, Request> req;
    std::vector<int64_t> order;                 // tags in arrival order
};

namespace {

// slots of `k` columns: D[slot[k]] = S[k]
__global__ void scatter_cols(int n, const int32_t *__restrict__ slot, const double *__restrict__ S,
                             double *__restrict__ D) {
    int k = blockIdx.y;
    const double *s = S + (int64_t)k * 2 * n;
    double *d = D + (int64_t)slot[k] * 2 * n;
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < 2LL * n; r += (int64_t)gridDim.x * blockDim.x)
        d[r] = s[r];
}

bool request_finished(const plx_batch *b, const plx_batch::Request &r) {
    for (int s : r.slots)
        if (b->st.slots[s].state != RefineState::Slot::FINISHED) return false;
    return true;
}

int32_t batch_active(const plx_batch *b) {
    int32_t a = 0;
    for (const auto &s : b->st.slots) a += s.state == RefineState::Slot::ACTIVE;
    return a;
}

}  // namespace

extern "C" {

plx_status plx_batch_open(plx_geom *g, const plx_solve_desc *desc, plx_batch **out) {
    if (!g || !desc || !out) return PLX_ERR_ARG;
    *out = nullptr;
    return guarded(g->ctx, [&] {
        set_device(g->ctx);
        if (desc->mode != PLX_GMRES_MEM && desc->mode != PLX_GMRES_OTF)
            throw Error(PLX_ERR_ARG, "a batch solves by GMRES (on-memory or on the fly)");
        if (desc->precision < PLX_FP64 || desc->precision > PLX_MIXED_BF16) throw Error(PLX_ERR_ARG, "bad precision");
        if (desc->precision == PLX_FP64)
            throw Error(PLX_ERR_ARG, "a batch runs the refinement forms (mixed or FP64 refined)");
        const bool otf = desc->mode == PLX_GMRES_OTF;
        if (otf && is_bem(g)) throw Error(PLX_ERR_UNSUPPORTED, "BEM on the fly is not provided");
        if (!otf && !g->has_T) throw Error(PLX_ERR_ARG, "this mode needs the stored T (store_t at creation)");
        if (g->open_batches > 0) throw Error(PLX_ERR_ARG, "the geometry already has an open batch");
        const int n = g->n_var;
        RefineRequest rr;
        rr.inner_m = desc->inner_krylov > 0 ? std::min(desc->inner_krylov, n) : std::min(64, n);
        rr.inner_rel = desc->inner_tol > 0 ? desc->inner_tol : 1e-4;
        rr.max_outer = desc->max_outer > 0 ? desc->max_outer : 60;
        rr.outer_contraction = otf ? Contraction::FP64_OTF : Contraction::FP64;
        rr.inner_contraction = desc->precision == PLX_MIXED_BF16X3 ? Contraction::TC3
                               : desc->precision == PLX_MIXED_BF16 ? Contraction::TC1
                                                                   : rr.outer_contraction;
        rr.max_cycles = rr.inner_contraction == rr.outer_contraction ? 1 : 8;
        auto *b = new plx_batch();
        b->g = g;
        b->st.own(g, rr);
        // the batch owns the frequency table from here on
        g->n_freq = 0;
        g->omega.clear();
        g->alpha_w.clear();
        g->open_batches++;
        *out = b;
    });
}

plx_status plx_batch_add(plx_batch *b, int64_t tag, int32_t n_freq, const double *omega, const double *alpha_w,
                         int32_t pol_mask, double tol) {
    if (!b || !omega || n_freq < 1) return PLX_ERR_ARG;
    plx_geom *g = b->g;
    return guarded(g->ctx, [&] {
        TraceRange trace_("plx_batch_add");
        set_device(g->ctx);
        plx_ctx *ctx = g->ctx;
        cudaStream_t st = ctx->stream;
        if (tag < 0 || b->req.count(tag)) throw Error(PLX_ERR_ARG, "request tags are distinct and non-negative");
        if (g->model == PLX_WFQFMU && !alpha_w) throw Error(PLX_ERR_ARG, "alpha_w is required for wFQFMu");
        if (is_bem(g) && !alpha_w) throw Error(PLX_ERR_ARG, "eps(w) (alpha_w) is required for BEM");
        if (!(tol > 0.0)) throw Error(PLX_ERR_ARG, "tolerance must be positive");
        std::vector<int32_t> pols;
        for (int p = 0; p < 3; ++p)
            if (pol_mask & (1 << p)) pols.push_back(p);
        if (pols.empty()) throw Error(PLX_ERR_ARG, "empty polarisation mask");
        const int n = g->n_var, np = (int)pols.size(), C = n_freq * np;
        // append the frequencies to the geometry's tables
        plx_batch::Request r;
        r.f0 = g->n_freq;
        r.n_freq = n_freq;
        r.pols = pols;
        const int per = is_bem(g) ? 1 : g->n_types;
        g->omega.insert(g->omega.end(), omega, omega + n_freq);
        if (alpha_w)
            for (size_t e = 0; e < (size_t)per * n_freq; ++e) g->alpha_w.push_back({alpha_w[2 * e], alpha_w[2 * e + 1]});
        g->n_freq += n_freq;
        upload_frequency_tables(g);
        // slots: free ones first, then grown
        RefineState &S = b->st;
        int used = 0;
        for (const auto &s : S.slots) used += s.state != RefineState::Slot::FREE;
        S.grow(used + C);
        for (int c = 0, s = 0; c < C; ++c) {
            while (S.slots[s].state != RefineState::Slot::FREE) ++s;
            RefineState::Slot &sl = S.slots[s];
            sl = RefineState::Slot();
            sl.state = RefineState::Slot::ACTIVE;
            sl.freq = r.f0 + c / np;
            sl.pol = pols[c % np];
            sl.tol = tol;
            sl.tag = tag;
            r.slots.push_back(s);
        }
        // right-hand sides into the slots; x = 0, r = b
        std::vector<int32_t> cf(C), cp(C);
        for (int c = 0; c < C; ++c) {
            cf[c] = S.slots[r.slots[c]].freq;
            cp[c] = S.slots[r.slots[c]].pol;
        }
        DevArray<int32_t> dF, dP, dS;
        DevArray<double> Bt, Z;
        dF.alloc(ctx, C);
        dP.alloc(ctx, C);
        dS.alloc(ctx, C);
        Bt.alloc(ctx, (size_t)C * 2 * n);
        Z.alloc(ctx, (size_t)C * 2 * n);
        PLX_CHECK_CUDA(cudaMemcpyAsync(dF.p, cf.data(), C * 4, cudaMemcpyHostToDevice, st));
        PLX_CHECK_CUDA(cudaMemcpyAsync(dP.p, cp.data(), C * 4, cudaMemcpyHostToDevice, st));
        PLX_CHECK_CUDA(cudaMemcpyAsync(dS.p, r.slots.data(), C * 4, cudaMemcpyHostToDevice, st));
        PLX_CHECK_CUDA(cudaMemsetAsync(Z.p, 0, (size_t)C * 2 * n * 8, st));
        rhs_batch(g, OpBatch{C, dF.p}, dP.p, Bt.p);
        const int gr = std::min(n_blocks(2LL * n, 256), 1024);
        scatter_cols<<<dim3(gr, C), 256, 0, st>>>(n, dS.p, Bt.p, S.ownB.p);
        scatter_cols<<<dim3(gr, C), 256, 0, st>>>(n, dS.p, Bt.p, S.R.p);
        scatter_cols<<<dim3(gr, C), 256, 0, st>>>(n, dS.p, Z.p, S.ownX.p);
        ctx->launches += 3;
        PLX_CHECK_CUDA(cudaGetLastError());
        PLX_CHECK_CUDA(cudaStreamSynchronize(st));
        b->req[tag] = std::move(r);
        b->order.push_back(tag);
    });
}

plx_status plx_batch_step(plx_batch *b, int32_t *n_active) {
    if (!b) return PLX_ERR_ARG;
    return plx_batch_step_group(&b, 1, n_active);
}

plx_status plx_batch_step_group(plx_batch *const *batches, int32_t count, int32_t *n_active) {
    if (!batches || count < 1 || !batches[0]) return PLX_ERR_ARG;
    plx_ctx *ctx = batches[0]->g->ctx;
    return guarded(ctx, [&] {
        TraceRange trace_("plx_batch_step");
        set_device(ctx);
        std::vector<RefineState *> states;
        for (int i = 0; i < count; ++i) {
            if (!batches[i] || batches[i]->g->ctx != ctx)
                throw Error(PLX_ERR_ARG, "grouped batches must share one context");
            for (int k = 0; k < i; ++k)
                if (batches[k]->g == batches[i]->g) throw Error(PLX_ERR_ARG, "one batch per geometry in a group");
            states.push_back(&batches[i]->st);
        }
        const int64_t l0 = ctx->launches;
        PLX_CHECK_CUDA(cudaEventRecord(ctx->ev0, ctx->stream));
        refine_group_step(states);
        int32_t a = 0;
        bool timed_out = false;
        for (int i = 0; i < count; ++i) {
            batches[i]->st.update_status();      // finished columns are known right after the step
            a += batch_active(batches[i]);
            plx_geom *g = batches[i]->g;
            if (g->d_tc_err.p && tc_error(g) != 0) timed_out = true;
        }
        PLX_CHECK_CUDA(cudaEventRecord(ctx->ev1, ctx->stream));
        PLX_CHECK_CUDA(cudaEventSynchronize(ctx->ev1));
        float ms = 0.f;
        PLX_CHECK_CUDA(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
        for (int i = 0; i < count; ++i) {
            batches[i]->g->last_ms = ms;
            batches[i]->g->last_launches = ctx->launches - l0;
        }
        if (timed_out) throw Error(PLX_ERR_CUDA, "tensor-core contraction timed out waiting on its pipeline");
        if (n_active) *n_active = a;
    });
}

plx_status plx_batch_poll(plx_batch *b, int64_t *tag) {
    if (!b || !tag) return PLX_ERR_ARG;
    *tag = -1;
    for (int64_t t : b->order) {
        auto it = b->req.find(t);
        if (it != b->req.end() && request_finished(b, it->second)) {
            *tag = t;
            break;
        }
    }
    return PLX_OK;
}

plx_status plx_batch_take(plx_batch *b, int64_t tag, double *polar_out, double *results_out, int32_t *status_out,
                          int32_t *steps_out) {
    if (!b) return PLX_ERR_ARG;
    plx_geom *g = b->g;
    plx_status first_bad = PLX_OK;
    plx_status s = guarded(g->ctx, [&] {
        TraceRange trace_("plx_batch_take");
        set_device(g->ctx);
        plx_ctx *ctx = g->ctx;
        cudaStream_t st = ctx->stream;
        auto it = b->req.find(tag);
        if (it == b->req.end()) throw Error(PLX_ERR_ARG, "unknown request tag");
        plx_batch::Request &r = it->second;
        if (!request_finished(b, r)) throw Error(PLX_ERR_ARG, "the request is still being solved");
        const int n = g->n_var, C = (int)r.slots.size(), np = (int)r.pols.size();
        DevArray<int32_t> dS, dD;
        DevArray<double> Xg;
        DevArray<Cplx> dpol;
        dS.alloc(ctx, C);
        dD.alloc(ctx, C);
        Xg.alloc(ctx, (size_t)C * 2 * n);
        dpol.alloc(ctx, (size_t)C * 3);
        std::vector<int32_t> dst(C);
        for (int c = 0; c < C; ++c) dst[c] = c;
        PLX_CHECK_CUDA(cudaMemcpyAsync(dS.p, r.slots.data(), C * 4, cudaMemcpyHostToDevice, st));
        PLX_CHECK_CUDA(cudaMemcpyAsync(dD.p, dst.data(), C * 4, cudaMemcpyHostToDevice, st));
        copy_cols<<<dim3(std::min(n_blocks(2LL * n, 256), 1024), C), 256, 0, st>>>(n, dS.p, dD.p, b->st.ownX.p, Xg.p);
        ctx->launches++;
        polar_batch(g, C, nullptr, Xg.p, dpol.p);
        std::vector<Cplx> hp((size_t)C * 3);
        PLX_CHECK_CUDA(cudaMemcpyAsync(hp.data(), dpol.p, hp.size() * sizeof(Cplx), cudaMemcpyDeviceToHost, st));
        PLX_CHECK_CUDA(cudaStreamSynchronize(st));
        for (int f = 0; f < r.n_freq; ++f) {
            std::vector<Cplx> P(9, Cplx{0.0, 0.0});
            int32_t fst = PLX_OK;
            if (steps_out)
                for (int p = 0; p < 3; ++p) steps_out[3 * f + p] = 0;
            for (int k = 0; k < np; ++k) {
                const int c = f * np + k;
                const RefineState::Slot &sl = b->st.slots[r.slots[c]];
                for (int a = 0; a < 3; ++a) P[a + 3 * r.pols[k]] = hp[(size_t)3 * c + a];
                if (sl.status != PLX_OK && fst == PLX_OK) fst = sl.status;
                if (steps_out) steps_out[3 * f + r.pols[k]] = sl.inner_steps;
            }
            if (polar_out)
                for (int e = 0; e < 9; ++e) {
                    polar_out[2 * (9 * (size_t)f + e)] = P[e].re;
                    polar_out[2 * (9 * (size_t)f + e) + 1] = P[e].im;
                }
            if (results_out) results_row(P.data(), g->omega[r.f0 + f], results_out + 20 * (size_t)f);
            if (status_out) status_out[f] = fst;
            if (fst != PLX_OK && first_bad == PLX_OK) first_bad = (plx_status)fst;
        }
        for (int sidx : r.slots) b->st.slots[sidx] = RefineState::Slot();
        b->req.erase(it);
        b->order.erase(std::remove(b->order.begin(), b->order.end(), tag), b->order.end());
        if (b->req.empty()) {
            // nothing in flight: the frequency table starts again from empty
            g->n_freq = 0;
            g->omega.clear();
            g->alpha_w.clear();
        }
        if (first_bad == PLX_ERR_NOT_CONVERGED) ctx->last_error = "refinement ran out of outer steps";
        else if (first_bad == PLX_ERR_NAN) ctx->last_error = "non-finite residual in the refinement";
    });
    return s != PLX_OK ? s : first_bad;
}

int32_t plx_batch_active(const plx_batch *b) { return b ? batch_active(b) : 0; }

void plx_batch_close(plx_batch *b) {
    if (!b) return;
    plx_geom *g = b->g;
    try {
        set_device(g->ctx);
        PLX_CHECK_CUDA(cudaStreamSynchronize(g->ctx->stream));
    } catch (...) {
    }
    g->open_batches--;
    g->n_freq = 0;
    g->omega.clear();
    g->alpha_w.clear();
    delete b;
}

double plx_last_solve_ms(const plx_geom *g) { return g ? g->last_ms : 0.0; }
int64_t plx_last_solve_launches(const plx_geom *g) { return g ? g->last_launches : 0; }

}  // extern "C"
