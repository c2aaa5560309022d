// Frequency-independent device data of a geometry: the Drude/Fermi
// conductance K in CSR form and the dense interaction matrix T.
#include <algorithm>
#include <cmath>
#include <numeric>

#include "pair_tiles.cuh"
#include "plx_internal.h"

namespace plx {

namespace {

constexpr int kTile = 128;

// Counts (pass 0) or writes (pass 1) the off-diagonal entries of row i of K
// that are non-zero in either direction.  Source atoms are staged in shared
// memory tiles; the row is produced in increasing j, so columns are sorted.
template <int PASS>
__global__ void conductance_rows(int N, int nt, const double *__restrict__ pos,
                                 const int32_t *__restrict__ type,
                                 const double *__restrict__ fd, const double *__restrict__ fs,
                                 const double *__restrict__ r0, const double *__restrict__ aij,
                                 int32_t *__restrict__ count, const int32_t *__restrict__ rowptr,
                                 int32_t *__restrict__ col, double *__restrict__ kval,
                                 double *__restrict__ ktval) {
    __shared__ double sx[kTile], sy[kTile], sz[kTile];
    __shared__ int32_t st[kTile];
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    bool live = i < N;
    double xi = 0, yi = 0, zi = 0;
    int ti = 0;
    if (live) {
        xi = pos[i];
        yi = pos[N + i];
        zi = pos[2 * N + i];
        ti = type[i];
    }
    int c = 0;
    int64_t out = (PASS == 1 && live) ? rowptr[i] : 0;
    for (int j0 = 0; j0 < N; j0 += kTile) {
        int jj = j0 + threadIdx.x;
        __syncthreads();
        if (threadIdx.x < kTile && jj < N) {
            sx[threadIdx.x] = pos[jj];
            sy[threadIdx.x] = pos[N + jj];
            sz[threadIdx.x] = pos[2 * N + jj];
            st[threadIdx.x] = type[jj];
        }
        __syncthreads();
        int jn = min(kTile, N - j0);
        if (!live) continue;
        for (int t = 0; t < jn; ++t) {
            int j = j0 + t;
            if (j == i) continue;
            double dx = xi - sx[t], dy = yi - sy[t], dz = zi - sz[t];
            double r = sqrt(dx * dx + dy * dy + dz * dz);
            int tj = st[t];
            int p_ij = ti + nt * tj, p_ji = tj + nt * ti;
            double kij = plx_conductance(r, fd[p_ij], fs[p_ij], r0[p_ij], aij[ti]);
            double kji = plx_conductance(r, fd[p_ji], fs[p_ji], r0[p_ji], aij[tj]);
            if (kij != 0.0 || kji != 0.0) {
                if (PASS == 0) {
                    ++c;
                } else {
                    col[out] = j;
                    kval[out] = kij;
                    ktval[out] = kji;
                    ++out;
                }
            }
        }
    }
    if (PASS == 0 && live) count[i] = c;
}

// Dense T, row-major n_var x n_var.  One thread per ordered atom pair (i, j)
// writes the 1x1 (wFQ) or 4x4 (wFQFMu) block of rows of atom i and columns of
// atom j.  Rows/columns: q_i -> i, mu_i,k -> N + 3 i + k.
__global__ void dense_t_kernel(int N, int fmu, const double *__restrict__ pos,
                               const double *__restrict__ par, double *__restrict__ T) {
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    int i = blockIdx.y;
    if (j >= N) return;
    const int64_t nv = fmu ? 4LL * N : (int64_t)N;
    double rq_i = par[i], rm_i = par[N + i], eta_i = par[2 * N + i];
    double rq_j = par[j], rm_j = par[N + j];
    if (i == j) {
        T[(int64_t)i * nv + i] = (eta_i + eta_i) / 2.0;
        if (fmu) {
            for (int a = 0; a < 3; ++a) {
                int64_t ra = N + 3LL * i + a;
                T[i * nv + N + 3LL * j + a] = 0.0;
                T[ra * nv + j] = 0.0;
                for (int b = 0; b < 3; ++b) T[ra * nv + N + 3LL * j + b] = 0.0;
            }
        }
        return;
    }
    double dx = pos[i] - pos[j], dy = pos[N + i] - pos[N + j], dz = pos[2 * N + i] - pos[2 * N + j];
    if (!fmu) {
        T[(int64_t)i * nv + j] = plx_pair_qq(dx, dy, dz, rq_i, rq_j);
        return;
    }
    PairTile t;
    plx_pair_tile(dx, dy, dz, rq_i, rm_i, rq_j, rm_j, t);
    int64_t cq = j, cm = N + 3LL * j;
    T[(int64_t)i * nv + cq] = t.qq;
    for (int k = 0; k < 3; ++k) {
        T[(int64_t)i * nv + cm + k] = t.qm[k];
        T[(N + 3LL * i + k) * nv + cq] = t.mq[k];
    }
    const int mi[3][3] = {{0, 1, 2}, {1, 3, 4}, {2, 4, 5}};
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) T[(N + 3LL * i + a) * nv + cm + b] = t.mm[mi[a][b]];
}

}  // namespace

void build_conductance(plx_geom *g) {
    plx_ctx *ctx = g->ctx;
    const int N = g->n_atoms, nt = g->n_types;
    DevArray<double> d_fd, d_fs, d_r0, d_a;
    d_fd.alloc(ctx, nt * nt);
    d_fs.alloc(ctx, nt * nt);
    d_r0.alloc(ctx, nt * nt);
    d_a.alloc(ctx, nt);
    cudaStream_t st = ctx->stream;
    PLX_CHECK_CUDA(cudaMemcpyAsync(d_fd.p, g->fermi_d.data(), nt * nt * 8, cudaMemcpyHostToDevice, st));
    PLX_CHECK_CUDA(cudaMemcpyAsync(d_fs.p, g->fermi_s.data(), nt * nt * 8, cudaMemcpyHostToDevice, st));
    PLX_CHECK_CUDA(cudaMemcpyAsync(d_r0.p, g->r0.data(), nt * nt * 8, cudaMemcpyHostToDevice, st));
    PLX_CHECK_CUDA(cudaMemcpyAsync(d_a.p, g->a_ij.data(), nt * 8, cudaMemcpyHostToDevice, st));
    DevArray<int32_t> d_count;
    d_count.alloc(ctx, N);
    int blocks = n_blocks(N, kTile);
    conductance_rows<0><<<blocks, kTile, 0, st>>>(N, nt, g->d_pos.p, g->d_type.p, d_fd.p, d_fs.p,
                                                  d_r0.p, d_a.p, d_count.p, nullptr, nullptr,
                                                  nullptr, nullptr);
    ctx->launches++;
    PLX_CHECK_CUDA(cudaGetLastError());
    std::vector<int32_t> cnt(N);
    PLX_CHECK_CUDA(cudaMemcpyAsync(cnt.data(), d_count.p, N * 4, cudaMemcpyDeviceToHost, st));
    PLX_CHECK_CUDA(cudaStreamSynchronize(st));
    std::vector<int32_t> rowptr(N + 1, 0);
    int64_t acc = 0;
    for (int i = 0; i < N; ++i) {
        rowptr[i] = (int32_t)acc;
        acc += cnt[i];
        if (acc > INT32_MAX) throw Error(PLX_ERR_UNSUPPORTED, "conductance has more than 2^31 non-zeros");
    }
    rowptr[N] = (int32_t)acc;
    g->nnz = acc;
    g->d_rowptr.alloc(ctx, N + 1);
    g->d_col.alloc(ctx, std::max<int64_t>(acc, 1));
    g->d_kval.alloc(ctx, std::max<int64_t>(acc, 1));
    g->d_ktval.alloc(ctx, std::max<int64_t>(acc, 1));
    PLX_CHECK_CUDA(cudaMemcpyAsync(g->d_rowptr.p, rowptr.data(), (N + 1) * 4, cudaMemcpyHostToDevice, st));
    conductance_rows<1><<<blocks, kTile, 0, st>>>(N, nt, g->d_pos.p, g->d_type.p, d_fd.p, d_fs.p,
                                                  d_r0.p, d_a.p, nullptr, g->d_rowptr.p, g->d_col.p,
                                                  g->d_kval.p, g->d_ktval.p);
    ctx->launches++;
    PLX_CHECK_CUDA(cudaGetLastError());
    PLX_CHECK_CUDA(cudaStreamSynchronize(st));
}

void build_dense_t(plx_geom *g) {
    plx_ctx *ctx = g->ctx;
    const int64_t nv = g->n_var;
    g->d_T.alloc(ctx, (size_t)(nv * nv));
    dim3 grid(n_blocks(g->n_atoms, 128), g->n_atoms);
    dense_t_kernel<<<grid, 128, 0, ctx->stream>>>(g->n_atoms, g->model == PLX_WFQFMU, g->d_pos.p,
                                                  g->d_par.p, g->d_T.p);
    ctx->launches++;
    PLX_CHECK_CUDA(cudaGetLastError());
    PLX_CHECK_CUDA(cudaStreamSynchronize(ctx->stream));
    g->has_T = true;
}

// Per-frequency tables.  Charge diagonal -z(w) with
// z = w (-w tau - i) / (2 n tau) (new_gmres_diagonal_shift_wfq,
// wfq_module.f90:398-424); dipole diagonal sum_t f_t,i / alpha_t(w)
// (wfqfmu_module.f90:698-746); Drude weights w_t = 2 n_t / (1/tau_t - i w)
// (construct_H_minus_L_matrix, matrix_module.f90:435-482).
void upload_frequency_tables(plx_geom *g) {
    const int nt = g->n_types, F = g->n_freq;
    if (is_bem(g)) {
        // z(w) = 2 pi (eps_s + eps(w)) / (eps_s - eps(w)) (new_gmres_diagonal_shift_bem,
        // bem_module.f90:977-997); alpha_w carries eps(w)
        g->bem_z.resize(F);
        for (int f = 0; f < F; ++f) {
            Cplx e = g->alpha_w[f];
            double nr = g->eps_solvent + e.re, ni = e.im;        // eps_s + eps
            double dr = g->eps_solvent - e.re, di = -e.im;       // eps_s - eps
            double m = dr * dr + di * di;
            double qr = (nr * dr + ni * di) / m, qi = (ni * dr - nr * di) / m;
            const double twopi = 6.283185307179586476925286766559;
            g->bem_z[f] = {twopi * qr, twopi * qi};
        }
        g->d_dq.alloc(g->ctx, F);
        PLX_CHECK_CUDA(cudaMemcpyAsync(g->d_dq.p, g->bem_z.data(), F * sizeof(Cplx), cudaMemcpyHostToDevice,
                                       g->ctx->stream));
        PLX_CHECK_CUDA(cudaStreamSynchronize(g->ctx->stream));
        return;
    }
    std::vector<Cplx> dq(nt * F), ia(nt * F), wr((size_t)nt * nt * F);
    for (int f = 0; f < F; ++f) {
        double w = g->omega[f];
        std::vector<double> wre(nt), wim(nt);
        for (int t = 0; t < nt; ++t) {
            double tau = g->tau[t], n = g->density[t];
            double den = 2.0 * n * tau;
            // z = w * (-w tau - i) / den ; diagonal = -z
            double zre = w * (-w * tau) / den, zim = w * (-1.0) / den;
            dq[t + nt * f] = {-zre, -zim};
            if (!g->alpha_w.empty()) {
                Cplx a = g->alpha_w[t + nt * f];
                double m = a.re * a.re + a.im * a.im;
                ia[t + nt * f] = {a.re / m, -a.im / m};
            } else {
                ia[t + nt * f] = {0.0, 0.0};
            }
            // w_t = 2 n / (1/tau - i w)
            double cr = 1.0 / tau, ci = -w;
            double cm = cr * cr + ci * ci;
            wre[t] = 2.0 * n * cr / cm;
            wim[t] = -2.0 * n * ci / cm;
        }
        for (int ti = 0; ti < nt; ++ti)
            for (int tj = 0; tj < nt; ++tj) {
                // w_tj / w_ti
                double m = wre[ti] * wre[ti] + wim[ti] * wim[ti];
                double re = (wre[tj] * wre[ti] + wim[tj] * wim[ti]) / m;
                double im = (wim[tj] * wre[ti] - wre[tj] * wim[ti]) / m;
                wr[ti + nt * tj + (size_t)nt * nt * f] = {re, im};
            }
    }
    plx_ctx *ctx = g->ctx;
    g->d_dq.alloc(ctx, nt * F);
    g->d_inv_alpha.alloc(ctx, nt * F);
    g->d_wratio.alloc(ctx, (size_t)nt * nt * F);
    cudaStream_t st = ctx->stream;
    PLX_CHECK_CUDA(cudaMemcpyAsync(g->d_dq.p, dq.data(), dq.size() * 16, cudaMemcpyHostToDevice, st));
    PLX_CHECK_CUDA(cudaMemcpyAsync(g->d_inv_alpha.p, ia.data(), ia.size() * 16, cudaMemcpyHostToDevice, st));
    PLX_CHECK_CUDA(cudaMemcpyAsync(g->d_wratio.p, wr.data(), wr.size() * 16, cudaMemcpyHostToDevice, st));
    PLX_CHECK_CUDA(cudaStreamSynchronize(st));
}

}  // namespace plx
