// The frequency-dependent operator A(w) = blockdiag(Kop(w), I) T + D(w) and
// the right-hand sides, for batches of columns (one frequency per column).
//
// Reference: product_matrix_vector_{wfq,wfqfmu} (wfq_module.f90:321-348,
// wfqfmu_module.f90:584-626) = T x (product_q_block_x / product_mu_block_x,
// matrix_module.f90:727-1001), then the charge rows through (K - P) or
// 1/2 (K + H(w)) (update_y_q, matrix_module.f90:1011-1098), dipole rows copied
// (update_y_mu, :1107-1125), then new_gmres_diagonal_shift.
#include <algorithm>

#include "pair_tiles.cuh"
#include "plx_internal.h"
#include "skinny.cuh"

namespace plx {

namespace {

// ---------------------------------------------------------------------------
// S^T = X^T T, tiled (R > 16): 64 x 128 output tiles, 8 x 8 per thread (four
// FMAs per shared-memory load, which keeps the FP64 pipe rather than shared
// memory the limit), the next k-slab prefetched into registers while the
// current one is multiplied.  Split over K in the SAME chunks as
// skinny_partial and reduced by skinny_reduce, and every output element is
// accumulated by one FMA chain in k order from zero, exactly as
// skinny_partial does, so a column's result does not depend on the number of
// columns in the batch.
// ---------------------------------------------------------------------------
constexpr int BM = 64, BN = 128, BK = 8, kTiledThreads = 128;

__global__ void __launch_bounds__(kTiledThreads) tiled_partial(int R, int n, int kchunk,
                                                               const double *__restrict__ Xt,
                                                               const double *__restrict__ T,
                                                               double *__restrict__ part) {
    __shared__ double As[2][BM][BK + 1];
    __shared__ double Bs[2][BK][BN];
    const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;          // 16 x 8 threads
    const int row0 = blockIdx.y * BM, col0 = blockIdx.x * BN;
    const int kbeg = blockIdx.z * kchunk, kend = min(n, kbeg + kchunk);
    constexpr int LA = BM * BK / kTiledThreads, LB = BK * BN / kTiledThreads;   // 4, 8
    double ra[LA], rb[LB];
    auto load = [&](int k0) {
#pragma unroll
        for (int q = 0; q < LA; ++q) {
            const int e = threadIdx.x + q * kTiledThreads, r = e / BK, k = e % BK;
            const int gr = row0 + r, gk = k0 + k;
            ra[q] = (gr < R && gk < kend) ? Xt[(int64_t)gr * n + gk] : 0.0;
        }
#pragma unroll
        for (int q = 0; q < LB; ++q) {
            const int e = threadIdx.x + q * kTiledThreads, k = e / BN, c = e % BN;
            const int gk = k0 + k, gc = col0 + c;
            rb[q] = (gk < kend && gc < n) ? T[(int64_t)gk * n + gc] : 0.0;
        }
    };
    auto store = [&](int buf) {
#pragma unroll
        for (int q = 0; q < LA; ++q) {
            const int e = threadIdx.x + q * kTiledThreads;
            As[buf][e / BK][e % BK] = ra[q];
        }
#pragma unroll
        for (int q = 0; q < LB; ++q) {
            const int e = threadIdx.x + q * kTiledThreads;
            Bs[buf][e / BN][e % BN] = rb[q];
        }
    };
    double acc[8][8];
#pragma unroll
    for (int u = 0; u < 8; ++u)
#pragma unroll
        for (int v = 0; v < 8; ++v) acc[u][v] = 0.0;
    if (kbeg < kend) {
        load(kbeg);
        store(0);
    }
    __syncthreads();
    int buf = 0;
    for (int k0 = kbeg; k0 < kend; k0 += BK) {
        const bool more = k0 + BK < kend;
        if (more) load(k0 + BK);
        const int kn = min(BK, kend - k0);
        for (int k = 0; k < kn; ++k) {
            double a[8], b[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) a[u] = As[buf][ty * 8 + u][k];
#pragma unroll
            for (int v = 0; v < 8; ++v) b[v] = Bs[buf][k][tx + 16 * v];
#pragma unroll
            for (int u = 0; u < 8; ++u)
#pragma unroll
                for (int v = 0; v < 8; ++v) acc[u][v] = fma(a[u], b[v], acc[u][v]);
        }
        if (more) store(buf ^ 1);
        __syncthreads();
        buf ^= 1;
    }
#pragma unroll
    for (int u = 0; u < 8; ++u) {
        const int gr = row0 + ty * 8 + u;
        if (gr >= R) continue;
#pragma unroll
        for (int v = 0; v < 8; ++v) {
            const int gc = col0 + tx + 16 * v;
            if (gc < n) part[((int64_t)blockIdx.z * R + gr) * n + gc] = acc[u][v];
        }
    }
}

// ---------------------------------------------------------------------------
// S^T = X^T T with T generated in place (matrix-free, R > 16): the tiled
// product above with its T slab computed from the pair formulas
// (plx_t_element) instead of loaded, so every element of T is evaluated once
// per 64-column row tile of X^T and a batch of many columns costs about one
// dense FP64 product.  Same K chunks and per-element FMA order as the stored
// kernels.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kTiledThreads) otf_tiled_partial(int R, int n, int kchunk, int N, int fmu,
                                                                   const double *__restrict__ pos,
                                                                   const double *__restrict__ par,
                                                                   const double *__restrict__ Xt,
                                                                   double *__restrict__ part) {
    __shared__ double As[BM][BK + 1];
    __shared__ double Bs[BK][BN];
    const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
    const int row0 = blockIdx.y * BM, col0 = blockIdx.x * BN;
    const int kbeg = blockIdx.z * kchunk, kend = min(n, kbeg + kchunk);
    double acc[8][8];
#pragma unroll
    for (int u = 0; u < 8; ++u)
#pragma unroll
        for (int v = 0; v < 8; ++v) acc[u][v] = 0.0;
    for (int k0 = kbeg; k0 < kend; k0 += BK) {
        __syncthreads();
        for (int e = threadIdx.x; e < BM * BK; e += kTiledThreads) {
            const int r = e / BK, k = e % BK, gr = row0 + r, gk = k0 + k;
            As[r][k] = (gr < R && gk < kend) ? Xt[(int64_t)gr * n + gk] : 0.0;
        }
#pragma unroll 1
        for (int e = threadIdx.x; e < BK * BN; e += kTiledThreads) {
            const int k = e / BN, c = e % BN, gk = k0 + k, gc = col0 + c;
            Bs[k][c] = (gk < kend && gc < n) ? plx_t_element(N, fmu != 0, pos, par, gk, gc) : 0.0;
        }
        __syncthreads();
        const int kn = min(BK, kend - k0);
        for (int k = 0; k < kn; ++k) {
            double a[8], b[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) a[u] = As[ty * 8 + u][k];
#pragma unroll
            for (int v = 0; v < 8; ++v) b[v] = Bs[k][tx + 16 * v];
#pragma unroll
            for (int u = 0; u < 8; ++u)
#pragma unroll
                for (int v = 0; v < 8; ++v) acc[u][v] = fma(a[u], b[v], acc[u][v]);
        }
    }
#pragma unroll
    for (int u = 0; u < 8; ++u) {
        const int gr = row0 + ty * 8 + u;
        if (gr >= R) continue;
#pragma unroll
        for (int v = 0; v < 8; ++v) {
            const int gc = col0 + tx + 16 * v;
            if (gc < n) part[((int64_t)blockIdx.z * R + gr) * n + gc] = acc[u][v];
        }
    }
}

// ---------------------------------------------------------------------------
// S = T X generated on the fly (matrix-free), CB columns per launch.
// One thread per target atom; source atoms staged in shared memory.
// ---------------------------------------------------------------------------
constexpr int kOtfThreads = 128;

template <int CB, bool FMU>
__global__ void __launch_bounds__(kOtfThreads) otf_contract(int N, int count, int nv,
                                                            const double *__restrict__ pos,
                                                            const double *__restrict__ par,
                                                            const double *__restrict__ X,
                                                            double *__restrict__ S) {
    constexpr int NC = FMU ? 4 : 1;            // components per atom
    __shared__ double sp[kOtfThreads][5];       // x, y, z, r_q, r_mu
    __shared__ double sxv[kOtfThreads][NC * 2 * CB];
    int i = blockIdx.x * kOtfThreads + threadIdx.x;
    bool live = i < N;
    double xi = 0, yi = 0, zi = 0, rqi = 1, rmi = 1, etai = 0;
    if (live) {
        xi = pos[i];
        yi = pos[N + i];
        zi = pos[2 * N + i];
        rqi = par[i];
        rmi = par[N + i];
        etai = par[2 * N + i];
    }
    double acc[NC][2][CB];
#pragma unroll
    for (int a = 0; a < NC; ++a)
#pragma unroll
        for (int p = 0; p < 2; ++p)
#pragma unroll
            for (int c = 0; c < CB; ++c) acc[a][p][c] = 0.0;
    for (int j0 = 0; j0 < N; j0 += kOtfThreads) {
        int j = j0 + threadIdx.x;
        __syncthreads();
        if (j < N) {
            sp[threadIdx.x][0] = pos[j];
            sp[threadIdx.x][1] = pos[N + j];
            sp[threadIdx.x][2] = pos[2 * N + j];
            sp[threadIdx.x][3] = par[j];
            sp[threadIdx.x][4] = par[N + j];
#pragma unroll
            for (int c = 0; c < CB; ++c) {
                const double *xc = X + (int64_t)c * 2 * nv;
                for (int p = 0; p < 2; ++p) {
                    sxv[threadIdx.x][(0 * 2 + p) * CB + c] = (c < count) ? xc[p * nv + j] : 0.0;
                    if (FMU)
                        for (int k = 0; k < 3; ++k)
                            sxv[threadIdx.x][((1 + k) * 2 + p) * CB + c] =
                                (c < count) ? xc[p * nv + N + 3 * j + k] : 0.0;
                }
            }
        }
        __syncthreads();
        if (!live) continue;
        int jn = min(kOtfThreads, N - j0);
        for (int t = 0; t < jn; ++t) {
            int jj = j0 + t;
            const double *xv = sxv[t];
            if (jj == i) {
#pragma unroll
                for (int p = 0; p < 2; ++p)
#pragma unroll
                    for (int c = 0; c < CB; ++c) acc[0][p][c] = fma(etai, xv[p * CB + c], acc[0][p][c]);
                continue;
            }
            double dx = xi - sp[t][0], dy = yi - sp[t][1], dz = zi - sp[t][2];
            if (!FMU) {
                double q = plx_pair_qq(dx, dy, dz, rqi, sp[t][3]);
#pragma unroll
                for (int p = 0; p < 2; ++p)
#pragma unroll
                    for (int c = 0; c < CB; ++c) acc[0][p][c] = fma(q, xv[p * CB + c], acc[0][p][c]);
                continue;
            }
            PairTile tl;
            plx_pair_tile(dx, dy, dz, rqi, rmi, sp[t][3], sp[t][4], tl);
#pragma unroll
            for (int p = 0; p < 2; ++p)
#pragma unroll
                for (int c = 0; c < CB; ++c) {
                    double xq = xv[(0 * 2 + p) * CB + c];
                    double m0 = xv[(1 * 2 + p) * CB + c];
                    double m1 = xv[(2 * 2 + p) * CB + c];
                    double m2 = xv[(3 * 2 + p) * CB + c];
                    acc[0][p][c] += tl.qq * xq + tl.qm[0] * m0 + tl.qm[1] * m1 + tl.qm[2] * m2;
                    acc[1][p][c] += tl.mq[0] * xq + tl.mm[0] * m0 + tl.mm[1] * m1 + tl.mm[2] * m2;
                    acc[2][p][c] += tl.mq[1] * xq + tl.mm[1] * m0 + tl.mm[3] * m1 + tl.mm[4] * m2;
                    acc[3][p][c] += tl.mq[2] * xq + tl.mm[2] * m0 + tl.mm[4] * m1 + tl.mm[5] * m2;
                }
        }
    }
    if (!live) return;
#pragma unroll
    for (int c = 0; c < CB; ++c) {
        if (c >= count) break;
        double *sc = S + (int64_t)c * 2 * nv;
#pragma unroll
        for (int p = 0; p < 2; ++p) {
            sc[p * nv + i] = acc[0][p][c];
            if (FMU)
                for (int k = 0; k < 3; ++k) sc[p * nv + N + 3 * i + k] = acc[1 + k][p][c];
        }
    }
}

// ---------------------------------------------------------------------------
// Charge rows: y_i = sum_j c_ij (s_j - s_i), c_ij = K_ij (one atom type) or
// 1/2 (K_ij + (w_tj/w_ti) K_ji) (several types), then + D_q(w) x_i.
// One warp per row and a chunk of kChargeCols columns.  A row of K holds a few
// hundred entries (the Fermi damping reaches ~4 nearest-neighbour distances);
// each lane keeps its share of the row (entries lane, lane + 32, ...) in
// registers and reuses it for every column, so the CSR is read once per row
// and chunk instead of once per column.  Per column every lane sums its
// entries in CSR order and the warp adds the lanes with a fixed butterfly, so
// a column's result does not depend on the batch it is in.
// ---------------------------------------------------------------------------
constexpr int kChargeCols = 32;
constexpr int kChargeReg = 16;              // entries per lane held in registers (rows up to 512)

template <bool HETERO>
__device__ __forceinline__ void charge_term(int nt, int ti, int tj, int f, double k, double kt,
                                            const Cplx *__restrict__ wratio, double dre, double dim,
                                            double &yre, double &yim) {
    if (!HETERO) {
        yre = fma(k, dre, yre);
        yim = fma(k, dim, yim);
    } else {
        Cplx w = wratio[ti + nt * tj + (int64_t)nt * nt * f];
        double cre = 0.5 * (k + w.re * kt), cim = 0.5 * (w.im * kt);
        yre += cre * dre - cim * dim;
        yim += cre * dim + cim * dre;
    }
}

template <bool HETERO>
__global__ void __launch_bounds__(256) charge_rows(int N, int nt, int nv, int count,
                                                   const int32_t *__restrict__ freq,
                                                   const int32_t *__restrict__ type,
                                                   const int32_t *__restrict__ rowptr,
                                                   const int32_t *__restrict__ col,
                                                   const double *__restrict__ kval,
                                                   const double *__restrict__ ktval,
                                                   const Cplx *__restrict__ wratio, const Cplx *__restrict__ dq,
                                                   const double *__restrict__ S, const double *__restrict__ X,
                                                   double *__restrict__ Y, double sign, int add_diag) {
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (i >= N) return;
    const int c0 = blockIdx.y * kChargeCols;
    const int c1 = min(count, c0 + kChargeCols);
    const int e0 = rowptr[i], e1 = rowptr[i + 1];
    const bool in_reg = e1 - e0 <= 32 * kChargeReg;
    const int ti = type[i];
    constexpr int HR = HETERO ? kChargeReg : 1;
    int rj[kChargeReg], rt[HR];
    double rk[kChargeReg], rkt[HR];
#pragma unroll
    for (int t = 0; t < kChargeReg; ++t) {
        const int e = e0 + lane + 32 * t;
        const bool live = in_reg && e < e1;
        rj[t] = live ? col[e] : 0;
        rk[t] = live ? kval[e] : 0.0;
        if (HETERO) {
            rkt[t % HR] = live ? ktval[e] : 0.0;
            rt[t % HR] = live ? type[rj[t]] : 0;
        }
    }
    for (int c = c0; c < c1; ++c) {
        const int f = freq[c];
        const double *sr = S + (int64_t)c * 2 * nv;
        const double *si = sr + nv;
        const double s_re = sr[i], s_im = si[i];
        double yre = 0.0, yim = 0.0;
        if (in_reg) {
#pragma unroll
            for (int t = 0; t < kChargeReg; ++t) {
                if (e0 + lane + 32 * t < e1) {
                    const int j = rj[t];
                    charge_term<HETERO>(nt, ti, HETERO ? rt[t % HR] : 0, f, rk[t], HETERO ? rkt[t % HR] : 0.0,
                                        wratio, sr[j] - s_re, si[j] - s_im, yre, yim);
                }
            }
        } else {
            for (int e = e0 + lane; e < e1; e += 32) {
                const int j = col[e];
                charge_term<HETERO>(nt, ti, HETERO ? type[j] : 0, f, kval[e], HETERO ? ktval[e] : 0.0, wratio,
                                    sr[j] - s_re, si[j] - s_im, yre, yim);
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            yre += __shfl_xor_sync(0xffffffffu, yre, o);
            yim += __shfl_xor_sync(0xffffffffu, yim, o);
        }
        if (lane == 0) {
            yre *= sign;
            yim *= sign;
            if (add_diag) {
                const Cplx d = dq[ti + nt * f];
                const double xr = X[(int64_t)c * 2 * nv + i], xi = X[(int64_t)c * 2 * nv + nv + i];
                yre += d.re * xr - d.im * xi;
                yim += d.re * xi + d.im * xr;
            }
            Y[(int64_t)c * 2 * nv + i] = yre;
            Y[(int64_t)c * 2 * nv + nv + i] = yim;
        }
    }
}

// Dipole rows: y = s + (sum_t f_t,i / alpha_t(w)) x.
__global__ void dipole_rows(int N, int nt, int nv, int count, const int32_t *__restrict__ freq,
                            const double *__restrict__ frac, const Cplx *__restrict__ inv_alpha,
                            const double *__restrict__ S, const double *__restrict__ X,
                            double *__restrict__ Y) {
    int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    int c = blockIdx.y;
    if (e >= 3LL * N || c >= count) return;
    int i = (int)(e / 3);
    int f = freq[c];
    double zre = 0.0, zim = 0.0;
    for (int t = 0; t < nt; ++t) {
        double fr = frac[t + (int64_t)nt * i];
        Cplx a = inv_alpha[t + nt * f];
        zre += fr * a.re;
        zim += fr * a.im;
    }
    int64_t r = N + e;
    const double *sc = S + (int64_t)c * 2 * nv;
    const double *xc = X + (int64_t)c * 2 * nv;
    double xr = xc[r], xi = xc[nv + r];
    Y[(int64_t)c * 2 * nv + r] = sc[r] + zre * xr - zim * xi;
    Y[(int64_t)c * 2 * nv + nv + r] = sc[nv + r] + zre * xi + zim * xr;
}

// Rows after a contraction with the folded A0 = blockdiag(K - P, I) T (one atom
// type): only the diagonal D(w) is left, y = s + D(w) x, with -z(w) on the
// charge rows and sum_t f_t,i / alpha_t(w) on the dipole rows.
__global__ void folded_rows(int N, int nt, int nv, int64_t ldS, int count, const int32_t *__restrict__ freq,
                            const int32_t *__restrict__ type, const Cplx *__restrict__ dq,
                            const double *__restrict__ frac, const Cplx *__restrict__ inv_alpha,
                            const double *__restrict__ S, const double *__restrict__ X,
                            double *__restrict__ Y) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    const int c = blockIdx.y;
    if (r >= nv || c >= count) return;
    const int f = freq[c];
    Cplx d = {0.0, 0.0};
    if (r < N) {
        d = dq[type[r] + nt * f];
    } else {
        const int i = (r - N) / 3;
        for (int t = 0; t < nt; ++t) {
            const double fr = frac[t + (int64_t)nt * i];
            const Cplx a = inv_alpha[t + nt * f];
            d.re += fr * a.re;
            d.im += fr * a.im;
        }
    }
    const int64_t base = (int64_t)c * 2 * nv, sb = (int64_t)c * 2 * ldS;
    const double xr = X[base + r], xi = X[base + nv + r];
    Y[base + r] = S[sb + r] + d.re * xr - d.im * xi;
    Y[base + nv + r] = S[sb + ldS + r] + d.re * xi + d.im * xr;
}

// Alloy correction after the folded contraction: for every interface row i,
//   y_i += sum_{j of another type} 1/2 (w_tj/w_ti(w) - 1) K_ji (s_j - s_i),
// s = T x of the interface atoms (rows n + position in J of the output).
// One thread per (interface row, column).
__global__ void iface_rows(int nx, int count, int nt, int nv, int64_t ldS, const int32_t *__restrict__ freq,
                           const int32_t *__restrict__ type, const int32_t *__restrict__ xrow,
                           const int32_t *__restrict__ xipos, const int32_t *__restrict__ xrowptr,
                           const int32_t *__restrict__ xcol, const int32_t *__restrict__ xtj,
                           const double *__restrict__ xkt, const Cplx *__restrict__ wratio,
                           const double *__restrict__ S, double *__restrict__ Y) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int c = blockIdx.y;
    if (t >= nx || c >= count) return;
    const int i = xrow[t], f = freq[c], ti = type[i];
    const double *sr = S + (int64_t)c * 2 * ldS + nv, *si = sr + ldS;
    const double s_re = sr[xipos[t]], s_im = si[xipos[t]];
    double yre = 0.0, yim = 0.0;
    for (int e = xrowptr[t]; e < xrowptr[t + 1]; ++e) {
        const int p = xcol[e];
        const Cplx w = wratio[ti + nt * xtj[e] + (int64_t)nt * nt * f];
        const double cre = 0.5 * (w.re - 1.0) * xkt[e], cim = 0.5 * w.im * xkt[e];
        const double dre = sr[p] - s_re, dim = si[p] - s_im;
        yre += cre * dre - cim * dim;
        yim += cre * dim + cim * dre;
    }
    Y[(int64_t)c * 2 * nv + i] += yre;
    Y[(int64_t)c * 2 * nv + nv + i] += yim;
}

// Static potential V_i (field along pol) for the right-hand side.
__global__ void potential_kernel(int N, int nv, int count, const int32_t *__restrict__ pol,
                                 const double *__restrict__ pos, double e0, int use_min,
                                 double mx, double my, double mz, double *__restrict__ V) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int c = blockIdx.y;
    if (i >= nv || c >= count) return;
    double v = 0.0;
    if (i < N) {
        int p = pol[c];
        double x = pos[(int64_t)p * N + i];
        double m = p == 0 ? mx : (p == 1 ? my : mz);
        v = use_min ? -e0 * fabs(x - m) : -e0 * x;
    }
    V[(int64_t)c * 2 * nv + i] = v;
    V[(int64_t)c * 2 * nv + nv + i] = 0.0;
}

// Dipole part of the right-hand side: E0 on the polarisation component.
__global__ void rhs_dipole(int N, int nv, int count, const int32_t *__restrict__ pol, double e0,
                           double *__restrict__ B) {
    int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    int c = blockIdx.y;
    if (e >= 3LL * N || c >= count) return;
    int k = (int)(e % 3);
    B[(int64_t)c * 2 * nv + N + e] = (k == pol[c]) ? e0 : 0.0;
    B[(int64_t)c * 2 * nv + nv + N + e] = 0.0;
}

// Frequency-independent parts of diag(blockdiag(Kop, I) T) on the charge rows.
__global__ void diag_parts(int N, int nt, const double *__restrict__ pos, const double *__restrict__ par,
                           const int32_t *__restrict__ type, const int32_t *__restrict__ rowptr,
                           const int32_t *__restrict__ col, const double *__restrict__ kval,
                           const double *__restrict__ ktval, double *__restrict__ a, double *__restrict__ b) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    double eta = par[2 * N + i], rq = par[i];
    double sa = 0.0;
    for (int t = 0; t < nt; ++t) b[(int64_t)i * nt + t] = 0.0;
    for (int e = rowptr[i]; e < rowptr[i + 1]; ++e) {
        int j = col[e];
        double tij = plx_pair_qq(pos[i] - pos[j], pos[N + i] - pos[N + j], pos[2 * N + i] - pos[2 * N + j], rq,
                                 par[j]);
        sa += kval[e] * (tij - eta);
        b[(int64_t)i * nt + type[j]] += ktval[e] * (tij - eta);
    }
    a[i] = sa;
}

// 1 / diag(A(w)) per column.
__global__ void diag_inverse_kernel(int N, int nt, int nv, int count, int hetero, const int32_t *__restrict__ freq,
                                    const int32_t *__restrict__ type, const double *__restrict__ a,
                                    const double *__restrict__ b, const Cplx *__restrict__ wratio,
                                    const Cplx *__restrict__ dq, const double *__restrict__ frac,
                                    const Cplx *__restrict__ inv_alpha, double *__restrict__ P) {
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    int c = blockIdx.y;
    if (r >= nv || c >= count) return;
    int f = freq[c];
    double re, im;
    if (r < N) {
        int ti = type[r];
        if (!hetero) {
            re = a[r];
            im = 0.0;
        } else {
            re = a[r];
            im = 0.0;
            for (int t = 0; t < nt; ++t) {
                Cplx w = wratio[ti + nt * t + (int64_t)nt * nt * f];
                double bt = b[(int64_t)r * nt + t];
                re += w.re * bt;
                im += w.im * bt;
            }
            re *= 0.5;
            im *= 0.5;
        }
        Cplx d = dq[ti + nt * f];
        re += d.re;
        im += d.im;
    } else {
        int i = (r - N) / 3;
        re = 0.0;
        im = 0.0;
        for (int t = 0; t < nt; ++t) {
            double fr = frac[t + (int64_t)nt * i];
            Cplx al = inv_alpha[t + nt * f];
            re += fr * al.re;
            im += fr * al.im;
        }
    }
    double m = re * re + im * im;
    double *pc = P + (int64_t)c * 2 * nv;
    pc[r] = m > 0.0 ? re / m : 1.0;
    pc[nv + r] = m > 0.0 ? -im / m : 0.0;
}

}  // namespace

void diagonal_inverse(plx_geom *g, const OpBatch &b, double *Pinv) {
    if (is_bem(g)) {
        bem_diagonal_inverse(g, b, Pinv);
        return;
    }
    plx_ctx *ctx = g->ctx;
    const int N = g->n_atoms, nt = g->n_types;
    if (!g->d_diag_a.p) {
        g->d_diag_a.alloc(ctx, N);
        g->d_diag_b.alloc(ctx, (size_t)N * nt);
        diag_parts<<<n_blocks(N, 128), 128, 0, ctx->stream>>>(N, nt, g->d_pos.p, g->d_par.p, g->d_type.p,
                                                              g->d_rowptr.p, g->d_col.p, g->d_kval.p,
                                                              g->d_ktval.p, g->d_diag_a.p, g->d_diag_b.p);
        ctx->launches++;
    }
    diag_inverse_kernel<<<dim3(n_blocks(g->n_var, 256), b.count), 256, 0, ctx->stream>>>(
        N, nt, g->n_var, b.count, nt > 1, b.d_freq, g->d_type.p, g->d_diag_a.p, g->d_diag_b.p, g->d_wratio.p,
        g->d_dq.p, g->d_frac.p, g->d_inv_alpha.p, Pinv);
    ctx->launches++;
    PLX_CHECK_CUDA(cudaGetLastError());
}

void contract_t_impl(plx_geom *g, int count, const double *X, double *S, bool on_the_fly);

void prof_begin(plx_ctx *ctx) {
    if (!ctx->profile) return;
    if (ctx->prof_used + 2 > ctx->prof_events.size()) {
        for (int k = 0; k < 2; ++k) {
            cudaEvent_t e;
            PLX_CHECK_CUDA(cudaEventCreate(&e));
            ctx->prof_events.push_back(e);
        }
    }
    PLX_CHECK_CUDA(cudaEventRecord(ctx->prof_events[ctx->prof_used], ctx->stream));
}

void prof_end(plx_ctx *ctx, int cat, double flops, double bytes) {
    if (!ctx->profile) return;
    PLX_CHECK_CUDA(cudaEventRecord(ctx->prof_events[ctx->prof_used + 1], ctx->stream));
    if (ctx->prof_cat.size() < ctx->prof_events.size() / 2) ctx->prof_cat.resize(ctx->prof_events.size() / 2);
    ctx->prof_cat[ctx->prof_used / 2] = cat;
    ctx->prof_used += 2;
    ctx->prof_flops[cat] += flops;
    ctx->prof_bytes[cat] += bytes;
    ctx->prof_launches[cat] += 1;
}

void contract_t(plx_geom *g, int count, const double *X, double *S, Contraction how) {
    plx_ctx *ctx = g->ctx;
    const double nn = (double)g->n_var;
    const bool otf = how == Contraction::FP64_OTF;
    if (otf && is_bem(g))
        throw Error(PLX_ERR_UNSUPPORTED, "BEM on the fly is not provided (the reference's BEM has no "
                                         "on-the-fly product either); use the on-memory mode");
    prof_begin(ctx);
    // algorithmic: 2 n^2 flops per real column (one product, whatever the
    // emulation); bytes: the stored T once at its storage precision, plus the
    // columns in and out
    double tbytes = 0.0;
    if (how == Contraction::TC3 || how == Contraction::TC1) {
        tc_contract(g, count, X, S, how == Contraction::TC3 ? 3 : 1);
        tbytes = (how == Contraction::TC3 ? 4.0 : 2.0) * nn * (double)g->ldk;
    } else {
        contract_t_impl(g, count, X, S, otf);
        tbytes = otf ? 0.0 : 8.0 * nn * nn;
    }
    prof_end(ctx, (how == Contraction::TC3 || how == Contraction::TC1) ? PROF_TC : PROF_FP64,
             2.0 * nn * nn * 2.0 * count, tbytes + 2.0 * 8.0 * nn * 2.0 * count);
}

void contract_t_impl(plx_geom *g, int count, const double *X, double *S, bool on_the_fly) {
    plx_ctx *ctx = g->ctx;
    cudaStream_t st = ctx->stream;
    const int n = g->n_var;
    const int R = 2 * count;
    if (on_the_fly && R > 16) {
        // many columns: tiled product with T generated per slab
        int ks, kchunk;
        skinny_split(n, ks, kchunk);
        size_t need = (size_t)ks * R * n;
        if (g->d_part.n < need) g->d_part.alloc(ctx, need);
        dim3 grid(n_blocks(n, BN), n_blocks(R, BM), ks);
        otf_tiled_partial<<<grid, kTiledThreads, 0, st>>>(R, n, kchunk, g->n_atoms, g->model == PLX_WFQFMU,
                                                          g->d_pos.p, g->d_par.p, X, g->d_part.p);
        skinny_reduce<<<n_blocks((int64_t)R * n, 256), 256, 0, st>>>(n, R, ks, g->d_part.p, S);
        ctx->launches += 2;
        PLX_CHECK_CUDA(cudaGetLastError());
        return;
    }
    if (on_the_fly) {
        const bool fmu = g->model == PLX_WFQFMU;
        for (int c0 = 0; c0 < count; c0 += 4) {
            int cb = std::min(4, count - c0);
            const double *Xc = X + (int64_t)c0 * 2 * n;
            double *Sc = S + (int64_t)c0 * 2 * n;
            int blocks = n_blocks(g->n_atoms, kOtfThreads);
            if (fmu)
                otf_contract<4, true><<<blocks, kOtfThreads, 0, st>>>(g->n_atoms, cb, n, g->d_pos.p,
                                                                     g->d_par.p, Xc, Sc);
            else
                otf_contract<4, false><<<blocks, kOtfThreads, 0, st>>>(g->n_atoms, cb, n, g->d_pos.p,
                                                                      g->d_par.p, Xc, Sc);
            ctx->launches++;
        }
        PLX_CHECK_CUDA(cudaGetLastError());
        return;
    }
    if (!g->has_T) throw Error(PLX_ERR_ARG, "geometry was created without the dense T matrix");
    // K split: depends on n only (not on the batch), see tiled_partial
    const int cb = n_blocks(n, kSkinnyCols);
    int ks, kchunk;
    skinny_split(n, ks, kchunk);
    size_t need = (size_t)ks * R * n;
    if (g->d_part.n < need) g->d_part.alloc(ctx, need);
    double *part = g->d_part.p;
    if (R <= 16) {
        dim3 grid(cb, ks);
        switch (R) {
#define PLX_SK(RR) \
    case RR: skinny_partial<RR><<<grid, kSkinnyCols, 0, st>>>(n, kchunk, X, g->d_T.p, part); break;
            PLX_SK(2) PLX_SK(4) PLX_SK(6) PLX_SK(8) PLX_SK(10) PLX_SK(12) PLX_SK(14) PLX_SK(16)
#undef PLX_SK
            default: throw Error(PLX_ERR_ARG, "bad skinny row count");
        }
    } else {
        dim3 grid(n_blocks(n, BN), n_blocks(R, BM), ks);
        tiled_partial<<<grid, kTiledThreads, 0, st>>>(R, n, kchunk, X, g->d_T.p, part);
    }
    skinny_reduce<<<n_blocks((int64_t)R * n, 256), 256, 0, st>>>(n, R, ks, part, S);
    ctx->launches += 2;
    PLX_CHECK_CUDA(cudaGetLastError());
}

static void finish_rows(plx_geom *g, const OpBatch &b, const double *S, const double *X,
                        double *Y) {
    plx_ctx *ctx = g->ctx;
    cudaStream_t st = ctx->stream;
    const int N = g->n_atoms, nv = g->n_var;
    dim3 gq(n_blocks((int64_t)N * 32, 256), n_blocks(b.count, kChargeCols));
    (g->n_types > 1 ? charge_rows<true> : charge_rows<false>)<<<gq, 256, 0, st>>>(N, g->n_types, nv, b.count, b.d_freq,
                                    g->d_type.p, g->d_rowptr.p, g->d_col.p, g->d_kval.p,
                                    g->d_ktval.p, g->d_wratio.p, g->d_dq.p, S, X, Y, 1.0, 1);
    ctx->launches++;
    if (g->model == PLX_WFQFMU) {
        dim3 gm(n_blocks(3LL * N, 256), b.count);
        dipole_rows<<<gm, 256, 0, st>>>(N, g->n_types, nv, b.count, b.d_freq, g->d_frac.p,
                                        g->d_inv_alpha.p, S, X, Y);
        ctx->launches++;
    }
    PLX_CHECK_CUDA(cudaGetLastError());
}

// Output of the folded tensor-core contraction of b.count columns: the work
// array, or for alloys (interface rows after the n operator rows) the
// geometry's fold buffer.
static double *folded_output(plx_geom *g, const OpBatch &b, double *work) {
    const int64_t M = tc_fold_rows(g);
    if (M <= g->n_var) return work;
    const size_t need = (size_t)b.count * 2 * M;
    if (g->d_fold_work.n < need) g->d_fold_work.alloc(g->ctx, need);
    return g->d_fold_work.p;
}

// Y = S + D(w) X after the folded contraction S = A0 X (and the interface
// correction of alloys).
static void folded_finish(plx_geom *g, const OpBatch &b, const double *S, const double *X, double *Y) {
    plx_ctx *ctx = g->ctx;
    const int64_t M = g->fold_rows;
    prof_begin(ctx);
    folded_rows<<<dim3(n_blocks(g->n_var, 256), b.count), 256, 0, ctx->stream>>>(
        g->n_atoms, g->n_types, g->n_var, M, b.count, b.d_freq, g->d_type.p, g->d_dq.p, g->d_frac.p,
        g->d_inv_alpha.p, S, X, Y);
    ctx->launches++;
    if (g->n_xrows > 0) {
        iface_rows<<<dim3(n_blocks(g->n_xrows, 128), b.count), 128, 0, ctx->stream>>>(
            g->n_xrows, b.count, g->n_types, g->n_var, M, b.d_freq, g->d_type.p, g->d_xrow.p, g->d_xipos.p,
            g->d_xrowptr.p, g->d_xcol.p, g->d_xtj.p, g->d_xkt.p, g->d_wratio.p, S, Y);
        ctx->launches++;
    }
    PLX_CHECK_CUDA(cudaGetLastError());
    prof_end(ctx, PROF_ROWS, 0.0, 0.0);
}

static double tc_bytes(plx_geom *g, Contraction how, int count) {
    const double nn = (double)g->n_var;
    return (how == Contraction::TC3 ? 4.0 : 2.0) * (double)g->fold_rows * (double)g->ldk + 2.0 * 8.0 * nn * 2.0 * count;
}

void apply_operator(plx_geom *g, const OpBatch &b, const double *X, double *Y, double *work,
                    Contraction how) {
    if (b.count == 0) return;
    if ((how == Contraction::TC3 || how == Contraction::TC1) && tc_folds_operator(g)) {
        // A(w) X = A0 X + D(w) X: one tensor-core contraction with the folded
        // matrix and a diagonal pass (no conductance rows per application)
        plx_ctx *ctx = g->ctx;
        const double nn = (double)g->n_var;
        double *S = folded_output(g, b, work);
        prof_begin(ctx);
        tc_contract(g, b.count, X, S, how == Contraction::TC3 ? 3 : 1, true);
        prof_end(ctx, PROF_TC, 2.0 * nn * nn * 2.0 * b.count, tc_bytes(g, how, b.count));
        folded_finish(g, b, S, X, Y);
        return;
    }
    contract_t(g, b.count, X, work, how);
    prof_begin(g->ctx);
    if (is_bem(g))
        bem_apply_rows(g, b, work, X, Y);
    else
        finish_rows(g, b, work, X, Y);
    prof_end(g->ctx, PROF_ROWS, 0.0, 0.0);
}

void apply_operator_group(const std::vector<OpInput> &items) {
    // the folded tensor-core contractions that can share a launch: same context,
    // same product count, distinct geometries
    std::vector<size_t> grp;
    for (size_t i = 0; i < items.size(); ++i) {
        const OpInput &it = items[i];
        if (it.b.count == 0 || !(it.how == Contraction::TC3 || it.how == Contraction::TC1) ||
            !tc_folds_operator(it.g))
            continue;
        bool ok = true;
        for (size_t k : grp)
            ok = ok && items[k].g != it.g && items[k].g->ctx == it.g->ctx && items[k].how == it.how;
        if (ok) grp.push_back(i);
    }
    if (grp.size() < 2) {
        for (const OpInput &it : items) apply_operator(it.g, it.b, it.X, it.Y, it.work, it.how);
        return;
    }
    plx_ctx *ctx = items[grp[0]].g->ctx;
    std::vector<TcItem> ti;
    std::vector<double *> S;
    double flops = 0.0, bytes = 0.0;
    for (size_t k : grp) {
        const OpInput &it = items[k];
        S.push_back(folded_output(it.g, it.b, it.work));
        ti.push_back(TcItem{it.g, it.b.count, it.X, S.back(), it.how == Contraction::TC3 ? 3 : 1, true});
        const double nn = (double)it.g->n_var;
        flops += 2.0 * nn * nn * 2.0 * it.b.count;
        bytes += tc_bytes(it.g, it.how, it.b.count);
    }
    prof_begin(ctx);
    tc_contract_group(ti);
    prof_end(ctx, PROF_TC, flops, bytes);
    for (size_t j = 0; j < grp.size(); ++j) {
        const OpInput &it = items[grp[j]];
        folded_finish(it.g, it.b, S[j], it.X, it.Y);
    }
    for (size_t i = 0; i < items.size(); ++i)
        if (std::find(grp.begin(), grp.end(), i) == grp.end()) {
            const OpInput &it = items[i];
            apply_operator(it.g, it.b, it.X, it.Y, it.work, it.how);
        }
}

void rhs_batch(plx_geom *g, const OpBatch &b, const int32_t *d_pol, double *Bout) {
    if (b.count == 0) return;
    if (is_bem(g)) {
        bem_rhs(g, b, d_pol, Bout);
        return;
    }
    plx_ctx *ctx = g->ctx;
    cudaStream_t st = ctx->stream;
    const int N = g->n_atoms, nv = g->n_var;
    double mn[3] = {0, 0, 0};
    if (g->rhs_potential) {
        for (int k = 0; k < 3; ++k) {
            mn[k] = g->coord[k];
            for (int i = 0; i < N; ++i) mn[k] = std::min(mn[k], g->coord[k + 3 * i]);
        }
    }
    DevArray<double> V;
    V.alloc(ctx, (size_t)b.count * 2 * nv);
    potential_kernel<<<dim3(n_blocks(nv, 256), b.count), 256, 0, st>>>(
        N, nv, b.count, d_pol, g->d_pos.p, g->e0, g->rhs_potential, mn[0], mn[1], mn[2], V.p);
    dim3 gq(n_blocks((int64_t)N * 32, 256), n_blocks(b.count, kChargeCols));
    // b_q = -Kop(w) V  (rhs_module.f90:140-390); no diagonal term
    (g->n_types > 1 ? charge_rows<true> : charge_rows<false>)<<<gq, 256, 0, st>>>(N, g->n_types, nv, b.count, b.d_freq,
                                    g->d_type.p, g->d_rowptr.p, g->d_col.p, g->d_kval.p,
                                    g->d_ktval.p, g->d_wratio.p, g->d_dq.p, V.p, V.p, Bout, -1.0, 0);
    ctx->launches += 2;
    if (g->model == PLX_WFQFMU) {
        dim3 gm(n_blocks(3LL * N, 256), b.count);
        rhs_dipole<<<gm, 256, 0, st>>>(N, nv, b.count, d_pol, g->e0, Bout);
        ctx->launches++;
    }
    PLX_CHECK_CUDA(cudaGetLastError());
    PLX_CHECK_CUDA(cudaStreamSynchronize(st));
}

}  // namespace plx
