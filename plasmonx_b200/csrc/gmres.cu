// Batched complex GMRES in FP64 with the reference's semantics
// (src/solvers/gmres_module.f90:30-228), one independent Krylov space per
// column (frequency x polarisation), all columns advanced in lock step so that
// every Arnoldi step is ONE batched operator application.
//
// Per column, exactly as the reference: x0 = 0, v1 = b/||b||, Arnoldi with
// modified Gram-Schmidt for j < 25 and classical Gram-Schmidt with one
// re-orthogonalisation for j >= 25, Givens rotations with reference-BLAS
// zrotg/zrot semantics, the logged residual |g_{j+1}| compared with the
// absolute tolerance, then the triangular solve, x += V y and the true
// residual ||b - A x|| deciding convergence; no restart.
//
// Storage: Krylov vectors are kept in "slabs", one per step j, each holding
// the j-th basis vector of every column ([C][2][n] split complex), allocated
// when the step is reached so that memory follows the actual iteration count.
// The inner solves of a refinement may keep their basis in FP32 (half the
// projection traffic); dot products, Hessenberg, rotations and the iterate stay
// FP64, and the refinement's FP64 residual absorbs the storage rounding.
// Columns that converge leave the active list; the operator and the Arnoldi
// kernels only touch active columns.
#include <algorithm>
#include <cmath>
#include <memory>

#include "plx_internal.h"

namespace plx {

namespace {

constexpr int kRows = 2048;     // rows per block in the Arnoldi kernels
constexpr int kThreads = 256;

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Block reduction of two doubles; result valid in thread 0.
__device__ __forceinline__ void block_sum2(double &a, double &b) {
    __shared__ double ra[32], rb[32];
    a = warp_sum(a);
    b = warp_sum(b);
    int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) {
        ra[w] = a;
        rb[w] = b;
    }
    __syncthreads();
    if (w == 0) {
        int nw = blockDim.x >> 5;
        a = l < nw ? ra[l] : 0.0;
        b = l < nw ? rb[l] : 0.0;
        a = warp_sum(a);
        b = warp_sum(b);
    }
}

// Copies column act[k] of slab j into the compact batch X[k].
template <typename VT>
__global__ void gather_cols(int n, const int32_t *__restrict__ act, const VT *__restrict__ slab,
                            double *__restrict__ X) {
    int k = blockIdx.y;
    const VT *src = slab + (int64_t)act[k] * 2 * n;
    double *dst = X + (int64_t)k * 2 * n;
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < 2LL * n;
         r += (int64_t)gridDim.x * blockDim.x)
        dst[r] = src[r];
}

// Partial complex dots conj(V_i[c]) . W[k] for i in [i0, i1) over one chunk of
// kDotRows rows: every thread keeps kDotPT entries of W in registers and all
// eight warps work on every basis vector (warp reduction, then a fixed-order
// sum over the warps), so the kernel is bandwidth-bound for any number of
// basis vectors, including the single-vector projections of modified
// Gram-Schmidt.
constexpr int kDotPT = 4;
constexpr int kDotRows = kThreads * kDotPT;

template <typename VT>
__global__ void __launch_bounds__(kThreads) dots_partial(int n, int i0, int i1,
                                                         const int32_t *__restrict__ act,
                                                         VT *const *__restrict__ slabs,
                                                         const double *__restrict__ W,
                                                         double2 *__restrict__ part) {
    __shared__ double2 red[kThreads / 32][32];
    const int k = blockIdx.y, c = act[k];
    const int r0 = blockIdx.x * kDotRows;
    const double *wr = W + (int64_t)k * 2 * n;
    double wre[kDotPT], wim[kDotPT];
#pragma unroll
    for (int q = 0; q < kDotPT; ++q) {
        int r = r0 + threadIdx.x + kThreads * q;
        wre[q] = r < n ? wr[r] : 0.0;
        wim[q] = r < n ? wr[n + r] : 0.0;
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ni = i1 - i0;
    for (int g0 = 0; g0 < ni; g0 += 32) {
        const int gn = min(32, ni - g0);
        for (int t = 0; t < gn; ++t) {
            const VT *v = slabs[i0 + g0 + t] + (int64_t)c * 2 * n;
            double re = 0.0, im = 0.0;
#pragma unroll
            for (int q = 0; q < kDotPT; ++q) {
                int r = r0 + threadIdx.x + kThreads * q;
                if (r < n) {
                    double vr = (double)v[r], vi = (double)v[n + r];
                    re += vr * wre[q] + vi * wim[q];      // conj(v) * w
                    im += vr * wim[q] - vi * wre[q];
                }
            }
            re = warp_sum(re);
            im = warp_sum(im);
            if (lane == 0) red[warp][t] = make_double2(re, im);
        }
        __syncthreads();
        if (threadIdx.x < gn) {
            double2 s = make_double2(0.0, 0.0);
            for (int w = 0; w < kThreads / 32; ++w) {
                s.x += red[w][threadIdx.x].x;
                s.y += red[w][threadIdx.x].y;
            }
            part[((int64_t)k * gridDim.x + blockIdx.x) * ni + g0 + threadIdx.x] = s;
        }
        __syncthreads();
    }
}

// The same partial dots for projections onto eight or more basis vectors
// (classical Gram-Schmidt): the chunk of W is staged in shared memory once and
// each warp takes whole basis vectors, 32 rows per lane with the loads of 16
// rows in flight, so one warp reduction serves 1,024 rows of a vector (the
// kernel above pays one per 128 rows and keeps only 8 loads in flight a warp).
// Same chunking and partial layout as dots_partial.
template <typename VT>
__global__ void __launch_bounds__(kThreads) dots_wide(int n, int i0, int i1,
                                                      const int32_t *__restrict__ act,
                                                      VT *const *__restrict__ slabs,
                                                      const double *__restrict__ W,
                                                      double2 *__restrict__ part) {
    __shared__ double wsh[2][kDotRows];
    const int k = blockIdx.y, c = act[k];
    const int r0 = blockIdx.x * kDotRows;
    const int rn = min(kDotRows, n - r0);
    const double *wr = W + (int64_t)k * 2 * n;
    for (int t = threadIdx.x; t < kDotRows; t += kThreads) {
        wsh[0][t] = t < rn ? wr[r0 + t] : 0.0;
        wsh[1][t] = t < rn ? wr[n + r0 + t] : 0.0;
    }
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ni = i1 - i0;
    for (int ii = warp; ii < ni; ii += kThreads / 32) {
        const VT *v = slabs[i0 + ii] + (int64_t)c * 2 * n + r0;
        double re = 0.0, im = 0.0;
        constexpr int kBatch = 16;
        for (int q0 = 0; q0 < kDotRows / 32; q0 += kBatch) {
            VT vr[kBatch], vi[kBatch];
            if (rn == kDotRows) {
#pragma unroll
                for (int q = 0; q < kBatch; ++q) {
                    vr[q] = v[lane + 32 * (q0 + q)];
                    vi[q] = v[n + lane + 32 * (q0 + q)];
                }
            } else {
#pragma unroll
                for (int q = 0; q < kBatch; ++q) {
                    const int t = lane + 32 * (q0 + q);
                    vr[q] = t < rn ? v[t] : VT(0);
                    vi[q] = t < rn ? v[n + t] : VT(0);
                }
            }
#pragma unroll
            for (int q = 0; q < kBatch; ++q) {
                const int t = lane + 32 * (q0 + q);
                const double a = wsh[0][t], b = wsh[1][t];          // zero beyond rn
                re += (double)vr[q] * a + (double)vi[q] * b;        // conj(v) * w
                im += (double)vr[q] * b - (double)vi[q] * a;
            }
        }
        re = warp_sum(re);
        im = warp_sum(im);
        if (lane == 0) part[((int64_t)k * gridDim.x + blockIdx.x) * ni + ii] = make_double2(re, im);
    }
}

// Sums the chunk partials: h[k][ii] = sum_b part[k][b][ii]; optionally accumulates
// into H column j (Hcol[c][i0+ii] += h) when Hslab != nullptr.
__global__ void dots_finish(int nchunk, int ni, int i0, const int32_t *__restrict__ act,
                            const double2 *__restrict__ part, double2 *__restrict__ h,
                            double2 *__restrict__ Hcol, int hstride, int accumulate) {
    int k = blockIdx.y;
    int ii = blockIdx.x * blockDim.x + threadIdx.x;
    if (ii >= ni) return;
    double2 s = make_double2(0.0, 0.0);
    for (int b = 0; b < nchunk; ++b) {
        double2 p = part[((int64_t)k * nchunk + b) * ni + ii];
        s.x += p.x;
        s.y += p.y;
    }
    h[(int64_t)k * ni + ii] = s;
    if (Hcol) {
        double2 *dst = Hcol + (int64_t)act[k] * hstride + i0 + ii;
        if (accumulate) {
            dst->x += s.x;
            dst->y += s.y;
        } else {
            *dst = s;
        }
    }
}

// W[k] -= sum_{ii} V_{i0+ii}[c] h[k][ii]   (sign = -1), or X[c] += ... (sign = +1,
// target indexed by column instead of compact position when by_col != 0).
// Each thread owns kCombineRows rows (strided by the block); the loads of a
// batch of basis vectors are issued before their products are summed (the
// per-row sum runs over ii in ascending order whatever the batching).  Four
// rows per thread measured the same as one (0.65 s of orthogonalisation per two
// spectra of the 41,892-unknown sphere either way), so one it is.
constexpr int kCombineRows = 1;
template <typename VT>
__global__ void __launch_bounds__(kThreads) combine(int n, int i0, int ni, int hld, int hoff,
                                                    const int32_t *__restrict__ act,
                                                    VT *const *__restrict__ slabs,
                                                    const double2 *__restrict__ h, double sign,
                                                    double *__restrict__ Y, int by_col) {
    extern __shared__ double2 sh[];                       // ni coefficients, then ni column pointers
    const VT **col = reinterpret_cast<const VT **>(sh + ni);
    int k = blockIdx.y, c = act[k];
    for (int t = threadIdx.x; t < ni; t += blockDim.x) {
        sh[t] = h[(int64_t)k * hld + hoff + t];
        col[t] = slabs[i0 + t] + (int64_t)c * 2 * n;
    }
    __syncthreads();
    constexpr int RW = kCombineRows;
    const int rbase = blockIdx.x * (kThreads * RW) + threadIdx.x;
    if (rbase >= n) return;
    int rr[RW];
    bool in[RW];
#pragma unroll
    for (int u = 0; u < RW; ++u) {
        rr[u] = rbase + kThreads * u;
        in[u] = rr[u] < n;
        if (!in[u]) rr[u] = rbase;          // a valid row; its sum is not stored
    }
    double ar[RW], ai[RW];
#pragma unroll
    for (int u = 0; u < RW; ++u) ar[u] = ai[u] = 0.0;
    constexpr int kBatch = RW == 1 ? 8 : 4;   // basis vectors whose loads are in flight together
    int ii = 0;
    for (; ii + kBatch <= ni; ii += kBatch) {
        VT vr[kBatch][RW], vi[kBatch][RW];
#pragma unroll
        for (int q = 0; q < kBatch; ++q)
#pragma unroll
            for (int u = 0; u < RW; ++u) {
                vr[q][u] = col[ii + q][rr[u]];
                vi[q][u] = col[ii + q][n + rr[u]];
            }
#pragma unroll
        for (int q = 0; q < kBatch; ++q) {
            const double2 hh = sh[ii + q];
#pragma unroll
            for (int u = 0; u < RW; ++u) {
                ar[u] += (double)vr[q][u] * hh.x - (double)vi[q][u] * hh.y;
                ai[u] += (double)vr[q][u] * hh.y + (double)vi[q][u] * hh.x;
            }
        }
    }
    for (; ii < ni; ++ii) {
        const VT *v = col[ii];
        const double2 hh = sh[ii];
#pragma unroll
        for (int u = 0; u < RW; ++u) {
            const double vr = (double)v[rr[u]], vi = (double)v[n + rr[u]];
            ar[u] += vr * hh.x - vi * hh.y;
            ai[u] += vr * hh.y + vi * hh.x;
        }
    }
    double *y = Y + (int64_t)(by_col ? c : k) * 2 * n;
#pragma unroll
    for (int u = 0; u < RW; ++u) {
        if (!in[u]) continue;
        y[rr[u]] += sign * ar[u];
        y[n + rr[u]] += sign * ai[u];
    }
}

// ||W[k]||_2 (dznrm2): partial sums of squares per chunk.
__global__ void norm_partial(int n, const double *__restrict__ W, double *__restrict__ part) {
    int k = blockIdx.y;
    const double *w = W + (int64_t)k * 2 * n;
    int r0 = blockIdx.x * kRows, rn = min(kRows, n - r0);
    double s = 0.0, dummy = 0.0;
    for (int t = threadIdx.x; t < rn; t += blockDim.x) {
        double a = w[r0 + t], b = w[n + r0 + t];
        s += a * a + b * b;
    }
    block_sum2(s, dummy);
    if (threadIdx.x == 0) part[(int64_t)k * gridDim.x + blockIdx.x] = s;
}

__global__ void norm_finish(int nchunk, int count, const double *__restrict__ part,
                            double *__restrict__ out) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) return;
    double s = 0.0;
    for (int b = 0; b < nchunk; ++b) s += part[(int64_t)k * nchunk + b];
    out[k] = sqrt(s);
}

// v_{j+1}[c] = W[k] / h_{j+1,j} (left zero when the norm is zero, as the
// reference leaves the zero-filled column untouched); H(j+1, j) = norm.
template <typename VT>
__global__ void normalize(int n, const int32_t *__restrict__ act, const double *__restrict__ nrm,
                          const double *__restrict__ W, VT *__restrict__ slab_next,
                          double2 *__restrict__ Hcol, int hstride, int jrow) {
    int k = blockIdx.y, c = act[k];
    double s = nrm[k];
    double inv = s != 0.0 ? 1.0 / s : 0.0;
    const double *w = W + (int64_t)k * 2 * n;
    VT *v = slab_next + (int64_t)c * 2 * n;
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < 2LL * n;
         r += (int64_t)gridDim.x * blockDim.x)
        v[r] = (VT)(s != 0.0 ? w[r] * inv : 0.0);
    if (blockIdx.x == 0 && threadIdx.x == 0) Hcol[(int64_t)c * hstride + jrow] = make_double2(s, 0.0);
}

// v_1 = b / ||b||; g_1 = ||b||.
template <typename VT>
__global__ void start_vectors(int n, const int32_t *__restrict__ act, const double *__restrict__ nrm,
                              const double *__restrict__ B, VT *__restrict__ slab0,
                              double2 *__restrict__ g, int gstride) {
    int k = blockIdx.y, c = act[k];
    double s = nrm[k];
    const double *b = B + (int64_t)c * 2 * n;
    VT *v = slab0 + (int64_t)c * 2 * n;
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < 2LL * n;
         r += (int64_t)gridDim.x * blockDim.x)
        v[r] = (VT)(b[r] * (1.0 / s));
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        g[(int64_t)c * gstride] = make_double2(s, 0.0);
        for (int i = 1; i < gstride; ++i) g[(int64_t)c * gstride + i] = make_double2(0.0, 0.0);
    }
}

__device__ __forceinline__ double cabs_(double2 a) { return hypot(a.x, a.y); }

__device__ __forceinline__ void zrot_(double2 &x, double2 &y, double c, double2 s) {
    double2 nx = make_double2(c * x.x + (s.x * y.x - s.y * y.y), c * x.y + (s.x * y.y + s.y * y.x));
    // y' = c y - conj(s) x
    double2 ny = make_double2(c * y.x - (s.x * x.x + s.y * x.y), c * y.y - (s.x * x.y - s.y * x.x));
    x = nx;
    y = ny;
}

// Givens update of column j for every active column (one thread each).
// Hcols[j] points to the slab of H column j ([C][hstride] complex).
__global__ void givens(int count, int j, const int32_t *__restrict__ act,
                       double2 *const *__restrict__ Hcols, int hstride, double *__restrict__ cs,
                       double2 *__restrict__ sn, double2 *__restrict__ g, int gstride, int cstride,
                       double *__restrict__ resid) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) return;
    int c = act[k];
    double2 *h = Hcols[j] + (int64_t)c * hstride;
    double *csc = cs + (int64_t)c * cstride;
    double2 *snc = sn + (int64_t)c * cstride;
    for (int i = 0; i < j; ++i) zrot_(h[i], h[i + 1], csc[i], snc[i]);
    double2 ca = h[j], cb = h[j + 1];
    double cj;
    double2 sj;
    if (cabs_(ca) == 0.0) {
        cj = 0.0;
        sj = make_double2(1.0, 0.0);
    } else {
        double aa = cabs_(ca), ab = cabs_(cb);
        double scale = aa + ab;
        double2 cas = make_double2(ca.x / scale, ca.y / scale), cbs = make_double2(cb.x / scale, cb.y / scale);
        double t1 = cabs_(cas), t2 = cabs_(cbs);
        double norm = scale * sqrt(t1 * t1 + t2 * t2);
        double2 alpha = make_double2(ca.x / aa, ca.y / aa);
        cj = aa / norm;
        double2 s = cmul(alpha, cconj(cb));
        sj = make_double2(s.x / norm, s.y / norm);
    }
    csc[j] = cj;
    snc[j] = sj;
    double2 *gc = g + (int64_t)c * gstride;
    zrot_(gc[j], gc[j + 1], cj, sj);
    zrot_(h[j], h[j + 1], cj, sj);
    h[j + 1] = make_double2(0.0, 0.0);
    resid[k] = cabs_(gc[j + 1]);
}

// y = R^{-1} g for the triangular R = H(0..j, 0..j) (ztrsv 'U','N','N'): one
// warp per triggered column, column-oriented back substitution with the
// updates of y spread over the lanes; y stored compactly [k][j+1].
__global__ void tri_solve(int count, int j, const int32_t *__restrict__ act,
                          double2 *const *__restrict__ Hcols, int hstride,
                          const double2 *__restrict__ g, int gstride, double2 *__restrict__ y) {
    extern __shared__ double2 ys[];
    int k = blockIdx.x;
    if (k >= count) return;
    int c = act[k];
    int m = j + 1;
    for (int i = threadIdx.x; i < m; i += 32) ys[i] = g[(int64_t)c * gstride + i];
    __syncwarp();
    for (int i = m - 1; i >= 0; --i) {
        const double2 *col = Hcols[i] + (int64_t)c * hstride;
        double2 rii = col[i];
        double d = rii.x * rii.x + rii.y * rii.y;
        double2 v = ys[i];
        double2 yi = make_double2((v.x * rii.x + v.y * rii.y) / d, (v.y * rii.x - v.x * rii.y) / d);
        __syncwarp();
        if (threadIdx.x == 0) ys[i] = yi;
        for (int l = threadIdx.x; l < i; l += 32) {
            double2 p = cmul(col[l], yi);
            ys[l].x -= p.x;
            ys[l].y -= p.y;
        }
        __syncwarp();
    }
    for (int i = threadIdx.x; i < m; i += 32) y[(int64_t)k * m + i] = ys[i];
}

// R[k] = B[c] - AX[k] with c = act[k]; in place into AX.
__global__ void residual(int n, const int32_t *__restrict__ act, const double *__restrict__ B,
                         double *__restrict__ AX) {
    int k = blockIdx.y, c = act[k];
    const double *b = B + (int64_t)c * 2 * n;
    double *r = AX + (int64_t)k * 2 * n;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < 2LL * n;
         t += (int64_t)gridDim.x * blockDim.x)
        r[t] = b[t] - r[t];
}

__global__ void gather_x(int n, const int32_t *__restrict__ act, const double *__restrict__ X,
                         double *__restrict__ out) {
    int k = blockIdx.y;
    const double *src = X + (int64_t)act[k] * 2 * n;
    double *dst = out + (int64_t)k * 2 * n;
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < 2LL * n;
         r += (int64_t)gridDim.x * blockDim.x)
        dst[r] = src[r];
}

// Y[k] *= P[idx[k]] elementwise (complex), or in place on the column itself
// when by_col (Y indexed by idx[k]).
__global__ void scale_cols(int n, const int32_t *__restrict__ idx, const double *__restrict__ P,
                           double *__restrict__ Y, int by_col) {
    int k = blockIdx.y, c = idx[k];
    const double *p = P + (int64_t)c * 2 * n;
    double *y = Y + (int64_t)(by_col ? c : k) * 2 * n;
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x) {
        double pr = p[r], pi = p[n + r], yr = y[r], yi = y[n + r];
        y[r] = pr * yr - pi * yi;
        y[n + r] = pr * yi + pi * yr;
    }
}

int grid_rows(int64_t n2) { return (int)std::min<int64_t>(n_blocks(n2, 256), 1024); }

// combine() over at most kCombine basis vectors per launch (shared-memory bound).
constexpr int kCombine = 1024;
template <typename VT>
int64_t combine_chunked(cudaStream_t st, int n, int i0, int ni, int count, const int32_t *act,
                        VT *const *slabs, const double2 *h, double sign, double *Y, int by_col) {
    int64_t launches = 0;
    for (int c0 = 0; c0 < ni; c0 += kCombine) {
        int cn = std::min(kCombine, ni - c0);
        // h is [count][ni]; pass the row stride through a shifted view per chunk
        combine<VT><<<dim3(n_blocks(n, kThreads * kCombineRows), count), kThreads,
                      cn * (sizeof(double2) + sizeof(VT *)), st>>>(
            n, i0 + c0, cn, ni, c0, act, slabs, h, sign, Y, by_col);
        ++launches;
    }
    return launches;
}

}  // namespace

// Norms ||v[k]|| of a compact batch (used for ||b|| and the true residual).
static void batch_norms(plx_geom *g, int count, const double *V, DevArray<double> &part,
                        DevArray<double> &out) {
    plx_ctx *ctx = g->ctx;
    const int n = g->n_var;
    int nchunk = n_blocks(n, kRows);
    norm_partial<<<dim3(nchunk, count), kThreads, 0, ctx->stream>>>(n, V, part.p);
    norm_finish<<<n_blocks(count, 128), 128, 0, ctx->stream>>>(nchunk, count, part.p, out.p);
    ctx->launches += 2;
}

// One batched GMRES solve, advanced one Arnoldi step at a time so that the
// operator application of every step can be shared with other solves (a
// grouped tensor-core launch over several geometries): begin(), then while
// wants_product(): pre() -> the caller forms W = A X of the returned batch ->
// post(); then end().  gmres_batched runs it with its own operator.
template <typename VT>
class GmresRun final : public GmresStepper {
  public:
    GmresRun(plx_geom *g, const GmresRequest &rq, const double *d_B, double *d_X, GmresResult &res)
        : g_(g), ctx_(g->ctx), st_(g->ctx->stream), rq_(rq), d_B_(d_B), d_X_(d_X), res_(res) {}

    void begin() {
        const int n = g_->n_var;
        C_ = (int)rq_.freq.size();
        m_ = std::min(rq_.m, n);
        res_.status.assign(C_, PLX_OK);
        res_.steps.assign(C_, 0);
        res_.trace.assign(rq_.record_trace ? (size_t)C_ * m_ : 0, 0.0);
        if (C_ == 0) return;
        if (m_ < 1) throw Error(PLX_ERR_ARG, "GMRES dimension must be positive");
        nchunk_ = n_blocks(n, kRows);
        ndot_ = n_blocks(n, kDotRows);
        if ((size_t)(m_ + 1) * sizeof(double2) > 200 * 1024) throw Error(PLX_ERR_ARG, "GMRES dimension above 12800");
        once_per_device(reinterpret_cast<const void *>(tri_solve), ctx_->device, [] {
            PLX_CHECK_CUDA(cudaFuncSetAttribute(tri_solve, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
            PLX_CHECK_CUDA(cudaFuncSetAttribute(combine<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * 1024));
            PLX_CHECK_CUDA(cudaFuncSetAttribute(combine<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * 1024));
        });
        hstride_ = m_ + 1;   // rows of an H column (0..m)
        d_act_.alloc(ctx_, C_);
        d_freq_act_.alloc(ctx_, C_);
        d_cols_.alloc(ctx_, C_);
        Xa_.alloc(ctx_, (size_t)C_ * 2 * n);
        Wa_.alloc(ctx_, (size_t)C_ * 2 * n);
        work_.alloc(ctx_, (size_t)C_ * 2 * n);
        nrm_part_.alloc(ctx_, (size_t)C_ * nchunk_);
        nrm_.alloc(ctx_, C_);
        cs_.alloc(ctx_, (size_t)C_ * m_);
        sn_.alloc(ctx_, (size_t)C_ * m_);
        gv_.alloc(ctx_, (size_t)C_ * hstride_);
        hbuf_.alloc(ctx_, (size_t)C_ * hstride_);
        ybuf_.alloc(ctx_, (size_t)C_ * hstride_);
        std::vector<DevArray<VT>>(m_ + 1).swap(slabs_);
        std::vector<DevArray<double2>>(m_).swap(hcols_);
        d_slabs_.alloc(ctx_, m_ + 1);
        d_hcols_.alloc(ctx_, m_);
        h_slabs_.assign(m_ + 1, nullptr);
        h_hcols_.assign(m_, nullptr);
        PLX_CHECK_CUDA(cudaMemsetAsync(d_X_, 0, (size_t)C_ * 2 * n * 8, st_));
        jac_ = rq_.jacobi && rq_.inner;
        if (jac_) {
            DevArray<int32_t> d_fall;
            d_fall.alloc(ctx_, C_);
            PLX_CHECK_CUDA(cudaMemcpyAsync(d_fall.p, rq_.freq.data(), C_ * 4, cudaMemcpyHostToDevice, st_));
            Pinv_.alloc(ctx_, (size_t)C_ * 2 * n);
            diagonal_inverse(g_, OpBatch{C_, d_fall.p}, Pinv_.p);
        }
        // active list: every column with ||b|| > 0 (the reference returns x = 0 otherwise)
        act_.resize(C_);
        for (int c = 0; c < C_; ++c) act_[c] = c;
        PLX_CHECK_CUDA(cudaMemcpyAsync(d_act_.p, act_.data(), C_ * 4, cudaMemcpyHostToDevice, st_));
        batch_norms(g_, C_, d_B_, nrm_part_, nrm_);   // B is [C] in column order == compact order here
        std::vector<double> bnorm(C_);
        PLX_CHECK_CUDA(cudaMemcpyAsync(bnorm.data(), nrm_.p, C_ * 8, cudaMemcpyDeviceToHost, st_));
        PLX_CHECK_CUDA(cudaStreamSynchronize(st_));
        slabs_[0].alloc(ctx_, (size_t)C_ * 2 * n);
        h_slabs_[0] = slabs_[0].p;
        start_vectors<VT><<<dim3(grid_rows(2LL * n), C_), 256, 0, st_>>>(n, d_act_.p, nrm_.p, d_B_, slabs_[0].p,
                                                                      gv_.p, hstride_);
        ctx_->launches++;
        act_.clear();
        for (int c = 0; c < C_; ++c) {
            if (!std::isfinite(bnorm[c])) {
                res_.status[c] = PLX_ERR_NAN;
            } else if (bnorm[c] > 0.0) {
                act_.push_back(c);
            }
        }
        upload_active();
        resid_.assign(C_, 0.0);
        j_ = 0;
    }

    bool wants_product() const override { return C_ > 0 && j_ < m_ && !act_.empty(); }

    // w = A v_j for every active column: the batch the caller multiplies
    OpInput pre() override {
        const int n = g_->n_var;
        const int na = (int)act_.size();
        gather_cols<VT><<<dim3(grid_rows(2LL * n), na), 256, 0, st_>>>(n, d_act_.p, h_slabs_[j_], Xa_.p);
        ctx_->launches++;
        if (jac_) {
            scale_cols<<<dim3(grid_rows(n), na), 256, 0, st_>>>(n, d_act_.p, Pinv_.p, Xa_.p, 0);
            ctx_->launches++;
        }
        return OpInput{g_, OpBatch{na, d_freq_act_.p}, Xa_.p, Wa_.p, work_.p, rq_.contraction};
    }

    // the Arnoldi step on W, the least-squares update and the convergence test
    void post() override {
        const int n = g_->n_var;
        const int j = j_;
        const int na = (int)act_.size();
        hcols_[j].alloc(ctx_, (size_t)C_ * hstride_);
        h_hcols_[j] = hcols_[j].p;
        slabs_[j + 1].alloc(ctx_, (size_t)C_ * 2 * n);
        h_slabs_[j + 1] = slabs_[j + 1].p;
        PLX_CHECK_CUDA(cudaMemcpyAsync(d_slabs_.p + j + 1, &h_slabs_[j + 1], sizeof(VT *), cudaMemcpyHostToDevice, st_));
        if (j == 0)
            PLX_CHECK_CUDA(cudaMemcpyAsync(d_slabs_.p, &h_slabs_[0], sizeof(VT *), cudaMemcpyHostToDevice, st_));
        PLX_CHECK_CUDA(cudaMemcpyAsync(d_hcols_.p + j, &h_hcols_[j], sizeof(double2 *), cudaMemcpyHostToDevice, st_));
        PLX_CHECK_CUDA(cudaMemsetAsync(hcols_[j].p, 0, (size_t)C_ * hstride_ * 16, st_));
        size_t need = (size_t)na * ndot_ * (j + 1);
        if (part_.n < need) part_.alloc(ctx_, std::max(need, part_.n * 2));
        auto project = [&](int i0, int i1, int accumulate) {
            int ni = i1 - i0;
            if (ni >= 8)
                dots_wide<VT><<<dim3(ndot_, na), kThreads, 0, st_>>>(n, i0, i1, d_act_.p, d_slabs_.p, Wa_.p, part_.p);
            else
                dots_partial<VT><<<dim3(ndot_, na), kThreads, 0, st_>>>(n, i0, i1, d_act_.p, d_slabs_.p, Wa_.p,
                                                                        part_.p);
            dots_finish<<<dim3(n_blocks(ni, 128), na), 128, 0, st_>>>(ndot_, ni, i0, d_act_.p, part_.p, hbuf_.p,
                                                                       hcols_[j].p, hstride_, accumulate);
            ctx_->launches += 2 + combine_chunked(st_, n, i0, ni, na, d_act_.p, d_slabs_.p, hbuf_.p, -1.0, Wa_.p, 0);
        };
        prof_begin(ctx_);
        if (j + 1 < 25 && !rq_.inner) {
            for (int i = 0; i <= j; ++i) project(i, i + 1, 0);        // modified Gram-Schmidt
        } else {
            project(0, j + 1, 0);                                     // classical GS ...
            if (!rq_.single_pass) project(0, j + 1, 1);               // ... and re-orthogonalise
        }
        batch_norms(g_, na, Wa_.p, nrm_part_, nrm_);
        prof_end(ctx_, PROF_ORTHO, 0.0, 0.0);
        prof_begin(ctx_);
        normalize<VT><<<dim3(grid_rows(2LL * n), na), 256, 0, st_>>>(n, d_act_.p, nrm_.p, Wa_.p, slabs_[j + 1].p,
                                                                    hcols_[j].p, hstride_, j + 1);
        givens<<<n_blocks(na, 128), 128, 0, st_>>>(na, j, d_act_.p, d_hcols_.p, hstride_, cs_.p, sn_.p, gv_.p,
                                                  hstride_, m_, nrm_.p);
        ctx_->launches += 2;
        prof_end(ctx_, PROF_LSQ, 0.0, 0.0);
        PLX_CHECK_CUDA(cudaGetLastError());
        PLX_CHECK_CUDA(cudaMemcpyAsync(resid_.data(), nrm_.p, na * 8, cudaMemcpyDeviceToHost, st_));
        PLX_CHECK_CUDA(cudaStreamSynchronize(st_));
        // --- convergence test -----------------------------------------------------
        std::vector<int32_t> trig;
        for (int k = 0; k < na; ++k) {
            int c = act_[k];
            res_.steps[c] = j + 1;
            if (rq_.record_trace) res_.trace[(size_t)c * m_ + j] = resid_[k];
            const double tc = rq_.tols.empty() ? rq_.tol : rq_.tols[c];
            if (!std::isfinite(resid_[k])) res_.status[c] = PLX_ERR_NAN;
            else if (resid_[k] < tc || (rq_.inner && j == m_ - 1)) trig.push_back(c);
        }
        std::vector<char> done(C_, 0);
        for (int c : act_)
            if (res_.status[c] == PLX_ERR_NAN) done[c] = 1;
        if (!trig.empty() && rq_.inner) {
            // inner solve of a refinement: take the least-squares solution as is
            const int nt = (int)trig.size();
            PLX_CHECK_CUDA(cudaMemcpyAsync(d_cols_.p, trig.data(), nt * 4, cudaMemcpyHostToDevice, st_));
            tri_solve<<<nt, 32, (j + 1) * sizeof(double2), st_>>>(nt, j, d_cols_.p, d_hcols_.p, hstride_, gv_.p,
                                                                  hstride_, ybuf_.p);
            ctx_->launches += 1 + combine_chunked(st_, n, 0, j + 1, nt, d_cols_.p, d_slabs_.p, ybuf_.p, 1.0, d_X_, 1);
            if (jac_) {
                scale_cols<<<dim3(grid_rows(n), nt), 256, 0, st_>>>(n, d_cols_.p, Pinv_.p, d_X_, 1);
                ctx_->launches++;
            }
            for (int c : trig) done[c] = 1;
            for (int c : trig)
                if (resid_[std::find(act_.begin(), act_.end(), c) - act_.begin()] >=
                    (rq_.tols.empty() ? rq_.tol : rq_.tols[c]))
                    res_.status[c] = PLX_ERR_NOT_CONVERGED;   // inner dimension used up (not an error)
        } else if (!trig.empty()) {
            const int nt = (int)trig.size();
            PLX_CHECK_CUDA(cudaMemcpyAsync(d_cols_.p, trig.data(), nt * 4, cudaMemcpyHostToDevice, st_));
            tri_solve<<<nt, 32, (j + 1) * sizeof(double2), st_>>>(nt, j, d_cols_.p, d_hcols_.p, hstride_, gv_.p,
                                                                  hstride_, ybuf_.p);
            ctx_->launches += combine_chunked(st_, n, 0, j + 1, nt, d_cols_.p, d_slabs_.p, ybuf_.p, 1.0, d_X_, 1);
            gather_x<<<dim3(grid_rows(2LL * n), nt), 256, 0, st_>>>(n, d_cols_.p, d_X_, Xa_.p);
            ctx_->launches += 2;
            std::vector<int32_t> tf(nt);
            for (int t = 0; t < nt; ++t) tf[t] = rq_.freq[trig[t]];
            DevArray<int32_t> d_tf;
            d_tf.alloc(ctx_, nt);
            PLX_CHECK_CUDA(cudaMemcpyAsync(d_tf.p, tf.data(), nt * 4, cudaMemcpyHostToDevice, st_));
            OpBatch tb{nt, d_tf.p};
            apply_operator(g_, tb, Xa_.p, Wa_.p, work_.p,
                           Contraction::FP64 == rq_.contraction || Contraction::FP64_OTF == rq_.contraction
                               ? rq_.contraction
                               : Contraction::FP64);
            residual<<<dim3(grid_rows(2LL * n), nt), 256, 0, st_>>>(n, d_cols_.p, d_B_, Wa_.p);
            ctx_->launches++;
            batch_norms(g_, nt, Wa_.p, nrm_part_, nrm_);
            std::vector<double> tres(nt);
            PLX_CHECK_CUDA(cudaMemcpyAsync(tres.data(), nrm_.p, nt * 8, cudaMemcpyDeviceToHost, st_));
            PLX_CHECK_CUDA(cudaStreamSynchronize(st_));
            for (int t = 0; t < nt; ++t)
                if (tres[t] < rq_.tol) done[trig[t]] = 1;
                else if (!std::isfinite(tres[t])) {
                    res_.status[trig[t]] = PLX_ERR_NAN;
                    done[trig[t]] = 1;
                }
        }
        std::vector<int32_t> keep;
        for (int c : act_)
            if (!done[c]) keep.push_back(c);
        if (keep.size() != act_.size()) {
            act_.swap(keep);
            if (!act_.empty()) upload_active();
        }
        ++j_;
    }

    void end() override {
        for (int c : act_) res_.status[c] = PLX_ERR_NOT_CONVERGED;
        act_.clear();
        PLX_CHECK_CUDA(cudaStreamSynchronize(st_));
    }

  private:
    void upload_active() {
        std::vector<int32_t> fa(act_.size());
        for (size_t k = 0; k < act_.size(); ++k) fa[k] = rq_.freq[act_[k]];
        PLX_CHECK_CUDA(cudaMemcpyAsync(d_act_.p, act_.data(), act_.size() * 4, cudaMemcpyHostToDevice, st_));
        PLX_CHECK_CUDA(cudaMemcpyAsync(d_freq_act_.p, fa.data(), fa.size() * 4, cudaMemcpyHostToDevice, st_));
    }

    plx_geom *g_;
    plx_ctx *ctx_;
    cudaStream_t st_;
    GmresRequest rq_;
    const double *d_B_;
    double *d_X_;
    GmresResult &res_;
    int C_ = 0, m_ = 0, j_ = 0, nchunk_ = 0, ndot_ = 0, hstride_ = 0;
    bool jac_ = false;
    std::vector<int32_t> act_;
    std::vector<double> resid_;
    DevArray<int32_t> d_act_, d_freq_act_, d_cols_;
    DevArray<double> Xa_, Wa_, work_, nrm_part_, nrm_, cs_, Pinv_;
    DevArray<double2> sn_, gv_, hbuf_, part_, ybuf_;
    std::vector<DevArray<VT>> slabs_;
    std::vector<DevArray<double2>> hcols_;
    DevArray<VT *> d_slabs_;
    DevArray<double2 *> d_hcols_;
    std::vector<VT *> h_slabs_;
    std::vector<double2 *> h_hcols_;
};

std::unique_ptr<GmresStepper> make_gmres(plx_geom *g, const GmresRequest &rq, const double *d_B, double *d_X,
                                         GmresResult &res) {
    if (rq.inner && rq.basis_fp32) {
        auto r = std::make_unique<GmresRun<float>>(g, rq, d_B, d_X, res);
        r->begin();
        return r;
    }
    auto r = std::make_unique<GmresRun<double>>(g, rq, d_B, d_X, res);
    r->begin();
    return r;
}

void gmres_batched(plx_geom *g, const GmresRequest &rq, const double *d_B, double *d_X,
                   GmresResult &res) {
    auto run = make_gmres(g, rq, d_B, d_X, res);
    while (run->wants_product()) {
        OpInput in = run->pre();
        apply_operator(in.g, in.b, in.X, in.Y, in.work, in.how);
        run->post();
    }
    run->end();
}

}  // namespace plx
