// Direct solve of the scalar-shift models through one Hessenberg reduction.
//
// For one-type wFQ (construct_dynamic_matrix_wfq, wfq_module.f90:214-254) and
// BEM DPCM (construct_dynamic_matrix_bem, bem_module.f90:881-933) the matrix
// complex_inversion factors at every frequency (algorithm_module.f90:510-541)
// is a real, frequency-independent A0 plus a complex multiple of the identity:
//     wFQ:   A(w) = (K - P) T - z(w) I          (one Drude z for every atom)
//     DPCM:  A(w) = D + z(w) I                  (z = 2 pi (eps_s + eps)/(eps_s - eps))
// so one orthogonal reduction A0 = Q H Q^T (H upper Hessenberg; Householder
// reflectors, backward stable) serves every frequency:
//     A(w) x = b   <=>   (H + s(w) I) y = Q^T b,   x = Q y,
// and each frequency costs O(n^2): Q^T b and Q y by the stored reflectors, and
// (H + s I) y = c by Givens rotations (QR of a Hessenberg matrix, no pivoting
// needed) and back substitution.  One CTA solves one frequency (all its
// right-hand sides), so a whole grid is one launch; the reduction itself is
// n - 2 steps of four short kernels, once per geometry.  The result is the
// solution of the same linear system as the reference's zgetrf/zgetrs, to
// rounding (both factorisations are backward stable).
#include <algorithm>
#include <cmath>

#include "plx_internal.h"

namespace plx {

namespace {

constexpr int kT = 256;

__device__ __forceinline__ double block_sum(double v, double *red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) red[w] = v;
    __syncthreads();
    double t = 0.0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t += red[k];
    return t;
}

__device__ __forceinline__ double2 block_sum2(double2 v, double *red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
        v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
    }
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) {
        red[2 * w] = v.x;
        red[2 * w + 1] = v.y;
    }
    __syncthreads();
    double2 t = make_double2(0.0, 0.0);
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) {
        t.x += red[2 * k];
        t.y += red[2 * k + 1];
    }
    return t;
}

// A0 of one-type wFQ, column-major: A0(r, c) = sum_e K_e (T[j_e][c] - T[r][c])
// (update_y_q of matrix_module.f90:1011-1098 applied to the columns of T).
__global__ void wfq_a0(int N, const int32_t *__restrict__ rowptr, const int32_t *__restrict__ col,
                       const double *__restrict__ kval, const double *__restrict__ T, double *__restrict__ A) {
    const int c = blockIdx.y;
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= N) return;
    // T symmetric: T[j][c] = T[c][j], read along the column c contiguously
    const double trc = T[(int64_t)c * N + r];
    double a = 0.0;
    for (int e = rowptr[r]; e < rowptr[r + 1]; ++e) a += kval[e] * (T[(int64_t)c * N + col[e]] - trc);
    A[(int64_t)c * N + r] = a;
}

// Householder vector of column k: v (rows k+1..n-1) into V[:, k], beta = 2 / v^T v,
// A[k+1, k] = alpha, A[k+2.., k] = 0.  One block.
__global__ void hh_vector(int n, int k, double *__restrict__ A, double *__restrict__ V, double *__restrict__ beta) {
    __shared__ double red[64];
    double *a = A + (int64_t)k * n;
    const double x0 = a[k + 1];          // read before any thread writes the column
    double s = 0.0;
    for (int i = k + 2 + threadIdx.x; i < n; i += blockDim.x) s += a[i] * a[i];
    const double tail = block_sum(s, red);
    const double nrm = sqrt(x0 * x0 + tail);
    double *v = V + (int64_t)k * n;
    if (nrm == 0.0 || tail == 0.0) {
        // nothing to eliminate: identity reflector
        for (int i = k + 1 + threadIdx.x; i < n; i += blockDim.x) v[i] = 0.0;
        if (threadIdx.x == 0) beta[k] = 0.0;
        return;
    }
    const double alpha = x0 >= 0.0 ? -nrm : nrm;
    const double v0 = x0 - alpha;
    for (int i = k + 1 + threadIdx.x; i < n; i += blockDim.x) {
        v[i] = i == k + 1 ? v0 : a[i];
        a[i] = i == k + 1 ? alpha : 0.0;
    }
    if (threadIdx.x == 0) beta[k] = 2.0 / (v0 * v0 + tail);
}

// Left: A[k+1.., j] -= beta v (v^T A[k+1.., j]) for every column j > k (one block per column).
__global__ void hh_left(int n, int k, double *__restrict__ A, const double *__restrict__ V,
                        const double *__restrict__ beta) {
    __shared__ double red[64];
    const double b = beta[k];
    if (b == 0.0) return;
    const int j = k + 1 + blockIdx.x;
    double *a = A + (int64_t)j * n;
    const double *v = V + (int64_t)k * n;
    double s = 0.0;
    for (int i = k + 1 + threadIdx.x; i < n; i += blockDim.x) s += v[i] * a[i];
    const double w = b * block_sum(s, red);
    for (int i = k + 1 + threadIdx.x; i < n; i += blockDim.x) a[i] -= w * v[i];
}

// Right, first half: u = A[:, k+1..] v (one thread per row).
__global__ void hh_right_u(int n, int k, const double *__restrict__ A, const double *__restrict__ V,
                           const double *__restrict__ beta, double *__restrict__ u) {
    if (beta[k] == 0.0) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double *v = V + (int64_t)k * n;
    double s = 0.0;
    for (int j = k + 1; j < n; ++j) s += A[(int64_t)j * n + i] * v[j];
    u[i] = s;
}

// Right, second half: A[:, j] -= beta v_j u for every column j > k.
__global__ void hh_right_update(int n, int k, double *__restrict__ A, const double *__restrict__ V,
                                const double *__restrict__ beta, const double *__restrict__ u) {
    const double b = beta[k];
    if (b == 0.0) return;
    const int j = k + 1 + blockIdx.y;
    const double f = b * V[(int64_t)k * n + j];
    double *a = A + (int64_t)j * n;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) a[i] -= f * u[i];
}

// H row-major (the rows the Givens sweep reads), upper Hessenberg part.
__global__ void hess_rows(int n, const double *__restrict__ A, double *__restrict__ Hr) {
    const int r = blockIdx.y;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x)
        Hr[(int64_t)r * n + c] = c >= r - 1 ? A[(int64_t)c * n + r] : 0.0;
}

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }

// One frequency per block: for each of its `cols` right-hand sides (split
// complex [2][n] in B, columns col0.. of the batch) solve (H + s I) y = Q^T b and
// write x = Q y into X.  R (the triangular factor, rows packed, n (n + 1) / 2
// complex) lives in this block's slice of Rbuf; carry, y and x in shared memory
// (dynamic: (1 + cols) n complex).
__global__ void __launch_bounds__(kT) hess_solve(int n, int cols, const int32_t *__restrict__ freq_of_block,
                                                 const Cplx *__restrict__ shift, const double *__restrict__ Hr,
                                                 const double *__restrict__ V, const double *__restrict__ beta,
                                                 const double *__restrict__ B, double *__restrict__ X,
                                                 double2 *__restrict__ Rbuf, int *__restrict__ singular) {
    extern __shared__ double2 sh[];
    __shared__ double red[64];
    __shared__ double2 rot[2];          // c (real in .x), s
    const int blk = blockIdx.x;
    const Cplx sv = shift[freq_of_block[blk]];
    const double2 s = make_double2(sv.re, sv.im);
    double2 *carry = sh;                // n
    double2 *y = sh + n;                // cols x n
    double2 *R = Rbuf + (int64_t)blk * ((int64_t)n * (n + 1) / 2);
    // load the right-hand sides
    for (int c = 0; c < cols; ++c) {
        const double *b = B + ((int64_t)blk * cols + c) * 2 * n;
        for (int i = threadIdx.x; i < n; i += blockDim.x) y[(int64_t)c * n + i] = make_double2(b[i], b[n + i]);
    }
    __syncthreads();
    // y = Q^T b: reflectors k = 0 .. n-3 in order
    for (int k = 0; k + 2 < n; ++k) {
        const double bk = beta[k];
        if (bk == 0.0) continue;
        const double *v = V + (int64_t)k * n;
        for (int c = 0; c < cols; ++c) {
            double2 *yc = y + (int64_t)c * n;
            double2 p = make_double2(0.0, 0.0);
            for (int i = k + 1 + threadIdx.x; i < n; i += blockDim.x) {
                p.x += v[i] * yc[i].x;
                p.y += v[i] * yc[i].y;
            }
            p = block_sum2(p, red);
            for (int i = k + 1 + threadIdx.x; i < n; i += blockDim.x) {
                yc[i].x -= bk * p.x * v[i];
                yc[i].y -= bk * p.y * v[i];
            }
            __syncthreads();
        }
    }
    // Givens QR of (H + s I): carry row 0, then rotate it against rows 1..n-1
    for (int j = threadIdx.x; j < n; j += blockDim.x)
        carry[j] = make_double2(Hr[j] + (j == 0 ? s.x : 0.0), j == 0 ? s.y : 0.0);
    __syncthreads();
    int64_t roff = 0;                   // offset of packed row k of R
    for (int k = 0; k + 1 < n; ++k) {
        const double *h = Hr + (int64_t)(k + 1) * n;   // row k + 1 (columns k.. are its nonzeros)
        if (threadIdx.x == 0) {
            // zrotg on (carry[k], h[k]): c real, sn complex, r = alpha |(a, b)|
            const double2 a = carry[k];
            const double bb = h[k];
            const double aa = hypot(a.x, a.y);
            double2 cs, sn;
            if (aa == 0.0) {
                cs = make_double2(0.0, 0.0);
                sn = make_double2(1.0, 0.0);
            } else {
                const double nr = hypot(aa, bb);
                const double2 al = make_double2(a.x / aa, a.y / aa);
                cs = make_double2(aa / nr, 0.0);
                sn = make_double2(al.x * bb / nr, al.y * bb / nr);     // alpha conj(b) / norm, b real
            }
            rot[0] = cs;
            rot[1] = sn;
        }
        __syncthreads();
        const double c = rot[0].x;
        const double2 sn = rot[1];
        // R row k = c carry + sn next ; new carry = -conj(sn) carry + c next   (columns j >= k)
        for (int j = k + threadIdx.x; j < n; j += blockDim.x) {
            const double2 a = carry[j];
            const double2 nx = make_double2(h[j] + (j == k + 1 ? s.x : 0.0), j == k + 1 ? s.y : 0.0);
            const double2 r = make_double2(c * a.x + (sn.x * nx.x - sn.y * nx.y), c * a.y + (sn.x * nx.y + sn.y * nx.x));
            const double2 sc = cconj(sn);
            R[roff + (j - k)] = r;
            carry[j] = make_double2(c * nx.x - (sc.x * a.x - sc.y * a.y), c * nx.y - (sc.x * a.y + sc.y * a.x));
        }
        // the same rotation on every right-hand side
        if (threadIdx.x < cols) {
            double2 *yc = y + (int64_t)threadIdx.x * n;
            const double2 a = yc[k], b2 = yc[k + 1];
            const double2 sc = cconj(sn);
            yc[k] = make_double2(c * a.x + (sn.x * b2.x - sn.y * b2.y), c * a.y + (sn.x * b2.y + sn.y * b2.x));
            yc[k + 1] = make_double2(c * b2.x - (sc.x * a.x - sc.y * a.y), c * b2.y - (sc.x * a.y + sc.y * a.x));
        }
        __syncthreads();
        roff += n - k;
    }
    if (threadIdx.x == 0) R[roff] = carry[n - 1];
    __syncthreads();
    // back substitution R x = y (rows packed: row i starts at i n - i (i - 1) / 2)
    for (int c = 0; c < cols; ++c) {
        double2 *yc = y + (int64_t)c * n;
        for (int i = n - 1; i >= 0; --i) {
            const int64_t ro = (int64_t)i * n - (int64_t)i * (i - 1) / 2;
            double2 p = make_double2(0.0, 0.0);
            for (int j = i + 1 + threadIdx.x; j < n; j += blockDim.x) {
                const double2 t = cmul(R[ro + (j - i)], yc[j]);
                p.x += t.x;
                p.y += t.y;
            }
            p = block_sum2(p, red);
            if (threadIdx.x == 0) {
                const double2 d = R[ro];
                const double m = d.x * d.x + d.y * d.y;
                if (m == 0.0) atomicExch(singular, 1);
                const double2 num = make_double2(yc[i].x - p.x, yc[i].y - p.y);
                yc[i] = m == 0.0 ? make_double2(0.0, 0.0)
                                 : make_double2((num.x * d.x + num.y * d.y) / m, (num.y * d.x - num.x * d.y) / m);
            }
            __syncthreads();
        }
    }
    // x = Q y: reflectors in reverse order
    for (int k = n - 3; k >= 0; --k) {
        const double bk = beta[k];
        if (bk == 0.0) continue;
        const double *v = V + (int64_t)k * n;
        for (int c = 0; c < cols; ++c) {
            double2 *yc = y + (int64_t)c * n;
            double2 p = make_double2(0.0, 0.0);
            for (int i = k + 1 + threadIdx.x; i < n; i += blockDim.x) {
                p.x += v[i] * yc[i].x;
                p.y += v[i] * yc[i].y;
            }
            p = block_sum2(p, red);
            for (int i = k + 1 + threadIdx.x; i < n; i += blockDim.x) {
                yc[i].x -= bk * p.x * v[i];
                yc[i].y -= bk * p.y * v[i];
            }
            __syncthreads();
        }
    }
    for (int c = 0; c < cols; ++c) {
        double *x = X + ((int64_t)blk * cols + c) * 2 * n;
        const double2 *yc = y + (int64_t)c * n;
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            x[i] = yc[i].x;
            x[n + i] = yc[i].y;
        }
    }
}

}  // namespace

bool hessenberg_applies(const plx_geom *g, int cols) {
    if (!g->has_T || g->n_var < 3) return false;
    // carry row and right-hand sides in one block's shared memory
    if ((size_t)(1 + cols) * g->n_var * sizeof(double2) > 200 * 1024) return false;
    if (g->model == PLX_BEM_DPCM) return true;
    return g->model == PLX_WFQ && g->n_types == 1;
}

// Shift s(w) of every frequency: A(w) = A0 + s(w) I.
static std::vector<Cplx> hessenberg_shifts(const plx_geom *g) {
    std::vector<Cplx> s(g->n_freq);
    for (int f = 0; f < g->n_freq; ++f) {
        if (is_bem(g)) {
            s[f] = g->bem_z[f];
        } else {
            // the charge diagonal -z(w) of the one atom type (upload_frequency_tables)
            const double w = g->omega[f], tau = g->tau[0], dn = g->density[0];
            const double den = 2.0 * dn * tau;
            s[f] = {-(w * (-w * tau) / den), -(w * (-1.0) / den)};
        }
    }
    return s;
}

void build_hessenberg(plx_geom *g) {
    if (g->d_hess_rows.p) return;
    plx_ctx *ctx = g->ctx;
    cudaStream_t st = ctx->stream;
    const int n = g->n_var;
    DevArray<double> A, u;
    A.alloc(ctx, (size_t)n * n);
    u.alloc(ctx, n);
    g->d_hess_v.alloc(ctx, (size_t)n * n);
    g->d_hess_beta.alloc(ctx, std::max(n, 1));
    PLX_CHECK_CUDA(cudaMemsetAsync(g->d_hess_beta.p, 0, (size_t)std::max(n, 1) * 8, st));
    if (is_bem(g)) {
        // D stored transposed (d_T[j][i] = D(i, j)) is D column-major
        PLX_CHECK_CUDA(cudaMemcpyAsync(A.p, g->d_T.p, (size_t)n * n * 8, cudaMemcpyDeviceToDevice, st));
    } else {
        wfq_a0<<<dim3(n_blocks(n, 128), n), 128, 0, st>>>(n, g->d_rowptr.p, g->d_col.p, g->d_kval.p, g->d_T.p, A.p);
        ctx->launches++;
    }
    for (int k = 0; k + 2 < n; ++k) {
        hh_vector<<<1, kT, 0, st>>>(n, k, A.p, g->d_hess_v.p, g->d_hess_beta.p);
        hh_left<<<n - k - 1, kT, 0, st>>>(n, k, A.p, g->d_hess_v.p, g->d_hess_beta.p);
        hh_right_u<<<n_blocks(n, kT), kT, 0, st>>>(n, k, A.p, g->d_hess_v.p, g->d_hess_beta.p, u.p);
        hh_right_update<<<dim3(n_blocks(n, kT), n - k - 1), kT, 0, st>>>(n, k, A.p, g->d_hess_v.p,
                                                                          g->d_hess_beta.p, u.p);
        ctx->launches += 4;
    }
    g->d_hess_rows.alloc(ctx, (size_t)n * n);
    hess_rows<<<dim3(n_blocks(n, kT), n), kT, 0, st>>>(n, A.p, g->d_hess_rows.p);
    ctx->launches++;
    PLX_CHECK_CUDA(cudaGetLastError());
    PLX_CHECK_CUDA(cudaStreamSynchronize(st));
}

// Solves A(w_f) x = b for the frequencies of `freqs` (cols right-hand sides each,
// B and X [freqs.size() * cols][2][n], frequency-major).  Returns false when a
// frequency's triangular factor has a zero on its diagonal (singular A(w)).
bool hessenberg_solve(plx_geom *g, const std::vector<int32_t> &freqs, int cols, const double *B, double *X) {
    build_hessenberg(g);
    plx_ctx *ctx = g->ctx;
    cudaStream_t st = ctx->stream;
    const int n = g->n_var;
    const int F = (int)freqs.size();
    if (F == 0) return true;
    const std::vector<Cplx> shifts = hessenberg_shifts(g);
    DevArray<Cplx> d_shift;
    d_shift.alloc(ctx, shifts.size());
    PLX_CHECK_CUDA(cudaMemcpyAsync(d_shift.p, shifts.data(), shifts.size() * sizeof(Cplx), cudaMemcpyHostToDevice, st));
    const size_t smem = (size_t)(1 + cols) * n * sizeof(double2);
    if (smem > 200 * 1024) throw Error(PLX_ERR_UNSUPPORTED, "order too large for the shifted Hessenberg solve");
    once_per_device(reinterpret_cast<const void *>(hess_solve), ctx->device, [] {
        PLX_CHECK_CUDA(cudaFuncSetAttribute(hess_solve, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    });
    // waves of frequencies whose triangular factors fit a quarter of the budget
    const size_t rbytes = (size_t)n * (n + 1) / 2 * sizeof(double2);
    const uint64_t avail = ctx->budget > ctx->in_use ? ctx->budget - ctx->in_use : 0;
    const int wave = (int)std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)F, avail / 4 / rbytes));
    DevArray<double2> R;
    DevArray<int32_t> d_f;
    DevArray<int> sing;
    R.alloc(ctx, (size_t)wave * n * (n + 1) / 2);
    d_f.alloc(ctx, F);
    sing.alloc(ctx, 1);
    PLX_CHECK_CUDA(cudaMemcpyAsync(d_f.p, freqs.data(), F * 4, cudaMemcpyHostToDevice, st));
    PLX_CHECK_CUDA(cudaMemsetAsync(sing.p, 0, sizeof(int), st));
    for (int f0 = 0; f0 < F; f0 += wave) {
        const int nf = std::min(wave, F - f0);
        const size_t off = (size_t)f0 * cols * 2 * n;
        hess_solve<<<nf, kT, smem, st>>>(n, cols, d_f.p + f0, d_shift.p, g->d_hess_rows.p, g->d_hess_v.p,
                                        g->d_hess_beta.p, B + off, X + off, R.p, sing.p);
        ctx->launches++;
        PLX_CHECK_CUDA(cudaGetLastError());
    }
    int hs = 0;
    PLX_CHECK_CUDA(cudaMemcpyAsync(&hs, sing.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    PLX_CHECK_CUDA(cudaStreamSynchronize(st));
    return hs == 0;
}

}  // namespace plx
