// Few-column FP64 contraction S^T = X^T T (R <= 16 real columns): T is
// streamed once, split over K into chunks whose partial sums are reduced in a
// fixed order.  Shared by the operator (operator.cu) and the no-allocation
// entry point (noalloc.cu).
#pragma once

#include <algorithm>
#include <cstdint>

namespace plx {
namespace {

constexpr int kSkinnyCols = 256;
constexpr int kSkinnyK = 32;

template <int R>
__global__ void __launch_bounds__(kSkinnyCols) skinny_partial(int n, int kchunk,
                                                              const double *__restrict__ Xt,
                                                              const double *__restrict__ T,
                                                              double *__restrict__ part) {
    __shared__ double xs[kSkinnyK][R];
    int col = blockIdx.x * kSkinnyCols + threadIdx.x;
    int k0 = blockIdx.y * kchunk;
    int k1 = min(n, k0 + kchunk);
    double acc[R];
#pragma unroll
    for (int r = 0; r < R; ++r) acc[r] = 0.0;
    for (int kb = k0; kb < k1; kb += kSkinnyK) {
        int kn = min(kSkinnyK, k1 - kb);
        __syncthreads();
        for (int e = threadIdx.x; e < kSkinnyK * R; e += kSkinnyCols) {
            int r = e / kSkinnyK, kk = e % kSkinnyK;
            xs[kk][r] = (kk < kn) ? Xt[(int64_t)r * n + kb + kk] : 0.0;
        }
        __syncthreads();
        if (col < n) {
            const double *Tp = T + (int64_t)kb * n + col;
            for (int kk = 0; kk < kn; ++kk) {
                double t = __ldg(Tp + (int64_t)kk * n);
#pragma unroll
                for (int r = 0; r < R; ++r) acc[r] = fma(xs[kk][r], t, acc[r]);
            }
        }
    }
    if (col < n) {
#pragma unroll
        for (int r = 0; r < R; ++r) part[((int64_t)blockIdx.y * R + r) * n + col] = acc[r];
    }
}

__global__ void skinny_reduce(int n, int R, int ks, const double *__restrict__ part,
                              double *__restrict__ S) {
    int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (int64_t)R * n) return;
    double s = 0.0;
    for (int k = 0; k < ks; ++k) s += part[(int64_t)k * R * n + idx];
    S[idx] = s;
}

// Number of K chunks and their length for a contraction of order n; depends on
// n only, so that a column's sums do not depend on the batch it is part of.
inline void skinny_split(int n, int &ks, int &kchunk) {
    const int cb = (n + kSkinnyCols - 1) / kSkinnyCols;
    ks = std::max(1, std::min(64, (592 + cb - 1) / cb));
    kchunk = (n + ks - 1) / ks;
    ks = (n + kchunk - 1) / kchunk;
}

}  // namespace
}  // namespace plx
