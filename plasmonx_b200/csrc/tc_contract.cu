// Tensor-core T contraction for the mixed-precision solve (sm_100a, tcgen05).
//
// S = T X for a batch of R real columns, with T (n x n, symmetric) and X split
// into BF16 high and low parts, T = Th + Tl, X = Xh + Xl, and
//     S = Th Xh + Th Xl + Tl Xh        (FP32 accumulation in tensor memory),
// i.e. every product carries ~16 significant bits of each operand; the dropped
// Tl Xl term is below 2^-16 of the result.  The result is written as FP64 so the
// rest of the operator (conductance rows, frequency diagonal) stays unchanged.
//
// GEMM mapping (all operands K-major, the layout tcgen05 reads natively):
//   A = T   rows m of T, contiguous along k         (M = n_var)
//   B = X^T column c of X, contiguous along k        (N = R real columns)
//   D = TMEM accumulators 128 x BN (FP32), lane = row m, column = c
// One CTA computes a 256 x BN tile of S as two 128-row accumulators (TMEM
// columns [0, BN) and [BN, 2 BN)) that share every B tile, which halves the
// B traffic from L2 per row of T; 4 warps: thread 0 issues the TMA
// loads, thread 32 issues the MMAs, all 128 threads drain TMEM in the
// epilogue.  Operand tiles are 32 elements (64 bytes) deep along k and are
// loaded by TMA with the 64-byte swizzle that the UMMA descriptors describe;
// the small stages allow 4-6 of them in flight.
// Every wait on an mbarrier is bounded.  The pipeline waits use the context's
// limit (plx_set_wait_limit); a CTA whose wait runs out records an error code
// and gives up, in this order: the MMA issuer still commits `done`, which
// arrives only when every MMA it has issued has finished; all threads wait for
// it, so no MMA reads shared memory or writes tensor memory after that point;
// the producer then waits for the loads it has issued to land, so no copy
// writes into shared memory after the CTA exits; then the tensor memory is
// freed and the CTA returns without storing a result.  These clean-up waits
// use their own, long limit (kDrainLimit), never the pipeline limit.  If one of
// them runs out as well (a copy or an MMA that never completes: the hardware
// has stopped answering) the CTA records that error too and exits anyway; the
// call then fails and nothing it wrote is used.
#include <cuda.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <cstring>

#include "pair_tiles.cuh"
#include "plx_internal.h"

namespace plx {

namespace {

constexpr int kUM = 128;          // rows per tcgen05.mma (TMEM lanes)
constexpr int kBM = 2 * kUM;      // rows of T per CTA: two accumulators share every B tile
constexpr int kBK = 32;           // k per stage (64 bytes of BF16: the 64-byte swizzle atom)
constexpr int kLdAlign = 64;      // k padding of the split operands (zeros)
constexpr int kUmmaK = 16;        // k per tcgen05.mma (kind::f16)
constexpr uint32_t kDrainLimit = 1u << 22;  // clean-up waits after an abort (seconds at most)
constexpr int kSmemBudget = 227 * 1024 - 1024 - 256;   // pipeline stages (after alignment and barriers)

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait: returns false when `limit` polls pass, or early when another
// thread of the CTA has raised `abort`; records `code` in *err on failure.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, uint32_t limit, volatile int *abort,
                                          int *err, int code) {
    for (uint32_t it = 0; it < limit; ++it) {
        if (mbar_try_wait(bar, parity)) return true;
        if (abort && (it & 255u) == 255u && *abort) return false;
    }
    if (err) atomicCAS(err, 0, code);
    return false;
}

// Plain bulk copy of `bytes` contiguous bytes into shared memory (addresses
// 16-byte aligned, size a multiple of 16), completing on `bar`.
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(src)), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void tma_load_2d(const CUtensorMap *map, uint64_t *bar, void *dst, int x, int y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
            smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

// UMMA shared-memory descriptor, K-major operand with the 64-byte swizzle:
// 8-row x 64-byte swizzle atoms stacked every 512 bytes (stride byte offset),
// leading byte offset 16 bytes (unused for this layout), descriptor version 1,
// layout type 4 (64-byte swizzle) in bits [61,64).
__device__ __forceinline__ uint64_t umma_desc_sw64(const void *smem) {
    uint64_t addr = smem_u32(smem);
    uint64_t d = 0;
    d |= (addr >> 4) & 0x3FFFull;           // start address, bits [0,14)
    d |= (uint64_t)(16 >> 4) << 16;         // leading byte offset, bits [16,30)
    d |= (uint64_t)(512 >> 4) << 32;        // stride byte offset, bits [32,46)
    d |= (uint64_t)1 << 46;                 // version, bits [46,48)
    d |= (uint64_t)4 << 61;                 // layout: 64-byte swizzle
    return d;
}

// Instruction descriptor, kind::f16: BF16 x BF16 -> FP32, both K-major.
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int M, int N) {
    return (1u << 4)                        // D format F32
           | (1u << 7)                      // A format BF16
           | (1u << 10)                     // B format BF16
           | ((uint32_t)(N >> 3) << 17)     // N / 8
           | ((uint32_t)(M >> 4) << 24);    // M / 16
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ void umma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_u32(bar))
                 : "memory");
}

// Work of one launch: the output tiles (256 rows x bn columns, column tile
// fastest so that the tiles sharing one row block of an operand run side by
// side and its second read comes from L2) of one or several groups -- a group
// is one contraction S = A X of one geometry.  A group's first `full` tiles are
// computed whole, one CTA each, and stored as FP64 into S; each of its
// remaining tiles is split over k into q pieces of kper k-tiles, one CTA each,
// which store FP32 partial sums into P (piece j at P + j * 256 * bn,
// [column][row]); reduce_pieces adds a tile's pieces in order.  With the
// pieces filling the last wave, every SM gets the same work (whole tiles plus
// one piece) instead of a last wave that leaves SMs idle.  Several groups in one
// launch run whole tiles only, the groups ordered by decreasing k length, so
// that the hardware's in-order dispatch of CTAs to free SMs balances them.
constexpr int kMaxGroups = 6;
struct TcGroup {
    int M, R, bn, ktiles;       // rows, real columns, column tile, k-tiles (32 deep)
    int unit0;                  // first CTA of the group
    int full, q, kper, ctiles;  // schedule (see above)
    const uint8_t *ah, *al;     // A high / low, tile-ordered and pre-swizzled (16 KB per stage tile)
    double *S;                  // [R][M] FP64
    float *P;                   // pieces of the split tiles
    int *err;                   // the geometry's error word (first bounded wait that ran out)
};
struct TcLaunch {
    CUtensorMap map[kMaxGroups][4];   // [2], [3]: X high, X low ([0], [1] unused: A goes by bulk copy)
    TcGroup grp[kMaxGroups];
    int ngroups;
    int stages;                 // pipeline depth
    int bn_max;                 // shared-memory / tensor-memory sizing
    uint32_t wait_limit;
};

// Bytes of one pipeline stage: the A and X tiles its products read -- high and
// low parts for three products, the high parts alone for one (whose stages are
// then half as large and twice as many fit).
__host__ __device__ constexpr int tc_stage_bytes(int bn, int nprod) {
    return (nprod > 1 ? 2 : 1) * (kBM * kBK * 2 + bn * kBK * 2);
}

template <int NPROD>
__global__ void __launch_bounds__(128, 1) tc_contract_kernel(const __grid_constant__ TcLaunch p) {
    // this CTA's group and unit: a whole tile, or one k-piece of a remaining tile
    int gi = 0;
    while (gi + 1 < p.ngroups && (int)blockIdx.x >= p.grp[gi + 1].unit0) ++gi;
    const TcGroup &G = p.grp[gi];
    const int u = (int)blockIdx.x - G.unit0;
    int tile, kt0, nk, piece = -1;
    if (u < G.full) {
        tile = u;
        kt0 = 0;
        nk = G.ktiles;
    } else {
        piece = u - G.full;
        tile = G.full + piece / G.q;
        kt0 = (piece % G.q) * G.kper;
        nk = min(G.ktiles, kt0 + G.kper) - kt0;
    }
    const int bn = G.bn, M = G.M, R = G.R, ktiles = G.ktiles;
    const int bnp = (bn + 31) & ~31;     // TMEM columns of one accumulator (32-aligned)
    const int STAGES = p.stages;
    const int kStage = tc_stage_bytes(p.bn_max, NPROD);
    const int kA = kBM * kBK * 2;
    const int mtile = tile / G.ctiles;
    int *err = G.err;
    const uint32_t wait_limit = p.wait_limit;
    // two accumulators of bn columns each (rows m0.. and m0 + 128..), at TMEM
    // columns 0 and bnp; bn_max is a multiple of 32
    const uint32_t tmem_cols = 2 * p.bn_max <= 64 ? 64 : (2 * p.bn_max <= 128 ? 128 : (2 * p.bn_max <= 256 ? 256 : 512));
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t *base = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint64_t *full = reinterpret_cast<uint64_t *>(base + STAGES * kStage);
    uint64_t *empty = full + STAGES;
    uint64_t *done = empty + STAGES;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(done + 1);
    volatile int *abort_flag = reinterpret_cast<volatile int *>(tmem_slot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int n0 = (tile % G.ctiles) * bn;
    const int m0 = mtile * kBM;

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(done, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(tmem_cols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;

    auto stage_ptr = [&](int s, int which) -> uint8_t * {
        // which: 0 A high, 1 A low, 2 X high, 3 X low (the low parts only for NPROD > 1)
        constexpr int parts = NPROD > 1 ? 2 : 1;
        uint8_t *st = base + s * kStage;
        return which < 2 ? st + which * kA : st + parts * kA + (which - 2) * (p.bn_max * kBK * 2);
    };

    int issued = 0;     // loads issued by the producer (thread 0)
    if (threadIdx.x == 0) {
        // ---------------- TMA producer ----------------
        const CUtensorMap *mp = p.map[gi];
        // one product (NPROD = 1) reads only the high parts: half the operand bytes
        const uint32_t tx = (uint32_t)(NPROD > 1 ? 2 * kA + 2 * bn * kBK * 2 : kA + bn * kBK * 2);
        for (int kt = 0; kt < nk; ++kt) {
            const int s = kt % STAGES;
            if (kt >= STAGES) {
                if (!mbar_wait(&empty[s], ((kt / STAGES) - 1) & 1, wait_limit, abort_flag, err, 1) || *abort_flag) {
                    *abort_flag = 1;
                    break;
                }
            }
            mbar_expect_tx(&full[s], tx);
            const int kx = (kt0 + kt) * kBK;
            const size_t aoff = (size_t)(mtile * ktiles + kt0 + kt) * kA;   // tile-ordered A
            bulk_load(stage_ptr(s, 0), G.ah + aoff, kA, &full[s]);
            if (NPROD > 1) bulk_load(stage_ptr(s, 1), G.al + aoff, kA, &full[s]);
            tma_load_2d(&mp[2], &full[s], stage_ptr(s, 2), kx, n0);
            if (NPROD > 1) tma_load_2d(&mp[3], &full[s], stage_ptr(s, 3), kx, n0);
            issued = kt + 1;
        }
    } else if (threadIdx.x == 32) {
        // ---------------- MMA issuer ----------------
        const uint32_t idesc = umma_idesc_bf16(kUM, bn);
        constexpr uint64_t kHalf = (uint64_t)(kUM * kBK * 2) >> 4;   // second 128 rows of an A tile
        for (int kt = 0; kt < nk; ++kt) {
            const int s = kt % STAGES;
            if (!mbar_wait(&full[s], (kt / STAGES) & 1, wait_limit, abort_flag, err, 2) || *abort_flag) {
                *abort_flag = 1;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint64_t dTh = umma_desc_sw64(stage_ptr(s, 0));
            const uint64_t dTl = umma_desc_sw64(stage_ptr(s, 1));
            const uint64_t dXh = umma_desc_sw64(stage_ptr(s, 2));
            const uint64_t dXl = umma_desc_sw64(stage_ptr(s, 3));
#pragma unroll
            for (int kk = 0; kk < kBK / kUmmaK; ++kk) {
                // advance 16 elements = 32 bytes = 2 descriptor units along k
                const uint64_t off = (uint64_t)(kk * kUmmaK * 2) >> 4;
                const uint32_t acc0 = (kt > 0 || kk > 0) ? 1u : 0u;
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const uint32_t td = tmem + (uint32_t)(h * bnp);
                    const uint64_t ho = h * kHalf;
                    umma_bf16(td, dTh + ho + off, dXh + off, idesc, acc0);
                    if (NPROD > 1) {
                        umma_bf16(td, dTh + ho + off, dXl + off, idesc, 1u);
                        umma_bf16(td, dTl + ho + off, dXh + off, idesc, 1u);
                    }
                }
            }
            umma_commit(&empty[s]);
        }
        // always: arrives once every MMA issued above has completed (also after
        // an abort, so that nothing below frees memory an MMA still uses)
        umma_commit(done);
    }
    __syncwarp();

    // ---------------- epilogue: TMEM -> S (FP64) or the piece's partial (FP32) ----------------
    bool fin = mbar_wait(done, 0, wait_limit, nullptr, err, 3);
    if (!fin) {
        *abort_flag = 1;
        fin = mbar_wait(done, 0, kDrainLimit, nullptr, err, 4);
    }
    // uniform over the CTA; a thread that raised the flag counts it itself
    const bool have = !__syncthreads_or(*abort_flag != 0 || !fin);
    if (!have && threadIdx.x == 0) {
        // let the loads already issued land before the CTA can exit: the last
        // phase of each stage (earlier phases completed before it was re-armed)
        for (int kt = issued > STAGES ? issued - STAGES : 0; kt < issued; ++kt)
            mbar_wait(&full[kt % STAGES], (kt / STAGES) & 1, kDrainLimit, nullptr, err, 5);
    }
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (have) {
#pragma unroll 1
      for (int h = 0; h < 2; ++h) {
        const int row = m0 + h * kUM + warp * 32 + lane;
#pragma unroll 1
        for (int c0 = 0; c0 < bn; c0 += 32) {
            uint32_t v[32];
            const int nc = min(32, bn - c0);           // 32, or 16 for the last chunk
            const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(h * bnp + c0);
            if (nc == 32) {
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
                    "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
                    "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
                    : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
                      "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
                      "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]),
                      "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]),
                      "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
                    : "r"(taddr));
            } else {
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
                    "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                    : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
                      "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
                      "=r"(v[14]), "=r"(v[15])
                    : "r"(taddr));
#pragma unroll
                for (int j = 16; j < 32; ++j) v[j] = 0u;
            }
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (piece >= 0) {
                // partial of a split tile: [column][256 rows] FP32, every element written
                float *pp = G.P + (int64_t)piece * kBM * bn + (h * kUM + warp * 32 + lane);
#pragma unroll
                for (int j = 0; j < 32; ++j)
                    if (j < nc) pp[(int64_t)(c0 + j) * kBM] = __uint_as_float(v[j]);
            } else if (row < M) {
#pragma unroll
                for (int j = 0; j < 32; ++j) {
                    const int c = n0 + c0 + j;
                    if (j < nc && c < R) G.S[(int64_t)c * M + row] = (double)__uint_as_float(v[j]);
                }
            }
        }
      }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(tmem_cols) : "memory");
    }
}

// The A operand (T, A0 or D^T split in BF16 high/low) is stored in the order
// the kernel reads it: [m-tile of 256 rows][k-slab of 32][256 rows][32 k], so
// every stage's tile (256 x 32) is one contiguous 16 KB block of HBM, and within
// the tile already in the shared-memory image the UMMA descriptors read: the
// 64-byte swizzle, in which the 16-byte chunk c of row r sits at chunk
// c ^ ((r >> 1) & 3) of its 64-byte row.  A stage's A tile is then one plain
// bulk copy.  Rows beyond n and k beyond n are zero.
__device__ __forceinline__ int64_t a_tile_pos(int64_t rr, int64_t kk) {
    return rr * kBK + ((((kk >> 3) ^ ((rr >> 1) & 3)) << 3) | (kk & 7));
}
__device__ __forceinline__ int64_t a_tiled(int64_t r, int64_t k, int64_t ktiles) {
    return ((r / kBM) * ktiles + k / kBK) * (int64_t)(kBM * kBK) + a_tile_pos(r % kBM, k % kBK);
}

__device__ __forceinline__ void split_store(double a, int64_t idx, __nv_bfloat16 *__restrict__ hi,
                                            __nv_bfloat16 *__restrict__ lo) {
    float x = (float)a;
    __nv_bfloat16 h = __float2bfloat16_rn(x);
    hi[idx] = h;
    lo[idx] = __float2bfloat16_rn(x - __bfloat162float(h));
}

// Row-major n x n FP64 matrix -> tiled BF16 pair; the output is walked in its
// own (contiguous) order.
__global__ void split_tiled(int n, int64_t ktiles, int64_t total, const double *__restrict__ in,
                            __nv_bfloat16 *__restrict__ hi, __nv_bfloat16 *__restrict__ lo) {
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t kk = e % kBK, rr = (e / kBK) % kBM, tk = e / ((int64_t)kBK * kBM);
        const int64_t r = (tk / ktiles) * kBM + rr, k = (tk % ktiles) * kBK + kk;
        const double a = (r < n && k < n) ? in[r * n + k] : 0.0;
        split_store(a, tk * (int64_t)(kBM * kBK) + a_tile_pos(rr, kk), hi, lo);
    }
}

// Transposed (BEM: d_T[j][i] = D(i, j)): out(r, k) = in[k][r], through a
// shared-memory tile of 32 k x 256 r; grid (ktiles, mtiles).
__global__ void split_tiled_t(int n, int64_t ktiles, const double *__restrict__ in, __nv_bfloat16 *__restrict__ hi,
                              __nv_bfloat16 *__restrict__ lo) {
    __shared__ float tile[kBK][kBM + 1];
    const int64_t k0 = (int64_t)blockIdx.x * kBK, r0 = (int64_t)blockIdx.y * kBM;
    for (int e = threadIdx.x; e < kBK * kBM; e += blockDim.x) {
        const int kk = e / kBM, rr = e % kBM;                      // coalesced along r
        const int64_t k = k0 + kk, r = r0 + rr;
        tile[kk][rr] = (k < n && r < n) ? (float)in[k * n + r] : 0.0f;
    }
    __syncthreads();
    const int64_t base = ((int64_t)blockIdx.y * ktiles + blockIdx.x) * kBM * kBK;
    for (int e = threadIdx.x; e < kBK * kBM; e += blockDim.x) {   // contiguous output block
        const int rr = e / kBK, kk = e % kBK;
        float x = tile[kk][rr];
        __nv_bfloat16 h = __float2bfloat16_rn(x);
        hi[base + a_tile_pos(rr, kk)] = h;
        lo[base + a_tile_pos(rr, kk)] = __float2bfloat16_rn(x - __bfloat162float(h));
    }
}

// No stored T (on-the-fly geometries): the split generated from the pair
// formulas, one block per TMA box (256 rows x 32 k, contiguous output).
__global__ void split_tiled_gen(int N, int n, int fmu, int64_t ktiles, const double *__restrict__ pos,
                                const double *__restrict__ par, __nv_bfloat16 *__restrict__ hi,
                                __nv_bfloat16 *__restrict__ lo) {
    const int64_t k0 = (int64_t)blockIdx.x * kBK, r0 = (int64_t)blockIdx.y * kBM;
    const int64_t base = ((int64_t)blockIdx.y * ktiles + blockIdx.x) * kBM * kBK;
    for (int e = threadIdx.x; e < kBK * kBM; e += blockDim.x) {
        const int64_t r = r0 + e / kBK, k = k0 + e % kBK;
        const double a = (r < n && k < n) ? plx_t_element(N, fmu != 0, pos, par, r, k) : 0.0;
        split_store(a, base + a_tile_pos(e / kBK, e % kBK), hi, lo);
    }
}

// Folded operator rows, split like T.  For a charge row i < N
//   A0[i][k] = sum_e c_e (T[j_e][k] - T[i][k])      (CSR order, FP64)
// with c_e = K_ij for one atom type (the charge rows of (K - P) T,
// update_y_q of matrix_module.f90:1011-1098, applied to T itself) and
// c_e = 1/2 (K_ij + K_ji) for alloys (the w-independent part of
// 1/2 (K + (w_j/w_i) K^T)); for a dipole row A0[r][k] = T[r][k]; the rows
// appended after n are the charge rows of T of the interface atoms.  T comes
// from the stored matrix or, without one, from the pair formulas.  One block
// per (row, column chunk); rows vary fastest over the grid, so the blocks
// running together share their neighbours' rows of T in L2.
// T rows [t_row0, ...) held in T (stored matrix: t_row0 = 0; a generated
// window of charge rows otherwise), or generated from the pair formulas.
__device__ __forceinline__ double t_value(const double *__restrict__ T, int64_t t_row0, int N, int n, int fmu,
                                          const double *__restrict__ pos, const double *__restrict__ par, int64_t r,
                                          int64_t k) {
    return T ? T[(r - t_row0) * n + k] : plx_t_element(N, fmu != 0, pos, par, r, k);
}

// Charge rows [a0, a0 + gridDim.x) of T generated into a window buffer.
__global__ void t_rows_gen(int N, int n, int fmu, int64_t a0, const double *__restrict__ pos,
                           const double *__restrict__ par, double *__restrict__ Tw) {
    const int64_t a = a0 + blockIdx.x;
    const int64_t k = (int64_t)blockIdx.y * blockDim.x + threadIdx.x;
    if (k < n) Tw[(int64_t)blockIdx.x * n + k] = plx_t_element(N, fmu != 0, pos, par, a, k);
}

__global__ void fold_split(int N, int n, int64_t ld, int64_t ktiles, int hetero, int fmu, int64_t r_begin,
                           int64_t t_row0,
                           const int32_t *__restrict__ rowptr, const int32_t *__restrict__ col,
                           const double *__restrict__ kval, const double *__restrict__ ktval,
                           const double *__restrict__ T, const double *__restrict__ pos,
                           const double *__restrict__ par, const int32_t *__restrict__ iface_atom,
                           __nv_bfloat16 *__restrict__ hi, __nv_bfloat16 *__restrict__ lo) {
    const int64_t r = r_begin + blockIdx.x;
    const int64_t k = (int64_t)blockIdx.y * blockDim.x + threadIdx.x;
    if (k >= ld) return;
    double a = 0.0;
    if (k < n) {
        if (r < N) {
            const double trk = t_value(T, t_row0, N, n, fmu, pos, par, r, k);
            for (int e = rowptr[r]; e < rowptr[r + 1]; ++e) {
                const double c = hetero ? 0.5 * (kval[e] + ktval[e]) : kval[e];
                a = fma(c, t_value(T, t_row0, N, n, fmu, pos, par, col[e], k) - trk, a);
            }
        } else if (r < n) {
            a = t_value(T, t_row0, N, n, fmu, pos, par, r, k);
        } else {
            a = t_value(T, t_row0, N, n, fmu, pos, par, iface_atom[r - n], k);
        }
    }
    split_store(a, a_tiled(r, k, ktiles), hi, lo);
}

// FP64 -> (BF16 high, BF16 low) split of a row-major [rows][cols] array into a
// zero-padded [rows_pad][ld] pair.
__global__ void split_bf16(int rows, int cols, int64_t ld_in, const double *__restrict__ in, int rows_pad,
                           int64_t ld_out, __nv_bfloat16 *__restrict__ hi, __nv_bfloat16 *__restrict__ lo) {
    int64_t total = (int64_t)rows_pad * ld_out;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
        int64_t r = e / ld_out, c = e % ld_out;
        float x = (r < rows && c < cols) ? (float)in[r * ld_in + c] : 0.0f;
        __nv_bfloat16 h = __float2bfloat16_rn(x);
        hi[e] = h;
        lo[e] = __float2bfloat16_rn(x - __bfloat162float(h));
    }
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
    // initialised once, thread-safely (function-local static)
    static const EncodeTiledFn fn = [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        PLX_CHECK_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
        if (!p || q != cudaDriverEntryPointSuccess) throw Error(PLX_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
        return reinterpret_cast<EncodeTiledFn>(p);
    }();
    return fn;
}

// 2-D BF16 tensor [outer][inner] with leading dimension ld (elements), boxes of
// (kBK inner x box_outer), 64-byte swizzle, zero fill out of bounds.
CUtensorMap make_map(const void *ptr, uint64_t inner, uint64_t outer, uint64_t ld, uint32_t box_outer) {
    CUtensorMap m;
    cuuint64_t dims[2] = {inner, outer};
    cuuint64_t strides[1] = {ld * 2};
    cuuint32_t box[2] = {(cuuint32_t)kBK, box_outer};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = encode_fn()(&m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void *>(ptr), dims, strides, box, estr,
                             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B,
                             CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) throw Error(PLX_ERR_CUDA, "cuTensorMapEncodeTiled failed: " + std::to_string((int)r));
    return m;
}

// Remaining tiles of a group: S = the sum of a tile's q FP32 pieces in piece
// order (FP64 sums), for the rows and columns inside the matrix.  One block per
// (tile, 32-column group); threads over the tile's 256 rows.
__global__ void reduce_pieces(int M, int R, int bn, int full, int ctiles, int q, const float *__restrict__ P,
                              double *__restrict__ S) {
    const int t = blockIdx.x;                       // remaining tile index
    const int tile = full + t;
    const int m0 = (tile / ctiles) * kBM, n0 = (tile % ctiles) * bn;
    const int r = threadIdx.x;                      // 0..255
    if (m0 + r >= M) return;
    for (int c = blockIdx.y * 32; c < min(bn, blockIdx.y * 32 + 32); ++c) {
        if (n0 + c >= R) break;
        double a = 0.0;
        for (int p = 0; p < q; ++p) a += (double)P[((int64_t)(t * q + p) * bn + c) * kBM + r];
        S[(int64_t)(n0 + c) * M + m0 + r] = a;
    }
}

int sm_count(int device) {
    int v = 0;
    PLX_CHECK_CUDA(cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, device));
    return v > 0 ? v : 1;
}

// Schedule of one group's `tiles` output tiles of `ktiles` k-tiles on `sms` SMs
// (one CTA per SM): whole tiles in full waves; the r = tiles mod sms tiles of
// the last wave are split into q = sms / r pieces (at least 8 k-tiles each)
// when that lets the pieces fill the wave -- otherwise (r close to sms, or no
// split possible) they run whole too.  Returns the group's number of CTAs.
int make_schedule(TcGroup &gp, int tiles, int sms, bool split) {
    gp.full = tiles;
    gp.q = 1;
    gp.kper = gp.ktiles;
    const int r = tiles % sms;
    if (!split || r == 0 || (double)r / sms >= 0.9) return tiles;
    int q = std::min(sms / r, gp.ktiles / 8);
    if (q < 2) return tiles;
    const int kper = (gp.ktiles + q - 1) / q;
    q = (gp.ktiles + kper - 1) / kper;              // no empty piece
    gp.full = tiles - r;
    gp.q = q;
    gp.kper = kper;
    return gp.full + r * q;
}

}  // namespace


void build_t_split(plx_geom *g) {
    if (g->d_Th.p) return;
    if (!g->has_T && is_bem(g)) throw Error(PLX_ERR_ARG, "BEM geometry without its Green-function matrix");
    const int64_t n = g->n_var;
    const int64_t ld = (n + kLdAlign - 1) / kLdAlign * kLdAlign;
    const int64_t rows = (n + kBM - 1) / kBM * kBM, ktiles = ld / kBK;
    g->ldk = ld;
    g->d_Th.alloc(g->ctx, (size_t)(rows * ld));
    g->d_Tl.alloc(g->ctx, (size_t)(rows * ld));
    auto *hi = reinterpret_cast<__nv_bfloat16 *>(g->d_Th.p);
    auto *lo = reinterpret_cast<__nv_bfloat16 *>(g->d_Tl.p);
    if (!g->has_T) {
        // on-the-fly geometry: the split is generated from the pair formulas
        split_tiled_gen<<<dim3((unsigned)ktiles, (unsigned)(rows / kBM)), 256, 0, g->ctx->stream>>>(
            g->n_atoms, (int)n, g->model == PLX_WFQFMU, ktiles, g->d_pos.p, g->d_par.p, hi, lo);
    } else if (g->t_symmetric) {
        split_tiled<<<4096, 256, 0, g->ctx->stream>>>((int)n, ktiles, rows * ld, g->d_T.p, hi, lo);
    } else {
        // stored transposed (BEM): split the transpose
        split_tiled_t<<<dim3((unsigned)ktiles, (unsigned)(rows / kBM)), 256, 0, g->ctx->stream>>>((int)n, ktiles,
                                                                                                 g->d_T.p, hi, lo);
    }
    g->ctx->launches++;
    PLX_CHECK_CUDA(cudaGetLastError());
    if (!g->d_tc_err.p) {
        g->d_tc_err.alloc(g->ctx, 1);
        PLX_CHECK_CUDA(cudaMemsetAsync(g->d_tc_err.p, 0, sizeof(int), g->ctx->stream));
    }
}

// Interface of an alloy: rows I with neighbours of another type, the atoms J
// whose T charge rows the correction needs (I and those neighbours), and the
// cross-type entries of I as a CSR over positions in J.
static void build_interface(plx_geom *g) {
    plx_ctx *ctx = g->ctx;
    cudaStream_t st = ctx->stream;
    const int N = g->n_atoms;
    std::vector<int32_t> rowptr(N + 1), type(N);
    std::vector<int32_t> col((size_t)g->nnz);
    std::vector<double> kt((size_t)g->nnz);
    PLX_CHECK_CUDA(cudaMemcpyAsync(rowptr.data(), g->d_rowptr.p, (N + 1) * 4, cudaMemcpyDeviceToHost, st));
    PLX_CHECK_CUDA(cudaMemcpyAsync(type.data(), g->d_type.p, N * 4, cudaMemcpyDeviceToHost, st));
    if (g->nnz) {
        PLX_CHECK_CUDA(cudaMemcpyAsync(col.data(), g->d_col.p, g->nnz * 4, cudaMemcpyDeviceToHost, st));
        PLX_CHECK_CUDA(cudaMemcpyAsync(kt.data(), g->d_ktval.p, g->nnz * 8, cudaMemcpyDeviceToHost, st));
    }
    PLX_CHECK_CUDA(cudaStreamSynchronize(st));
    std::vector<int32_t> pos(N, -1), J, rows, ptr(1, 0), xcol, xtj;
    std::vector<double> xkt;
    auto place = [&](int a) {
        if (pos[a] < 0) {
            pos[a] = (int32_t)J.size();
            J.push_back(a);
        }
    };
    for (int i = 0; i < N; ++i) {
        bool any = false;
        for (int e = rowptr[i]; e < rowptr[i + 1]; ++e)
            if (type[col[e]] != type[i]) any = true;
        if (!any) continue;
        place(i);
        rows.push_back(i);
        for (int e = rowptr[i]; e < rowptr[i + 1]; ++e) {
            const int j = col[e];
            if (type[j] == type[i]) continue;
            place(j);
            xcol.push_back(j);          // atom index for now
            xtj.push_back(type[j]);
            xkt.push_back(kt[e]);
        }
        ptr.push_back((int32_t)xcol.size());
    }
    for (auto &c : xcol) c = pos[c];
    std::vector<int32_t> ipos(rows.size());
    for (size_t t = 0; t < rows.size(); ++t) ipos[t] = pos[rows[t]];
    g->n_iface = (int)J.size();
    g->n_xrows = (int)rows.size();
    auto up_i = [&](DevArray<int32_t> &d, const std::vector<int32_t> &h) {
        d.alloc(ctx, std::max<size_t>(h.size(), 1));
        if (!h.empty()) PLX_CHECK_CUDA(cudaMemcpyAsync(d.p, h.data(), h.size() * 4, cudaMemcpyHostToDevice, st));
    };
    up_i(g->d_iface_atom, J);
    up_i(g->d_xrow, rows);
    up_i(g->d_xipos, ipos);
    up_i(g->d_xrowptr, ptr);
    up_i(g->d_xcol, xcol);
    up_i(g->d_xtj, xtj);
    g->d_xkt.alloc(ctx, std::max<size_t>(xkt.size(), 1));
    if (!xkt.empty()) PLX_CHECK_CUDA(cudaMemcpyAsync(g->d_xkt.p, xkt.data(), xkt.size() * 8, cudaMemcpyHostToDevice, st));
    PLX_CHECK_CUDA(cudaStreamSynchronize(st));
}

static void build_a_split(plx_geom *g) {
    if (g->d_Ah.p) return;
    const bool hetero = g->n_types > 1;
    if (hetero) build_interface(g);
    const int64_t n = g->n_var;
    const int64_t M = n + (hetero ? g->n_iface : 0);
    const int64_t ld = (n + kLdAlign - 1) / kLdAlign * kLdAlign;
    const int64_t rows = (M + kBM - 1) / kBM * kBM, ktiles = ld / kBK;
    g->ldk = ld;
    g->fold_rows = M;
    g->d_Ah.alloc(g->ctx, (size_t)(rows * ld));
    g->d_Al.alloc(g->ctx, (size_t)(rows * ld));
    // rows M..rows of the last m-tile are read by the kernel: zero them
    PLX_CHECK_CUDA(cudaMemsetAsync(g->d_Ah.p, 0, (size_t)(rows * ld) * 2, g->ctx->stream));
    PLX_CHECK_CUDA(cudaMemsetAsync(g->d_Al.p, 0, (size_t)(rows * ld) * 2, g->ctx->stream));
    const int fmu = g->model == PLX_WFQFMU, N = g->n_atoms;
    auto *hi = reinterpret_cast<__nv_bfloat16 *>(g->d_Ah.p);
    auto *lo = reinterpret_cast<__nv_bfloat16 *>(g->d_Al.p);
    const unsigned kchunks = (unsigned)((ld + 255) / 256);
    cudaStream_t st = g->ctx->stream;
    if (g->has_T) {
        fold_split<<<dim3((unsigned)M, kchunks), 256, 0, st>>>(
            N, (int)n, ld, ktiles, hetero, fmu, 0, 0, g->d_rowptr.p, g->d_col.p, g->d_kval.p, g->d_ktval.p, g->d_T.p,
            g->d_pos.p, g->d_par.p, g->d_iface_atom.p, hi, lo);
        g->ctx->launches++;
    } else {
        // matrix-free: dipole and interface rows generated element by element; the
        // charge rows folded chunk by chunk from a window of generated T rows that
        // covers the chunk's conductance neighbours (atoms are ordered in space, so
        // a window is the chunk plus the neighbours' reach)
        if (M > N) {
            fold_split<<<dim3((unsigned)(M - N), kchunks), 256, 0, st>>>(
                N, (int)n, ld, ktiles, hetero, fmu, N, 0, g->d_rowptr.p, g->d_col.p, g->d_kval.p, g->d_ktval.p,
                nullptr, g->d_pos.p, g->d_par.p, g->d_iface_atom.p, hi, lo);
            g->ctx->launches++;
        }
        std::vector<int32_t> rowptr(N + 1), col((size_t)g->nnz);
        PLX_CHECK_CUDA(cudaMemcpyAsync(rowptr.data(), g->d_rowptr.p, (N + 1) * 4, cudaMemcpyDeviceToHost, st));
        if (g->nnz) PLX_CHECK_CUDA(cudaMemcpyAsync(col.data(), g->d_col.p, g->nnz * 4, cudaMemcpyDeviceToHost, st));
        PLX_CHECK_CUDA(cudaStreamSynchronize(st));
        const int64_t max_rows = std::max<int64_t>(64, (int64_t)(6.0e9 / (8.0 * (double)n)));   // <= ~6 GB window
        DevArray<double> Tw;
        Tw.alloc(g->ctx, (size_t)(max_rows * n));
        int64_t r0 = 0;
        while (r0 < N) {
            // grow the chunk while its window fits
            int64_t r1 = r0, lo_w = r0, hi_w = r0;
            while (r1 < N) {
                int64_t l = std::min<int64_t>(lo_w, r1), h = std::max<int64_t>(hi_w, r1);
                for (int e = rowptr[r1]; e < rowptr[r1 + 1]; ++e) {
                    l = std::min<int64_t>(l, col[e]);
                    h = std::max<int64_t>(h, col[e]);
                }
                if (h - l + 1 > max_rows) break;
                lo_w = l;
                hi_w = h;
                ++r1;
            }
            if (r1 == r0) {
                // a single row reaching farther than the window: generate its T values in place
                fold_split<<<dim3(1, kchunks), 256, 0, st>>>(N, (int)n, ld, ktiles, hetero, fmu, r0, 0, g->d_rowptr.p,
                                                             g->d_col.p, g->d_kval.p, g->d_ktval.p, nullptr, g->d_pos.p,
                                                             g->d_par.p, g->d_iface_atom.p, hi, lo);
                g->ctx->launches++;
                r0 = r0 + 1;
                continue;
            }
            const int64_t W = hi_w - lo_w + 1;
            t_rows_gen<<<dim3((unsigned)W, (unsigned)((n + 255) / 256)), 256, 0, st>>>(N, (int)n, fmu, lo_w, g->d_pos.p,
                                                                                       g->d_par.p, Tw.p);
            fold_split<<<dim3((unsigned)(r1 - r0), kchunks), 256, 0, st>>>(
                N, (int)n, ld, ktiles, hetero, fmu, r0, lo_w, g->d_rowptr.p, g->d_col.p, g->d_kval.p, g->d_ktval.p,
                Tw.p, g->d_pos.p, g->d_par.p, g->d_iface_atom.p, hi, lo);
            g->ctx->launches += 2;
            PLX_CHECK_CUDA(cudaGetLastError());
            r0 = r1;
        }
        PLX_CHECK_CUDA(cudaStreamSynchronize(st));
    }
    PLX_CHECK_CUDA(cudaGetLastError());
    if (!g->d_tc_err.p) {
        g->d_tc_err.alloc(g->ctx, 1);
        PLX_CHECK_CUDA(cudaMemsetAsync(g->d_tc_err.p, 0, sizeof(int), g->ctx->stream));
    }
}

int64_t tc_fold_rows(plx_geom *g) {
    build_a_split(g);
    return g->fold_rows;
}

void tc_contract_group(const std::vector<TcItem> &items) {
    if (items.empty()) return;
    if ((int)items.size() > kMaxGroups) {
        // more contractions than one launch describes: in launches of kMaxGroups
        for (size_t i0 = 0; i0 < items.size(); i0 += kMaxGroups)
            tc_contract_group(std::vector<TcItem>(items.begin() + i0,
                                                  items.begin() + std::min(items.size(), i0 + kMaxGroups)));
        return;
    }
    plx_ctx *ctx = items[0].g->ctx;
    const int nprod = items[0].nprod;
    for (const TcItem &it : items)
        if (it.g->ctx != ctx || it.nprod != nprod)
            throw Error(PLX_ERR_ARG, "a grouped contraction needs one context and one product count");
    for (size_t i = 0; i < items.size(); ++i)
        for (size_t j = 0; j < i; ++j)
            if (items[i].g == items[j].g) {
                // one geometry twice: its column split buffers hold one operand at a time
                for (const TcItem &it : items) tc_contract_group({it});
                return;
            }
    const bool single = items.size() == 1;
    // longest k first: the hardware hands CTAs to free SMs in launch order
    std::vector<int> order(items.size());
    for (size_t i = 0; i < items.size(); ++i) order[i] = (int)i;
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int b) { return items[a].g->n_var > items[b].g->n_var; });
    TcLaunch L;
    std::memset(&L, 0, sizeof(L));
    L.ngroups = (int)items.size();
    L.wait_limit = ctx->wait_limit;
    int units = 0, bn_max = 32;
    const int sms = sm_count(ctx->device);
    struct Post {
        int gi, rem;
    };
    std::vector<Post> post;
    for (int k = 0; k < L.ngroups; ++k) {
        const TcItem &it = items[order[k]];
        plx_geom *g = it.g;
        if (it.folded)
            build_a_split(g);
        else
            build_t_split(g);
        const int n = g->n_var;
        // output rows: n, or the folded operand's rows (n plus interface rows); S is [R][M]
        const int M = it.folded ? (int)g->fold_rows : n;
        const int R = 2 * it.count;
        const int64_t ld = g->ldk;
        // column tiles: as few as possible, each a multiple of 16 columns (<= 256, the
        // MMA's N granularity, which keeps the padding of a tile under 16 columns)
        const int ntile = (R + 255) / 256;
        const int bn = ((R + ntile - 1) / ntile + 15) / 16 * 16;
        const int Rpad = ntile * bn;
        const size_t need = (size_t)Rpad * ld;
        if (g->d_Xh.n < need) {
            g->d_Xh.alloc(ctx, need);
            g->d_Xl.alloc(ctx, need);
        }
        split_bf16<<<std::min<int64_t>(4096, n_blocks((int64_t)Rpad * ld, 256)), 256, 0, ctx->stream>>>(
            R, n, n, it.X, Rpad, ld, reinterpret_cast<__nv_bfloat16 *>(g->d_Xh.p),
            reinterpret_cast<__nv_bfloat16 *>(g->d_Xl.p));
        ctx->launches++;
        L.map[k][2] = make_map(g->d_Xh.p, ld, Rpad, ld, bn);
        L.map[k][3] = make_map(g->d_Xl.p, ld, Rpad, ld, bn);
        TcGroup &gp = L.grp[k];
        // A in tile order, one contiguous pre-swizzled 16 KB block per stage tile
        gp.ah = reinterpret_cast<const uint8_t *>(it.folded ? g->d_Ah.p : g->d_Th.p);
        gp.al = reinterpret_cast<const uint8_t *>(it.folded ? g->d_Al.p : g->d_Tl.p);
        gp.M = M;
        gp.R = R;
        gp.bn = bn;
        gp.ktiles = (int)(ld / kBK);
        gp.ctiles = ntile;
        gp.unit0 = units;
        gp.S = it.S;
        const int mtiles = (M + kBM - 1) / kBM;
        units += make_schedule(gp, mtiles * ntile, sms, single);
        const int rem = mtiles * ntile - gp.full;
        if (rem > 0) {
            const size_t pn = (size_t)rem * gp.q * kBM * bn;
            if (g->d_tcpart.n < pn) g->d_tcpart.alloc(ctx, pn);
            gp.P = g->d_tcpart.p;
            post.push_back({k, rem});
        }
        bn_max = std::max(bn_max, (bn + 31) / 32 * 32);
        if (!g->d_tc_err.p) throw Error(PLX_ERR_CUDA, "tensor-core error word missing");
        gp.err = g->d_tc_err.p;
    }
    L.bn_max = bn_max;
    L.stages = std::min(8, kSmemBudget / tc_stage_bytes(bn_max, nprod));
    const int smem = L.stages * tc_stage_bytes(bn_max, nprod) + 1024 /* align */ + 256 /* barriers */;
    auto kern = nprod == 1 ? tc_contract_kernel<1> : tc_contract_kernel<3>;
    once_per_device(reinterpret_cast<const void *>(kern), ctx->device, [&] {
        PLX_CHECK_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024));
    });
    kern<<<units, 128, smem, ctx->stream>>>(L);
    ctx->launches++;
    PLX_CHECK_CUDA(cudaGetLastError());
    for (const Post &q : post) {
        const TcGroup &gp = L.grp[q.gi];
        reduce_pieces<<<dim3(q.rem, (gp.bn + 31) / 32), kBM, 0, ctx->stream>>>(gp.M, gp.R, gp.bn, gp.full, gp.ctiles, gp.q,
                                                                      gp.P, gp.S);
        ctx->launches++;
    }
    PLX_CHECK_CUDA(cudaGetLastError());
}

void tc_contract(plx_geom *g, int count, const double *X, double *S, int nprod, bool folded) {
    tc_contract_group({TcItem{g, count, X, S, nprod, folded}});
}

int tc_error(plx_geom *g) {
    if (!g->d_tc_err.p) return 0;
    int h = 0;
    PLX_CHECK_CUDA(cudaMemcpyAsync(&h, g->d_tc_err.p, sizeof(int), cudaMemcpyDeviceToHost, g->ctx->stream));
    PLX_CHECK_CUDA(cudaStreamSynchronize(g->ctx->stream));
    // reported once: the next call starts clean
    if (h) PLX_CHECK_CUDA(cudaMemsetAsync(g->d_tc_err.p, 0, sizeof(int), g->ctx->stream));
    return h;
}

}  // namespace plx
