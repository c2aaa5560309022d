// Neighbour counts per atom on the device (get_neighbours,
// src/target/target_module.f90:417-464): for every atom i, the atoms j != i
// within the nearest-neighbour distance r0 of the pair's elements, counted once
// in n_neighbours (which starts at 1, the atom itself) and once in the
// per-type counts -- in i's own type when the two elements are the same, in
// j's type otherwise (i's own type also starts at 1).  The wFQFMu dipole
// diagonal uses the fractions counts / n_neighbours.
//
// The reference tests every pair (O(N^2) on the host).  Here the atoms are
// binned on the host into a uniform grid of cells at least one cutoff wide (a
// counting sort, O(N)), and one device thread per atom tests the atoms of the
// 27 surrounding cells.  The distance is the reference's expression on the
// input Angstrom coordinates, sqrt((dx^2 + dy^2) + dz^2) * ToBohr with every
// operation rounded on its own (no fused multiply-add), so that pairs sitting
// exactly on r0 (fcc lattices at their nearest-neighbour spacing) fall on the
// same side as in the reference.
#include <algorithm>
#include <cmath>
#include <vector>

#include "plx_internal.h"

using namespace plx;

namespace {

constexpr int kMaxTypes = 16;
constexpr double kToBohr = 1.8897261254578281;

__global__ void neighbour_kernel(int n, int nt, const double *__restrict__ xyz /*[3][n] Angstrom*/,
                                 const int32_t *__restrict__ type, const int32_t *__restrict__ type_z,
                                 const double *__restrict__ r0, const int32_t *__restrict__ cell_of,
                                 const int32_t *__restrict__ cell_start, const int32_t *__restrict__ cell_atoms,
                                 int cx, int cy, int cz, int32_t *__restrict__ nb, int32_t *__restrict__ n_nb) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int cnt[kMaxTypes];
    for (int t = 0; t < nt; ++t) cnt[t] = 0;
    const int ti = type[i];
    cnt[ti] = 1;
    int total = 1;
    const double xi = xyz[i], yi = xyz[n + i], zi = xyz[2 * n + i];
    const int c = cell_of[i];
    const int ix = c % cx, iy = (c / cx) % cy, iz = c / (cx * cy);
    for (int dz = -1; dz <= 1; ++dz) {
        const int z = iz + dz;
        if (z < 0 || z >= cz) continue;
        for (int dy = -1; dy <= 1; ++dy) {
            const int y = iy + dy;
            if (y < 0 || y >= cy) continue;
            for (int dx = -1; dx <= 1; ++dx) {
                const int x = ix + dx;
                if (x < 0 || x >= cx) continue;
                const int cell = (z * cy + y) * cx + x;
                for (int k = cell_start[cell]; k < cell_start[cell + 1]; ++k) {
                    const int j = cell_atoms[k];
                    if (j == i) continue;
                    const double ddx = __dadd_rn(xyz[j], -xi), ddy = __dadd_rn(xyz[n + j], -yi),
                                 ddz = __dadd_rn(xyz[2 * n + j], -zi);
                    const double s = __dadd_rn(__dadd_rn(__dmul_rn(ddx, ddx), __dmul_rn(ddy, ddy)), __dmul_rn(ddz, ddz));
                    const double d = __dmul_rn(__dsqrt_rn(s), kToBohr);
                    const int tj = type[j];
                    if (d <= r0[ti + nt * tj]) {
                        ++total;
                        if (type_z[ti] == type_z[tj]) ++cnt[ti];
                        else ++cnt[tj];
                    }
                }
            }
        }
    }
    for (int t = 0; t < nt; ++t) nb[(int64_t)i * nt + t] = cnt[t];
    n_nb[i] = total;
}

}  // namespace

namespace plx {

void neighbour_counts(plx_ctx *ctx, int n, int nt, const double *coord_ang, const int32_t *atom_type,
                      const int32_t *type_z, const double *r0, int32_t *nb_out, int32_t *n_nb_out) {
    if (n < 1 || nt < 1 || !coord_ang || !atom_type || !type_z || !r0 || !nb_out || !n_nb_out)
        throw Error(PLX_ERR_ARG, "neighbour counts: empty geometry or null array");
    if (nt > kMaxTypes) throw Error(PLX_ERR_ARG, "neighbour counts: at most 16 atom types");
    for (int i = 0; i < n; ++i)
        if (atom_type[i] < 0 || atom_type[i] >= nt) throw Error(PLX_ERR_ARG, "atom_type out of range");
    double rmax = 0.0;
    for (int k = 0; k < nt * nt; ++k) {
        if (!(r0[k] >= 0.0) || !std::isfinite(r0[k])) throw Error(PLX_ERR_ARG, "neighbour distance not finite");
        rmax = std::max(rmax, r0[k]);
    }
    // cells at least one cutoff wide (Angstrom, with a margin for rounding);
    // no more cells than about 8 per atom
    double lo[3], hi[3];
    for (int k = 0; k < 3; ++k) {
        lo[k] = hi[k] = coord_ang[k];
        for (int i = 1; i < n; ++i) {
            lo[k] = std::min(lo[k], coord_ang[3 * (size_t)i + k]);
            hi[k] = std::max(hi[k], coord_ang[3 * (size_t)i + k]);
        }
    }
    double h = std::max(rmax / kToBohr * (1.0 + 1e-6), 1e-6);
    int dims[3];
    for (;;) {
        double cells = 1.0;
        for (int k = 0; k < 3; ++k) {
            dims[k] = (int)std::floor((hi[k] - lo[k]) / h) + 1;
            cells *= dims[k];
        }
        if (cells <= 8.0 * n + 64.0) break;
        h *= 1.5;
    }
    const int ncell = dims[0] * dims[1] * dims[2];
    std::vector<int32_t> cell_of(n), start(ncell + 1, 0), atoms(n);
    for (int i = 0; i < n; ++i) {
        int c[3];
        for (int k = 0; k < 3; ++k)
            c[k] = std::min(dims[k] - 1, (int)std::floor((coord_ang[3 * (size_t)i + k] - lo[k]) / h));
        cell_of[i] = (c[2] * dims[1] + c[1]) * dims[0] + c[0];
        ++start[cell_of[i] + 1];
    }
    for (int c = 0; c < ncell; ++c) start[c + 1] += start[c];
    {
        std::vector<int32_t> fill(start.begin(), start.end() - 1);
        for (int i = 0; i < n; ++i) atoms[fill[cell_of[i]]++] = i;
    }
    std::vector<double> xyz(3 * (size_t)n);
    for (int i = 0; i < n; ++i)
        for (int k = 0; k < 3; ++k) xyz[(size_t)k * n + i] = coord_ang[3 * (size_t)i + k];
    std::vector<int32_t> tz(type_z, type_z + nt);
    cudaStream_t st = ctx->stream;
    DevArray<double> d_xyz, d_r0;
    DevArray<int32_t> d_type, d_tz, d_cell, d_start, d_atoms, d_nb, d_nnb;
    d_xyz.alloc(ctx, xyz.size());
    d_r0.alloc(ctx, (size_t)nt * nt);
    d_type.alloc(ctx, n);
    d_tz.alloc(ctx, nt);
    d_cell.alloc(ctx, n);
    d_start.alloc(ctx, ncell + 1);
    d_atoms.alloc(ctx, n);
    d_nb.alloc(ctx, (size_t)n * nt);
    d_nnb.alloc(ctx, n);
    PLX_CHECK_CUDA(cudaMemcpyAsync(d_xyz.p, xyz.data(), xyz.size() * 8, cudaMemcpyHostToDevice, st));
    PLX_CHECK_CUDA(cudaMemcpyAsync(d_r0.p, r0, (size_t)nt * nt * 8, cudaMemcpyHostToDevice, st));
    PLX_CHECK_CUDA(cudaMemcpyAsync(d_type.p, atom_type, (size_t)n * 4, cudaMemcpyHostToDevice, st));
    PLX_CHECK_CUDA(cudaMemcpyAsync(d_tz.p, tz.data(), (size_t)nt * 4, cudaMemcpyHostToDevice, st));
    PLX_CHECK_CUDA(cudaMemcpyAsync(d_cell.p, cell_of.data(), (size_t)n * 4, cudaMemcpyHostToDevice, st));
    PLX_CHECK_CUDA(cudaMemcpyAsync(d_start.p, start.data(), start.size() * 4, cudaMemcpyHostToDevice, st));
    PLX_CHECK_CUDA(cudaMemcpyAsync(d_atoms.p, atoms.data(), (size_t)n * 4, cudaMemcpyHostToDevice, st));
    prof_begin(ctx);
    neighbour_kernel<<<n_blocks(n, 128), 128, 0, st>>>(n, nt, d_xyz.p, d_type.p, d_tz.p, d_r0.p, d_cell.p,
                                                       d_start.p, d_atoms.p, dims[0], dims[1], dims[2], d_nb.p,
                                                       d_nnb.p);
    ctx->launches++;
    PLX_CHECK_CUDA(cudaGetLastError());
    // plx_profile_read category 8: coordinates, types and cell lists in, counts out
    prof_end(ctx, 8, 0.0, 24.0 * n + 4.0 * (3.0 * n + start.size()) + 4.0 * (double)n * (nt + 1));
    PLX_CHECK_CUDA(cudaMemcpyAsync(nb_out, d_nb.p, (size_t)n * nt * 4, cudaMemcpyDeviceToHost, st));
    PLX_CHECK_CUDA(cudaMemcpyAsync(n_nb_out, d_nnb.p, (size_t)n * 4, cudaMemcpyDeviceToHost, st));
    PLX_CHECK_CUDA(cudaStreamSynchronize(st));
}

}  // namespace plx
