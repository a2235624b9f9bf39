// ELL route of libpdb200: cell list, fixed-capacity neighbour rows and the
// row-wise LJ / WCA pair kernels, plus the NVE and Langevin (BAOAB) steps built
// on them.
//
// Semantics follow ParticleDynamics.jl's device neighbour workspace
// (src/neighbors/DeviceNeighborCUDA.jl: displacement and decision kernels,
// binning, row construction, capacity commit), its row pair traversal
// (src/engine/PairTraversal.jl, src/engine/PairModels.jl,
// src/nonbonded/LJELLEngineKernels.jl) and its Langevin BAOAB kernels
// (src/engine/Langevin.jl, src/engine/Philox.jl).  The layout is this
// library's own:
//   * the rows are slot-major (slot t of particle i at t * N + i, the
//     reference's _ell_index), so the row loads of consecutive particles
//     coalesce;
//   * particles inside a cell are ordered by id, so rows (and the summation
//     order of the pair kernel) are reproducible;
//   * rows are built by one thread per particle in cell order (neighbouring
//     threads share candidate cells), and the last block to finish commits
//     the capacity check;
//   * the displacement maximum and the rebuild decision run in one kernel
//     (the last block decides), fused with the drift in the step engine;
//   * the pair kernel reads packed (x, y, z, 0) coordinates, G lanes per row
//     reduced by shuffles, with the closing half kick fused in the step.
#include <cmath>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "ell_common.cuh"
#include "internal.hpp"

using namespace pdb;

namespace pdb {

// Standalone decision over the current coordinates (decide_device_neighbors!).
template <int D>
__global__ void __launch_bounds__(ELL_THREADS) k_ell_decide(const float *__restrict__ x, const float *__restrict__ y,
                                                            const float *__restrict__ z, const float4 *__restrict__ ref,
                                                            int n, float Lx, float Ly, float Lz, float threshold,
                                                            long long *__restrict__ st) {
    if (st[E_ERROR] != 0) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const float L[3] = {Lx, Ly, Lz};
    float v = 0.f;
    if (i < n) {
        const float p[3] = {x[i], y[i], D == 3 ? z[i] : 0.f};
        v = ell_displacement<D>(p, ref[i], L, st[E_VALID] != 0);
    }
    if (ell_block_max_last(__float_as_uint(v), st, E_DMAX, E_TICKET_D)) {
        const float largest = __uint_as_float((unsigned)st[E_DMAX]);
        st[E_DMAX] = 0;
        st[E_TICKET_D] = 0;
        ell_decide<false>(st, largest, threshold, 0);
    }
}

// Cell of every particle (_kernel_cell_ids3g!, DeviceNeighborCUDA.jl:472-487; 2D
// _kernel_cell_ids2!) and the cell histogram.
template <int D>
__global__ void k_ell_bin(const float *__restrict__ x, const float *__restrict__ y, const float *__restrict__ z, int n,
                          float Lx, float Ly, float Lz, int nx, int ny, int nz, int *__restrict__ cell_of,
                          int *__restrict__ cell_count, const long long *__restrict__ st) {
    if (!ell_requested(st)) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float u = x[i] + 0.5f * Lx;
    u -= floorf(u / Lx) * Lx;
    float v = y[i] + 0.5f * Ly;
    v -= floorf(v / Ly) * Ly;
    int cx = (int)floorf(u * ((float)nx / Lx));
    int cy = (int)floorf(v * ((float)ny / Ly));
    cx = min(max(cx, 0), nx - 1);
    cy = min(max(cy, 0), ny - 1);
    int cz = 0;
    if (D == 3) {
        float w = z[i] + 0.5f * Lz;
        w -= floorf(w / Lz) * Lz;
        cz = min(max((int)floorf(w * ((float)nz / Lz)), 0), nz - 1);
    }
    const int c = (cz * ny + cy) * nx + cx;
    cell_of[i] = c;
    atomicAdd(&cell_count[c], 1);
}

// Exclusive scan of the cell histogram into cell_off (ncell + 1 entries); the histogram is
// reset to zero for use as scatter cursors.  One CTA, chunks staged in shared memory.
__global__ void __launch_bounds__(1024) k_ell_scan(int *__restrict__ cell_count, int *__restrict__ cell_off,
                                                   int ncell, const long long *__restrict__ st) {
    if (!ell_requested(st)) return;
    __shared__ int sb[ELL_SCAN_CHUNK + ELL_SCAN_CHUNK / 32];
    __shared__ int warp_tot[32];
    __shared__ int s_next;
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    int carry = 0;
    for (int c0 = 0; c0 < ncell; c0 += ELL_SCAN_CHUNK) {
        const int nc = min(ELL_SCAN_CHUNK, ncell - c0);
        for (int k = t; k < ELL_SCAN_CHUNK; k += blockDim.x) {
            sb[k + (k >> 5)] = k < nc ? cell_count[c0 + k] : 0;
            if (k < nc) cell_count[c0 + k] = 0;
        }
        __syncthreads();
        constexpr int PER = ELL_SCAN_CHUNK / 1024;
        int run = 0;
#pragma unroll
        for (int k = 0; k < PER; ++k) {
            const int i = t * PER + k;
            run += sb[i + (i >> 5)];
        }
        int inc = run;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const int yv = __shfl_up_sync(0xffffffffu, inc, off);
            if (lane >= off) inc += yv;
        }
        if (lane == 31) warp_tot[w] = inc;
        __syncthreads();
        if (w == 0) {
            const int tv = warp_tot[lane];
            int ti = tv;
#pragma unroll
            for (int off = 1; off < 32; off <<= 1) {
                const int yv = __shfl_up_sync(0xffffffffu, ti, off);
                if (lane >= off) ti += yv;
            }
            warp_tot[lane] = ti - tv;
        }
        __syncthreads();
        int ex = carry + warp_tot[w] + inc - run;
#pragma unroll
        for (int k = 0; k < PER; ++k) {
            const int i = t * PER + k;
            const int v = sb[i + (i >> 5)];
            sb[i + (i >> 5)] = ex;
            ex += v;
        }
        if (t == (int)blockDim.x - 1) s_next = ex;   // the exclusive prefix after the chunk
        __syncthreads();
        for (int k = t; k < nc; k += blockDim.x) cell_off[c0 + k] = sb[k + (k >> 5)];
        carry = s_next;
        __syncthreads();
    }
    if (t == 0) cell_off[ncell] = carry;
}

// _kernel_scatter_by_cell! (DenseNeighborCUDA.jl:61-72): atomic cursors per cell.
__global__ void k_ell_scatter(const int *__restrict__ cell_of, int n, const int *__restrict__ cell_off,
                              int *__restrict__ cursor, int *__restrict__ sorted, const long long *__restrict__ st) {
    if (!ell_requested(st)) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int c = cell_of[i];
    sorted[cell_off[c] + atomicAdd(&cursor[c], 1)] = i;
}

// Particles of a cell in ascending id (one warp per cell), which makes the rows and the pair
// sums independent of the atomic cursor order.  Cells above 32 entries rank through `tmp`.
// The cell's scatter cursor is reset to zero for the next build's histogram.
__global__ void k_ell_cellsort(const int *__restrict__ cell_off, int ncell, int *__restrict__ sorted,
                               int *__restrict__ tmp, int *__restrict__ cell_count, const long long *__restrict__ st) {
    if (!ell_requested(st)) return;
    const int c = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
    if (c >= ncell) return;   // uniform per warp
    if (lane == 0) cell_count[c] = 0;   // the scatter cursors become the next build's zeroed histogram
    const int a = cell_off[c], n = cell_off[c + 1] - a;
    if (n <= 1) return;
    if (n <= 32) {
        const int id = lane < n ? sorted[a + lane] : 0x7fffffff;
        int r = 0;
        for (int j = 0; j < n; ++j) r += __shfl_sync(0xffffffffu, id, j) < id ? 1 : 0;
        __syncwarp();
        if (lane < n) sorted[a + r] = id;
        return;
    }
    for (int k = lane; k < n; k += 32) {
        const int id = sorted[a + k];
        int r = 0;
        for (int j = 0; j < n; ++j) r += sorted[a + j] < id ? 1 : 0;
        tmp[a + r] = id;
    }
    __syncwarp();
    for (int k = lane; k < n; k += 32) sorted[a + k] = tmp[a + k];
}

// Row construction (_kernel_neighbors3g!, DeviceNeighborCUDA.jl:510-559; 2D _kernel_neighbors2!,
// DenseNeighborCUDA.jl:77-123): thread t takes particle sorted[t] and walks the cell-row stencil
// (z, then y offsets; x cells in range order), keeping j != i with r^2 <= r_list^2 (nearest
// image by one conditional shift).  Rows past the capacity are counted but not stored.  The
// build reference coordinates are refreshed; the last block commits (_device_commit_kernel!,
// DeviceNeighborCUDA.jl:345-404).
template <int D, bool ALLPAIRS>
__global__ void __launch_bounds__(ELL_THREADS) k_ell_rows(
    const float *__restrict__ x, const float *__restrict__ y, const float *__restrict__ z, int n,
    const int *__restrict__ sorted, const int *__restrict__ cell_of, const int *__restrict__ cell_off, float Lx,
    float Ly, float Lz, int nx, int ny, int nz, float rl2, int cap, int *__restrict__ rows, int *__restrict__ counts,
    float4 *__restrict__ ref, long long *__restrict__ st) {
    if (!ell_requested(st)) return;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    int found = 0;
    if (t < n) {
        const int i = ALLPAIRS ? t : sorted[t];
        const float xi = x[i], yi = y[i], zi = D == 3 ? z[i] : 0.f;
        const float hLx = 0.5f * Lx, hLy = 0.5f * Ly, hLz = 0.5f * Lz;
        auto visit = [&](int j) {
            if (j == i) return;
            const float dx = mic_fast(x[j] - xi, hLx, Lx);
            const float dy = mic_fast(y[j] - yi, hLy, Ly);
            float r2;
            if (D == 3) {
                const float dz = mic_fast(z[j] - zi, hLz, Lz);
                r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
            } else {
                r2 = fmaf(dx, dx, dy * dy);
            }
            if (r2 <= rl2) {
                if (found < cap) rows[(size_t)found * n + i] = j;
                ++found;
            }
        };
        if (ALLPAIRS) {
            for (int j = 0; j < n; ++j) visit(j);
        } else {
            const float rl = sqrtf(rl2);
            const float hx = Lx / (float)nx, hy = Ly / (float)ny, hz = Lz / (float)nz;
            const int Sx = ell_reach(rl, Lx, nx), Sy = ell_reach(rl, Ly, ny);
            const int Sz = D == 3 ? ell_reach(rl, Lz, nz) : 0;
            const int c0 = cell_of[i];
            const int cx = c0 % nx, tmp = c0 / nx, cy = tmp % ny, cz = tmp / ny;
            for (int oz = -Sz; oz <= Sz; ++oz) {
                int cz2 = cz + oz;
                cz2 -= cz2 >= nz ? nz : 0;
                cz2 += cz2 < 0 ? nz : 0;
                const float gz = (float)max(abs(oz) - 1, 0) * hz;
                for (int oy = -Sy; oy <= Sy; ++oy) {
                    int cy2 = cy + oy;
                    cy2 -= cy2 >= ny ? ny : 0;
                    cy2 += cy2 < 0 ? ny : 0;
                    const float gy = (float)max(abs(oy) - 1, 0) * hy;
                    const float g2 = fmaf(gy, gy, gz * gz);
                    if (g2 > rl2) continue;
                    const int row = (cz2 * ny + cy2) * nx;
                    int a1, b1, a2, b2;
                    ell_row_ranges(cx, g2, rl2, hx, Sx, nx, a1, b1, a2, b2);
                    for (int k = cell_off[row + a1]; k < cell_off[row + b1 + 1]; ++k) visit(sorted[k]);
                    if (a2 <= b2)
                        for (int k = cell_off[row + a2]; k < cell_off[row + b2 + 1]; ++k) visit(sorted[k]);
                }
            }
        }
        counts[i] = found;
        ref[i] = make_float4(xi, yi, zi, 0.f);
    }
    if (ell_block_max_last((unsigned)found, st, E_RMAX, E_TICKET_R)) {
        // commit: the largest row against the capacity
        const long long largest = st[E_RMAX];
        st[E_RMAX] = 0;
        st[E_TICKET_R] = 0;
        st[E_REQUIRED] = largest;
        if (largest > cap) {
            st[E_ERROR] = E_ERR_CAPACITY;
            st[E_VALID] = 0;
        } else {
            st[E_VALID] = 1;
            st[E_LAST_BUILD] = st[E_STEP];
            st[E_BUILDS] += 1;
        }
    }
}

// Row construction, cell-staged: one warp per cell.  The warp walks the same stencil segments
// in the same order as k_ell_rows (z, then y offsets; x cells in range order; each cell's
// particles in id order), stages the candidates (x, y, z, id) in shared memory once for the
// whole cell, and every lane (a particle of the cell) scans them with the same arithmetic as
// k_ell_rows, so the rows are identical entry by entry.  Chunks of ROWS_CAP candidates are
// scanned in turn when the stencil holds more.
constexpr int ROWS_WARPS = 4, ROWS_CAP = 640;   // 40 KB of staging per block (below the 48 KB default)
constexpr int ROWS_MIN_PER_CELL = 8;            // mean cell occupancy from which the cell-staged kernel is used

template <int D>
__global__ void __launch_bounds__(32 * ROWS_WARPS) k_ell_rows_cells(
    const float *__restrict__ x, const float *__restrict__ y, const float *__restrict__ z, int n,
    const int *__restrict__ sorted, const int *__restrict__ cell_off, float Lx, float Ly, float Lz, int nx, int ny,
    int nz, float rl2, int cap, int *__restrict__ rows, int *__restrict__ counts, float4 *__restrict__ ref,
    long long *__restrict__ st) {
    if (!ell_requested(st)) return;
    extern __shared__ float4 ell_stage[];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ncell = nx * ny * nz;
    const int c = blockIdx.x * ROWS_WARPS + w;
    float4 *sw = ell_stage + w * ROWS_CAP;
    unsigned fmax = 0;
    if (c < ncell) {   // warp-uniform
        const float hLx = 0.5f * Lx, hLy = 0.5f * Ly, hLz = 0.5f * Lz;
        const float rl = sqrtf(rl2);
        const float hx = Lx / (float)nx, hy = Ly / (float)ny, hz = Lz / (float)nz;
        const int Sx = ell_reach(rl, Lx, nx), Sy = ell_reach(rl, Ly, ny);
        const int Sz = D == 3 ? ell_reach(rl, Lz, nz) : 0;
        const int cx = c % nx, tmp = c / nx, cy = tmp % ny, cz = tmp / ny;
        const int p0 = cell_off[c], pn = cell_off[c + 1] - p0;
        for (int pg = 0; pg < pn; pg += 32) {
            const bool has = pg + lane < pn;
            const int i = has ? sorted[p0 + pg + lane] : -1;
            const float xi = has ? x[i] : 0.f, yi = has ? y[i] : 0.f, zi = (has && D == 3) ? z[i] : 0.f;
            // bounding box of this group's particles: a candidate farther than the list radius from the
            // box is farther from every particle of the group and is not staged (a conservative margin
            // keeps rounding from dropping a candidate that the exact test below would accept)
            float bl[3] = {has ? xi : INFINITY, has ? yi : INFINITY, has ? zi : INFINITY};
            float bh[3] = {has ? xi : -INFINITY, has ? yi : -INFINITY, has ? zi : -INFINITY};
#pragma unroll
            for (int d = 0; d < 3; ++d) {
#pragma unroll
                for (int off = 16; off > 0; off >>= 1) {
                    bl[d] = fminf(bl[d], __shfl_xor_sync(0xffffffffu, bl[d], off));
                    bh[d] = fmaxf(bh[d], __shfl_xor_sync(0xffffffffu, bh[d], off));
                }
            }
            const float bcx = 0.5f * (bl[0] + bh[0]), bcy = 0.5f * (bl[1] + bh[1]), bcz = 0.5f * (bl[2] + bh[2]);
            const float bhx = 0.5f * (bh[0] - bl[0]), bhy = 0.5f * (bh[1] - bl[1]), bhz = 0.5f * (bh[2] - bl[2]);
            const float rbox = rl * 1.0001f + 1e-3f;
            const float rbox2 = rbox * rbox;
            int found = 0;
            int fill = 0;
            auto scan = [&]() {
                __syncwarp();
                if (has) {
                    for (int t = 0; t < fill; ++t) {
                        const float4 cj = sw[t];
                        const int j = __float_as_int(cj.w);
                        if (j == i) continue;
                        const float dx = mic_fast(cj.x - xi, hLx, Lx);
                        const float dy = mic_fast(cj.y - yi, hLy, Ly);
                        float r2;
                        if (D == 3) {
                            const float dz = mic_fast(cj.z - zi, hLz, Lz);
                            r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
                        } else {
                            r2 = fmaf(dx, dx, dy * dy);
                        }
                        if (r2 <= rl2) {
                            if (found < cap) rows[(size_t)found * n + i] = j;
                            ++found;
                        }
                    }
                }
                __syncwarp();
                fill = 0;
            };
            auto stage = [&](int ka, int kb) {
                for (int k0 = ka; k0 < kb; k0 += 32) {
                    const bool in = lane < kb - k0;
                    const int j = in ? sorted[k0 + lane] : 0;
                    const float cx3 = in ? x[j] : 0.f, cy3 = in ? y[j] : 0.f, cz3 = (in && D == 3) ? z[j] : 0.f;
                    const float ex = fmaxf(fabsf(mic_fast(cx3 - bcx, hLx, Lx)) - bhx, 0.f);
                    const float ey = fmaxf(fabsf(mic_fast(cy3 - bcy, hLy, Ly)) - bhy, 0.f);
                    const float ez = D == 3 ? fmaxf(fabsf(mic_fast(cz3 - bcz, hLz, Lz)) - bhz, 0.f) : 0.f;
                    const bool keep = in && fmaf(ex, ex, fmaf(ey, ey, ez * ez)) <= rbox2;
                    const unsigned bal = __ballot_sync(0xffffffffu, keep);
                    const int nk = __popc(bal);
                    if (fill + nk > ROWS_CAP) scan();
                    if (keep)   // staged in the candidates' order
                        sw[fill + __popc(bal & ((1u << lane) - 1u))] = make_float4(cx3, cy3, cz3, __int_as_float(j));
                    fill += nk;
                }
            };
            for (int oz = -Sz; oz <= Sz; ++oz) {
                int cz2 = cz + oz;
                cz2 -= cz2 >= nz ? nz : 0;
                cz2 += cz2 < 0 ? nz : 0;
                const float gz = (float)max(abs(oz) - 1, 0) * hz;
                for (int oy = -Sy; oy <= Sy; ++oy) {
                    int cy2 = cy + oy;
                    cy2 -= cy2 >= ny ? ny : 0;
                    cy2 += cy2 < 0 ? ny : 0;
                    const float gy = (float)max(abs(oy) - 1, 0) * hy;
                    const float g2 = fmaf(gy, gy, gz * gz);
                    if (g2 > rl2) continue;
                    const int row = (cz2 * ny + cy2) * nx;
                    int a1, b1, a2, b2;
                    ell_row_ranges(cx, g2, rl2, hx, Sx, nx, a1, b1, a2, b2);
                    stage(cell_off[row + a1], cell_off[row + b1 + 1]);
                    if (a2 <= b2) stage(cell_off[row + a2], cell_off[row + b2 + 1]);
                }
            }
            scan();
            if (has) {
                counts[i] = found;
                ref[i] = make_float4(xi, yi, zi, 0.f);
            }
            fmax = max(fmax, (unsigned)found);
        }
    }
    if (ell_block_max_last(fmax, st, E_RMAX, E_TICKET_R)) {
        const long long largest = st[E_RMAX];
        st[E_RMAX] = 0;
        st[E_TICKET_R] = 0;
        st[E_REQUIRED] = largest;
        if (largest > cap) {
            st[E_ERROR] = E_ERR_CAPACITY;
            st[E_VALID] = 0;
        } else {
            st[E_VALID] = 1;
            st[E_LAST_BUILD] = st[E_STEP];
            st[E_BUILDS] += 1;
        }
    }
}

// Packed coordinates (x, y, z, 0) for the pair kernel's 16-byte neighbour loads.
template <int D>
__global__ void k_ell_pack(const float *__restrict__ x, const float *__restrict__ y, const float *__restrict__ z,
                           int n, float4 *__restrict__ xq) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) xq[i] = make_float4(x[i], y[i], D == 3 ? z[i] : 0.f, 0.f);
}

struct EllModel {
    int kind;        // PD_PAIR_LJ or PD_PAIR_WCA
    float eps, sig2, rc2, eshift;
};

struct EllKick {     // closing half kick fused into the pair kernel (step engine)
    float *vx, *vy, *vz;
    const float *inv_mass;
    float inv_mass_uniform, half_dt;
    int advance;     // advance the device step counter (last kernel of a step)
    float *dU, *ekin;   // Langevin bookkeeping of the closing kick (B2), or null
};

// Row pair kernel (_pair_cooperative_kernel!, PairTraversal.jl:66-125, with the UniformLJ /
// UniformWCA models of PairModels.jl:13-49): G lanes per particle stride its row; per pair the
// compensated periodic difference, nested multiply-add r^2, f/r = 24 eps (2 s12 - s6) / r^2 and
// u = 4 eps (s12 - s6) - shift (LJ) or + eps (WCA) inside (0, rc^2); each row gets half of every
// pair energy and half of its dyadic virial.  Forces are stored (not added).
template <int D, int G, bool ENERGY, bool KICK>
__global__ void __launch_bounds__(ELL_THREADS) k_ell_pairs(const float4 *__restrict__ xq, int n,
                                                           const int *__restrict__ rows,
                                                           const int *__restrict__ counts, float Lx, float Ly,
                                                           float Lz, EllModel m, float *__restrict__ fx,
                                                           float *__restrict__ fy, float *__restrict__ fz,
                                                           float *__restrict__ epot, float *__restrict__ vir,
                                                           EllKick kick, long long *__restrict__ st) {
    if (st[E_VALID] == 0) return;   // _device_if_valid!: no valid list, no forces
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = tid / G, lane = tid % G;
    const float hLx = 0.5f * Lx, hLy = 0.5f * Ly, hLz = 0.5f * Lz;
    constexpr int NV = D == 3 ? 6 : 3;
    float a[3] = {0.f, 0.f, 0.f}, e = 0.f, w[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k) w[k] = 0.f;
    if (i < n) {
        const float4 pi = xq[i];
        const int cnt = counts[i];
        auto pair = [&](float4 pj) {
            const float dx = periodic_delta(pi.x, pj.x, hLx, Lx);
            const float dy = periodic_delta(pi.y, pj.y, hLy, Ly);
            const float dz = D == 3 ? periodic_delta(pi.z, pj.z, hLz, Lz) : 0.f;
            const float r2 = D == 3 ? fmaf(dx, dx, fmaf(dy, dy, dz * dz)) : fmaf(dx, dx, dy * dy);
            if (r2 > 0.f && r2 < m.rc2) {
                const float ir2 = 1.f / r2;
                const float s2 = m.sig2 * ir2;
                const float s6 = s2 * s2 * s2;
                const float s12 = s6 * s6;
                const float fr = 24.f * m.eps * (2.f * s12 - s6) * ir2;
                const float fxv = fr * dx, fyv = fr * dy, fzv = fr * dz;
                a[0] += fxv;
                a[1] += fyv;
                if (D == 3) a[2] += fzv;
                if (ENERGY) {
                    const float u = 4.f * m.eps * (s12 - s6) + (m.kind == PD_PAIR_WCA ? m.eps : -m.eshift);
                    e += 0.5f * u;
                    if (D == 3) {
                        w[0] += 0.5f * dx * fxv;
                        w[1] += 0.5f * dy * fyv;
                        w[2] += 0.5f * dz * fzv;
                        w[3] += 0.5f * dx * fyv;
                        w[4] += 0.5f * dx * fzv;
                        w[5] += 0.5f * dy * fzv;
                    } else {
                        w[0] += 0.5f * dx * fxv;
                        w[1] += 0.5f * dy * fyv;
                        w[2] += 0.5f * dx * fyv;
                    }
                }
            }
        };
        int slot = lane;
        // two neighbours per iteration: both loads in flight before either is used
        for (; slot + G < cnt; slot += 2 * G) {
            const float4 p1 = xq[rows[(size_t)slot * n + i]];
            const float4 p2 = xq[rows[(size_t)(slot + G) * n + i]];
            pair(p1);
            pair(p2);
        }
        for (; slot < cnt; slot += G) pair(xq[rows[(size_t)slot * n + i]]);
    }
    // every lane reaches every shuffle
#pragma unroll
    for (int off = G / 2; off > 0; off >>= 1) {
#pragma unroll
        for (int d = 0; d < 3; ++d) a[d] += __shfl_down_sync(0xffffffffu, a[d], off, G);
        if (ENERGY) {
            e += __shfl_down_sync(0xffffffffu, e, off, G);
#pragma unroll
            for (int k = 0; k < NV; ++k) w[k] += __shfl_down_sync(0xffffffffu, w[k], off, G);
        }
    }
    if (lane == 0 && i < n) {
        fx[i] = a[0];
        fy[i] = a[1];
        if (D == 3) fz[i] = a[2];
        if (ENERGY) {
            epot[i] = e;
#pragma unroll
            for (int k = 0; k < NV; ++k) vir[(size_t)i * NV + k] = w[k];
        }
        if (KICK) {
            const float im = kick.inv_mass ? kick.inv_mass[i] : kick.inv_mass_uniform;
            const float c = kick.half_dt * im;
            const float v0 = fmaf(c, a[0], kick.vx[i]), v1 = fmaf(c, a[1], kick.vy[i]);
            const float v2 = D == 3 ? fmaf(c, a[2], kick.vz[i]) : 0.f;
            kick.vx[i] = v0;
            kick.vy[i] = v1;
            if (D == 3) kick.vz[i] = v2;
            if (kick.dU) {   // _b2_kernel! (Langevin.jl:141-160): power v.f and kinetic energy after B2
                kick.dU[i] += v0 * a[0] + v1 * a[1] + v2 * a[2];
                kick.ekin[i] = 0.5f * (v0 * v0 + v1 * v1 + v2 * v2) / im;
            }
        }
    }
    if (KICK && kick.advance && blockIdx.x == 0 && threadIdx.x == 0) st[E_STEP] += 1;
}

__global__ void k_ell_word(long long *st, int word, long long value) { st[word] = value; }

}  // namespace pdb

// ------------------------------------------------------------------ host side

struct pd_ell {
    pd_ell_params p;
    int dim = 3, n = 0;
    double box[3] = {0, 0, 0};
    float L[3] = {0, 0, 0};
    int nx = 1, ny = 1, nz = 1, ncell = 1;
    bool allpairs = false;
    float rl2 = 0.f, threshold = 0.f;
    int lanes = 1;
    int cap = 0;
    long long *st = nullptr;
    int *cell_of = nullptr, *cell_count = nullptr, *cell_off = nullptr, *sorted = nullptr, *tmp = nullptr;
    int *rows = nullptr, *counts = nullptr;
    float4 *ref = nullptr, *xq = nullptr;
};

namespace pdb {

static void ell_free(pd_ell *e) {
    dfree(e->st);
    dfree(e->cell_of);
    dfree(e->cell_count);
    dfree(e->cell_off);
    dfree(e->sorted);
    dfree(e->tmp);
    dfree(e->rows);
    dfree(e->counts);
    dfree(e->ref);
    dfree(e->xq);
}

EllModel ell_model(const pd_ell *e) {
    EllModel m;
    m.kind = e->p.model;
    m.eps = e->p.eps;
    m.sig2 = e->p.sigma * e->p.sigma;
    m.rc2 = e->p.rc2;
    m.eshift = e->p.eshift;
    return m;
}

// Decision + flag-gated rebuild kernels on stream s (the rebuild returns at once unless the
// device decided to rebuild).
int ell_rebuild_launch(pd_ell *e, const float *x, const float *y, const float *z, cudaStream_t s) {
    const int n = e->n, blocks = (n + ELL_THREADS - 1) / ELL_THREADS;
    const float Lx = e->L[0], Ly = e->L[1], Lz = e->L[2];
    if (!e->allpairs) {
        if (e->dim == 3)
            k_ell_bin<3><<<blocks, ELL_THREADS, 0, s>>>(x, y, z, n, Lx, Ly, Lz, e->nx, e->ny, e->nz, e->cell_of,
                                                        e->cell_count, e->st);
        else
            k_ell_bin<2><<<blocks, ELL_THREADS, 0, s>>>(x, y, z, n, Lx, Ly, Lz, e->nx, e->ny, e->nz, e->cell_of,
                                                        e->cell_count, e->st);
        PD_LAUNCHED();
        k_ell_scan<<<1, 1024, 0, s>>>(e->cell_count, e->cell_off, e->ncell, e->st);
        PD_LAUNCHED();
        k_ell_scatter<<<blocks, ELL_THREADS, 0, s>>>(e->cell_of, n, e->cell_off, e->cell_count, e->sorted, e->st);
        PD_LAUNCHED();
        k_ell_cellsort<<<(int)(((long long)e->ncell * 32 + 255) / 256), 256, 0, s>>>(e->cell_off, e->ncell, e->sorted,
                                                                                    e->tmp, e->cell_count, e->st);
        PD_LAUNCHED();
    }
#define PD_ELL_ROWS(DD, AP)                                                                                           \
    k_ell_rows<DD, AP><<<blocks, ELL_THREADS, 0, s>>>(x, y, z, n, e->sorted, e->cell_of, e->cell_off, Lx, Ly, Lz,    \
                                                      e->nx, e->ny, e->nz, e->rl2, e->cap, e->rows, e->counts, e->ref, \
                                                      e->st)
#define PD_ELL_ROWS_CELLS(DD)                                                                                         \
    k_ell_rows_cells<DD><<<(e->ncell + ROWS_WARPS - 1) / ROWS_WARPS, 32 * ROWS_WARPS,                                \
                           sizeof(float4) * ROWS_WARPS * ROWS_CAP, s>>>(x, y, z, n, e->sorted, e->cell_off, Lx, Ly,  \
                                                                        Lz, e->nx, e->ny, e->nz, e->rl2, e->cap,     \
                                                                        e->rows, e->counts, e->ref, e->st)
    // a warp per cell pays off once cells hold enough particles to occupy its lanes
    const bool cells = !e->allpairs && n >= ROWS_MIN_PER_CELL * e->ncell;
    if (e->dim == 3) {
        if (e->allpairs) PD_ELL_ROWS(3, true);
        else if (cells) PD_ELL_ROWS_CELLS(3);
        else PD_ELL_ROWS(3, false);
    } else {
        if (e->allpairs) PD_ELL_ROWS(2, true);
        else if (cells) PD_ELL_ROWS_CELLS(2);
        else PD_ELL_ROWS(2, false);
    }
#undef PD_ELL_ROWS
#undef PD_ELL_ROWS_CELLS
    PD_LAUNCHED();
    return PD_OK;
}

// The counting sort of particles into cells, shared with the batched replicas: exclusive scan of
// the histogram (which becomes the scatter cursors), the scatter, id order inside each cell; every
// kernel returns at once unless st asks for a rebuild.
int ell_sort_cells_launch(const int *cell_of, int n, int ncell, int *cell_count, int *cell_off, int *sorted, int *tmp,
                          long long *st, cudaStream_t s) {
    const int blocks = (n + ELL_THREADS - 1) / ELL_THREADS;
    k_ell_scan<<<1, 1024, 0, s>>>(cell_count, cell_off, ncell, st);
    PD_LAUNCHED();
    k_ell_scatter<<<blocks, ELL_THREADS, 0, s>>>(cell_of, n, cell_off, cell_count, sorted, st);
    PD_LAUNCHED();
    k_ell_cellsort<<<(int)(((long long)ncell * 32 + 255) / 256), 256, 0, s>>>(cell_off, ncell, sorted, tmp, cell_count,
                                                                             st);
    PD_LAUNCHED();
    return PD_OK;
}

int ell_decide_launch(pd_ell *e, const float *x, const float *y, const float *z, cudaStream_t s) {
    const int blocks = (e->n + ELL_THREADS - 1) / ELL_THREADS;
    if (e->dim == 3)
        k_ell_decide<3><<<blocks, ELL_THREADS, 0, s>>>(x, y, z, e->ref, e->n, e->L[0], e->L[1], e->L[2], e->threshold,
                                                       e->st);
    else
        k_ell_decide<2><<<blocks, ELL_THREADS, 0, s>>>(x, y, z, e->ref, e->n, e->L[0], e->L[1], e->L[2], e->threshold,
                                                       e->st);
    PD_LAUNCHED();
    return PD_OK;
}

template <int D, int G>
static void ell_pairs_g(pd_ell *e, float *fx, float *fy, float *fz, float *epot, float *vir, int energy,
                        const EllKick &kick, cudaStream_t s) {
    const int blocks = (int)(((long long)e->n * G + ELL_THREADS - 1) / ELL_THREADS);
    const EllModel m = ell_model(e);
    if (kick.vx) {
        if (energy)
            k_ell_pairs<D, G, true, true><<<blocks, ELL_THREADS, 0, s>>>(e->xq, e->n, e->rows, e->counts, e->L[0],
                                                                         e->L[1], e->L[2], m, fx, fy, fz, epot, vir,
                                                                         kick, e->st);
        else
            k_ell_pairs<D, G, false, true><<<blocks, ELL_THREADS, 0, s>>>(e->xq, e->n, e->rows, e->counts, e->L[0],
                                                                          e->L[1], e->L[2], m, fx, fy, fz, epot, vir,
                                                                          kick, e->st);
    } else {
        if (energy)
            k_ell_pairs<D, G, true, false><<<blocks, ELL_THREADS, 0, s>>>(e->xq, e->n, e->rows, e->counts, e->L[0],
                                                                          e->L[1], e->L[2], m, fx, fy, fz, epot, vir,
                                                                          kick, e->st);
        else
            k_ell_pairs<D, G, false, false><<<blocks, ELL_THREADS, 0, s>>>(e->xq, e->n, e->rows, e->counts, e->L[0],
                                                                           e->L[1], e->L[2], m, fx, fy, fz, epot, vir,
                                                                           kick, e->st);
    }
}

template <int D>
static void ell_pairs_d(pd_ell *e, float *fx, float *fy, float *fz, float *epot, float *vir, int energy,
                        const EllKick &kick, cudaStream_t s) {
    switch (e->lanes) {
        case 1: ell_pairs_g<D, 1>(e, fx, fy, fz, epot, vir, energy, kick, s); break;
        case 2: ell_pairs_g<D, 2>(e, fx, fy, fz, epot, vir, energy, kick, s); break;
        case 4: ell_pairs_g<D, 4>(e, fx, fy, fz, epot, vir, energy, kick, s); break;
        default: ell_pairs_g<D, 8>(e, fx, fy, fz, epot, vir, energy, kick, s); break;
    }
}

// The pair kernel over packed coordinates that are already in e->xq.
int ell_pairs_launch(pd_ell *e, float *fx, float *fy, float *fz, float *epot, float *vir, int energy,
                     const EllKick &kick, cudaStream_t s) {
    if (e->dim == 3) ell_pairs_d<3>(e, fx, fy, fz, epot, vir, energy, kick, s);
    else ell_pairs_d<2>(e, fx, fy, fz, epot, vir, energy, kick, s);
    PD_LAUNCHED();
    return PD_OK;
}

int ell_pack_launch(pd_ell *e, const float *x, const float *y, const float *z, cudaStream_t s) {
    const int blocks = (e->n + ELL_THREADS - 1) / ELL_THREADS;
    if (e->dim == 3) k_ell_pack<3><<<blocks, ELL_THREADS, 0, s>>>(x, y, z, e->n, e->xq);
    else k_ell_pack<2><<<blocks, ELL_THREADS, 0, s>>>(x, y, z, e->n, e->xq);
    PD_LAUNCHED();
    return PD_OK;
}

long long *ell_state(pd_ell *e) { return e->st; }
float4 *ell_packed(pd_ell *e) { return e->xq; }
float4 *ell_ref(pd_ell *e) { return e->ref; }
float ell_threshold(const pd_ell *e) { return e->threshold; }
int ell_dim(const pd_ell *e) { return e->dim; }
int ell_capacity(const pd_ell *e) { return e->cap; }

static int ell_alloc_rows(pd_ell *e, int cap) {
    PD_CHECK(cap > 0, PD_EINVAL, "Invalid ELL capacity");
    PD_CHECK((long long)e->n * cap <= 0x7fffffffLL, PD_EINVAL,
             "Neighbor table of %d particles x cap %d exceeds the Int32 index range; lower `cap`", e->n, cap);
    dfree(e->rows);
    int rc = dalloc(&e->rows, (size_t)e->n * cap);
    if (rc) return rc;
    PD_CUDA(cudaMemset(e->rows, 0xff, sizeof(int) * (size_t)e->n * cap));
    e->cap = cap;
    return PD_OK;
}

}  // namespace pdb

extern "C" {

int pd_ell_create(pd_ell **out, const pd_ell_params *p, const double box[3]) {
    PD_CHECK(out && p && box, PD_EINVAL, "pd_ell_create: null argument");
    *out = nullptr;
    PD_CHECK(p->dim == 2 || p->dim == 3, PD_EINVAL, "Device ELL supports 2D/3D boxes");
    PD_CHECK(p->n > 0, PD_EINVAL, "pd_ell_create: particle count must be positive");
    PD_CHECK(p->interval >= 1 && p->interval <= 100, PD_EINVAL, "Rebuild interval must be between 1 and 100");
    PD_CHECK(p->cap > 0, PD_EINVAL, "Invalid ELL capacity");
    PD_CHECK(std::isfinite(p->cutoff) && p->cutoff > 0, PD_EINVAL, "Cutoff must be positive and finite");
    PD_CHECK(std::isfinite(p->skin) && p->skin >= 0, PD_EINVAL, "Neighbor skin must be finite and nonnegative");
    PD_CHECK(p->model == PD_PAIR_LJ || p->model == PD_PAIR_WCA, PD_EINVAL, "pd_ell_create: unknown pair model %d",
             p->model);
    PD_CHECK(p->lanes == 0 || p->lanes == 1 || p->lanes == 2 || p->lanes == 4 || p->lanes == 8, PD_EINVAL,
             "pd_ell_create: lanes must be 0, 1, 2, 4 or 8");
    for (int d = 0; d < p->dim; ++d)
        PD_CHECK(std::isfinite(box[d]) && box[d] > 0, PD_EINVAL, "box lengths must be finite and positive");
    pd_ell *e = new pd_ell();
    e->p = *p;
    e->dim = p->dim;
    e->n = p->n;
    for (int d = 0; d < 3; ++d) {
        e->box[d] = d < p->dim ? box[d] : 1.0;
        e->L[d] = (float)e->box[d];
    }
    // cells of width >= r_list (_alloc_neighbor_matrix, NeighborAllocation.jl:28-54 with sub = 1)
    const float rl = (float)p->cutoff + (float)p->skin;
    const float cell = fmaxf(1e-6f, rl);
    e->rl2 = rl * rl;
    e->threshold = 0.25f * (float)p->skin * (float)p->skin;
    int ng[3] = {1, 1, 1};
    for (int d = 0; d < p->dim; ++d) ng[d] = std::max(1, (int)std::floor(e->L[d] / cell));
    for (int d = 0; d < p->dim; ++d) {
        if (2.0 * rl > e->box[d]) {
            delete e;
            set_error("neighbor list radius %g needs every box length above %g", (double)rl, 2.0 * rl);
            return PD_EINVAL;
        }
        if (ng[d] < 3) e->allpairs = true;   // small boxes: rows from all pairs (no cell is visited twice)
    }
    e->nx = ng[0];
    e->ny = ng[1];
    e->nz = ng[2];
    if (e->allpairs) e->nx = e->ny = e->nz = 1;
    e->ncell = e->nx * e->ny * e->nz;
    // lanes per row: the expected row length at this density
    if (p->lanes) {
        e->lanes = p->lanes;
    } else {
        double vol = 1.0;
        for (int d = 0; d < p->dim; ++d) vol *= e->box[d];
        const double shell = p->dim == 3 ? 4.18879 * (double)rl * rl * rl : 3.14159265 * (double)rl * rl;
        const double expected = p->n / vol * shell;
        e->lanes = expected < 12 ? 1 : expected < 40 ? 2 : 4;
    }
    int rc;
    if ((rc = dalloc(&e->st, E_LEN)) || (rc = dalloc(&e->cell_of, (size_t)e->n)) ||
        (rc = dalloc(&e->cell_count, (size_t)e->ncell)) || (rc = dalloc(&e->cell_off, (size_t)e->ncell + 1)) ||
        (rc = dalloc(&e->sorted, (size_t)e->n)) || (rc = dalloc(&e->tmp, (size_t)e->n)) ||
        (rc = dalloc(&e->counts, (size_t)e->n)) || (rc = dalloc(&e->ref, (size_t)e->n)) ||
        (rc = dalloc(&e->xq, (size_t)e->n)) || (rc = ell_alloc_rows(e, p->cap))) {
        ell_free(e);
        delete e;
        return rc;
    }
    long long init[E_LEN] = {0};
    init[E_INTERVAL] = p->interval;
    if (cudaMemcpy(e->st, init, sizeof init, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemset(e->cell_count, 0, sizeof(int) * (size_t)e->ncell) != cudaSuccess ||
        cudaMemset(e->counts, 0, sizeof(int) * (size_t)e->n) != cudaSuccess ||
        cudaMemset(e->ref, 0, sizeof(float4) * (size_t)e->n) != cudaSuccess) {
        ell_free(e);
        delete e;
        set_error("pd_ell_create: device initialisation failed");
        return PD_ECUDA;
    }
    *out = e;
    return PD_OK;
}

int pd_ell_destroy(pd_ell *e) {
    if (!e) return PD_OK;
    ell_free(e);
    delete e;
    return PD_OK;
}

int pd_ell_update(pd_ell *e, const float *x, const float *y, const float *z, pd_stream_t sp) {
    PD_CHECK(e && x && y && (e->dim == 2 || z), PD_EINVAL, "pd_ell_update: null argument");
    cudaStream_t s = (cudaStream_t)sp;
    int rc;
    if ((rc = ell_decide_launch(e, x, y, z, s))) return rc;
    return ell_rebuild_launch(e, x, y, z, s);
}

int pd_ell_request(pd_ell *e, pd_stream_t sp) {
    PD_CHECK(e, PD_EINVAL, "pd_ell_request: null handle");
    k_ell_word<<<1, 1, 0, (cudaStream_t)sp>>>(e->st, E_VALID, 0);
    PD_LAUNCHED();
    return PD_OK;
}

int pd_ell_forces(pd_ell *e, const float *x, const float *y, const float *z, float *fx, float *fy, float *fz,
                  float *epot, float *vir, int energy, pd_stream_t sp) {
    PD_CHECK(e && x && y && fx && fy && (e->dim == 2 || (z && fz)), PD_EINVAL, "pd_ell_forces: null argument");
    PD_CHECK(!energy || (epot && vir), PD_EINVAL, "pd_ell_forces: energy needs epot and vir");
    cudaStream_t s = (cudaStream_t)sp;
    int rc;
    if ((rc = ell_pack_launch(e, x, y, z, s))) return rc;
    EllKick kick;
    memset(&kick, 0, sizeof kick);
    return ell_pairs_launch(e, fx, fy, fz, epot, vir, energy, kick, s);
}

int pd_ell_status(pd_ell *e, pd_ell_stats *out) {
    PD_CHECK(e && out, PD_EINVAL, "pd_ell_status: null argument");
    long long h[E_LEN];
    PD_CUDA(cudaMemcpy(h, e->st, sizeof h, cudaMemcpyDeviceToHost));
    out->valid = h[E_VALID] != 0;
    out->error = (int)h[E_ERROR];
    out->requested = h[E_REQUEST] != 0;
    out->step = h[E_STEP];
    out->last_build = h[E_LAST_BUILD];
    out->interval = h[E_INTERVAL];
    out->checks = h[E_CHECKS];
    out->builds = h[E_BUILDS];
    out->required = h[E_REQUIRED];
    out->cap = e->cap;
    out->lanes = e->lanes;
    out->allpairs = e->allpairs ? 1 : 0;
    return PD_OK;
}

int pd_ell_rows(pd_ell *e, int **rows, int **counts) {
    PD_CHECK(e && rows && counts, PD_EINVAL, "pd_ell_rows: null argument");
    *rows = e->rows;
    *counts = e->counts;
    return PD_OK;
}

int pd_ell_resize(pd_ell *e, int cap) {
    PD_CHECK(e, PD_EINVAL, "pd_ell_resize: null handle");
    int rc = ell_alloc_rows(e, cap);
    if (rc) return rc;
    // rearm_capacity_rebuild!: clear the latched capacity error, request the rebuild again
    long long h[E_LEN];
    PD_CUDA(cudaMemcpy(h, e->st, sizeof h, cudaMemcpyDeviceToHost));
    if (h[E_ERROR] == E_ERR_CAPACITY) h[E_ERROR] = 0;
    h[E_VALID] = 0;
    PD_CUDA(cudaMemcpy(e->st, h, sizeof h, cudaMemcpyHostToDevice));
    return PD_OK;
}

}  // extern "C"

// ------------------------------------------------------------------ step engine on the ELL route

namespace pdb {

// Counter-based Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11 "Parallel random numbers: as easy
// as 1, 2, 3"), the generator of the reference's graph-safe Langevin noise (src/engine/Philox.jl:
// counter (particle, stream, step low, step high), key = the user seed).
__device__ __forceinline__ void philox4x32_10(unsigned c[4], unsigned k0, unsigned k1) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        if (r > 0) {
            k0 += 0x9E3779B9u;
            k1 += 0xBB67AE85u;
        }
        const unsigned long long p0 = (unsigned long long)0xD2511F53u * c[0];
        const unsigned long long p1 = (unsigned long long)0xCD9E8D57u * c[2];
        const unsigned hi0 = (unsigned)(p0 >> 32), lo0 = (unsigned)p0;
        const unsigned hi1 = (unsigned)(p1 >> 32), lo1 = (unsigned)p1;
        const unsigned n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
        c[0] = n0;
        c[1] = lo1;
        c[2] = n2;
        c[3] = lo0;
    }
}

// Uniform in the open interval (0, 1) from the top 24 bits, then a Box-Muller pair
// (Philox.jl: _open01, _box_muller).
__device__ __forceinline__ float open01(unsigned u) { return ((float)(u >> 8) + 0.5f) * 5.9604644775390625e-8f; }
__device__ __forceinline__ void box_muller(float u1, float u2, float &a, float &b) {
    const float r = sqrtf(-2.f * logf(u1));
    float sn, cs;
    sincospif(2.f * u2, &sn, &cs);
    a = r * cs;
    b = r * sn;
}

// Four standard normals for particle id (1-based), stream and step (philox_normals4).
__device__ __forceinline__ void philox_normals4(unsigned long long seed, unsigned long long step, unsigned id,
                                                unsigned stream, float out[4]) {
    unsigned c[4] = {id, stream, (unsigned)step, (unsigned)(step >> 32)};
    philox4x32_10(c, (unsigned)seed, (unsigned)(seed >> 32));
    box_muller(open01(c[0]), open01(c[1]), out[0], out[1]);
    box_muller(open01(c[2]), open01(c[3]), out[2], out[3]);
}

struct EllStepArgs {
    int n;
    float *x, *y, *z, *vx, *vy, *vz;
    const float *fx, *fy, *fz;
    const float *inv_mass;
    float inv_mass_uniform;
    float L[3];
    float dt;
    // Langevin (BAOAB, GJF)
    float gamma, noise;   // friction and noise scale sqrt(2 gamma kT dt)
    unsigned long long seed;
    float *f0x, *f0y, *f0z;   // GJF: the previous step's force
    float kick;               // BAOAB / BAOA: the B1 kick length, dt (BAOAB) or 2 dt (BAOA, no B2)
    float *dq, *dU, *ekin;    // Langevin bookkeeping (heat, work of the forces, kinetic energy), or null
    float4 *xq;
    const float4 *ref;
    float threshold;
};

__device__ __forceinline__ float wrap_half(float x, float L) {
    // _wrap (Langevin.jl:53-56): one shift into [-L/2, L/2)
    x -= (x >= 0.5f * L) ? L : 0.f;
    x += (x < -0.5f * L) ? L : 0.f;
    return x;
}

// Per-particle drift of the step (MODE 0: NVE half kick + drift, _nve_kick_drift3_kernel!;
// MODE 1: Langevin B1 A1 O A2, _baoa_kernel! of Langevin.jl:58-88 with FP64 intermediates and
// Philox noise keyed on the particle and the device step), the pack of the new coordinates, the
// displacement maximum and, in the last block, the rebuild decision.
template <int D, int MODE, bool COND>
__global__ void __launch_bounds__(ELL_THREADS) k_ell_drift(EllStepArgs a, long long *__restrict__ st,
                                                           cudaGraphConditionalHandle h) {
    if (st[E_ERROR] != 0) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = st[E_VALID] != 0;
    float disp = 0.f;
    if (i < a.n && valid) {
        const float im = a.inv_mass ? a.inv_mass[i] : a.inv_mass_uniform;
        float p[3] = {a.x[i], a.y[i], D == 3 ? a.z[i] : 0.f};
        float v[3] = {a.vx[i], a.vy[i], D == 3 ? a.vz[i] : 0.f};
        const float f[3] = {a.fx[i], a.fy[i], D == 3 ? a.fz[i] : 0.f};
        if (MODE == 0) {
            const float c = 0.5f * a.dt * im;
#pragma unroll
            for (int d = 0; d < D; ++d) {
                v[d] = fmaf(c, f[d], v[d]);
                p[d] = wrap_half(fmaf(a.dt, v[d], p[d]), a.L[d]);
            }
        } else if (MODE == 2) {
            // GJF positions (_gjf_pos_kernel!, Langevin.jl:164-181; gjf_pos_coefs, Masses.jl:47-56):
            // q = g dt / (2m), b = 1 / (1 + q), x += b dt v + b dt / (2m) (dt f + beta); the force is
            // kept as the old force of the velocity update
            const float q = a.gamma * a.dt * im / 2.f;
            const float b = 1.f / (1.f + q);
            const float coef = b * a.dt * im / 2.f;
            float xi[4];
            philox_normals4(a.seed, (unsigned long long)st[E_STEP], (unsigned)(i + 1), 0u, xi);
#pragma unroll
            for (int d = 0; d < D; ++d) {
                const float beta = a.noise * xi[d];
                const float dp = b * a.dt * v[d] + coef * (a.dt * f[d] + beta);
                p[d] = wrap_half(p[d] + dp, a.L[d]);
            }
            a.f0x[i] = f[0];
            a.f0y[i] = f[1];
            if (D == 3) a.f0z[i] = f[2];
        } else {
            const double dt = a.dt, imA = im, g = a.gamma;
            const double hk = (double)a.kick * imA / 2.0;   // kick = dt (BAOAB) or 2 dt (BAOA)
            double v1[3], x1[3], pw = 0.0;
#pragma unroll
            for (int d = 0; d < D; ++d) {
                v1[d] = (double)v[d] + hk * (double)f[d];        // B1
                x1[d] = (double)p[d] + 0.5 * dt * v1[d];         // A1
                pw += v1[d] * (double)f[d];
            }
            const double c = exp(-g * dt * imA);
            const double rr = sqrt((1.0 - c * c) * imA / (2.0 * g * dt));
            float xi[4];
            philox_normals4(a.seed, (unsigned long long)st[E_STEP], (unsigned)(i + 1), 0u, xi);
            double vb2 = 0.0, vbb = 0.0;
#pragma unroll
            for (int d = 0; d < D; ++d) {
                const double beta = (double)(a.noise * xi[d]);
                const double v2 = c * v1[d] + rr * beta;         // O
                const double vbar = 0.5 * (v1[d] + v2);
                vb2 += vbar * vbar;
                vbb += vbar * beta;
                v[d] = (float)v2;
                p[d] = wrap_half((float)(x1[d] + 0.5 * dt * v2), a.L[d]);   // A2
            }
            if (a.dq) {   // _baoa_kernel! (Langevin.jl:58-78): dU += v1.f after B1, dq += -g |vbar|^2 + vbar.beta / dt
                a.dU[i] += (float)pw;
                a.dq[i] += (float)(-g * vb2 + vbb / dt);
            }
        }
        a.x[i] = p[0];
        a.y[i] = p[1];
        a.vx[i] = v[0];
        a.vy[i] = v[1];
        if (D == 3) {
            a.z[i] = p[2];
            a.vz[i] = v[2];
        }
        a.xq[i] = make_float4(p[0], p[1], p[2], 0.f);
        disp = ell_displacement<D>(p, a.ref[i], a.L, true);
    }
    if (ell_block_max_last(__float_as_uint(disp), st, E_DMAX, E_TICKET_D)) {
        const float largest = __uint_as_float((unsigned)st[E_DMAX]);
        st[E_DMAX] = 0;
        st[E_TICKET_D] = 0;
        ell_decide<COND>(st, largest, a.threshold, h);
    }
}

// GJF velocities (_gjf_vel_kernel!, Langevin.jl:183-208; gjf_q, gjf_vel_coefs, Masses.jl:58-70):
// a = (1 - q) / (1 + q), b = 1 / (1 + q), v = a v + dt / (2m) (a f_old + f) + (b / m) beta with the
// same draw beta as the positions (same device step), in FP64; then the device step advances.
template <int D>
__global__ void __launch_bounds__(ELL_THREADS) k_ell_gjf_vel(EllStepArgs a, long long *__restrict__ st) {
    if (st[E_ERROR] != 0 || st[E_VALID] == 0) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < a.n) {
        const float im = a.inv_mass ? a.inv_mass[i] : a.inv_mass_uniform;
        const float q = a.gamma * a.dt * im / 2.f;
        const double aA = (double)((1.f - q) / (1.f + q)), bA = (double)(1.f / (1.f + q));
        const double kf = (double)a.dt * (double)im / 2.0, nf = bA * (double)im;
        float xi[4];
        philox_normals4(a.seed, (unsigned long long)st[E_STEP], (unsigned)(i + 1), 0u, xi);
        float *v[3] = {a.vx, a.vy, a.vz};
        const float *f[3] = {a.fx, a.fy, a.fz};
        const float *f0[3] = {a.f0x, a.f0y, a.f0z};
        double v2 = 0.0, psto = 0.0, pcons = 0.0;
#pragma unroll
        for (int d = 0; d < D; ++d) {
            const double beta = (double)(a.noise * xi[d]);
            const double vp = (double)v[d][i];
            const double vn = aA * vp + kf * (aA * (double)f0[d][i] + (double)f[d][i]) + nf * beta;
            v2 += vn * vn;
            psto += 0.5 * (vp + vn) * (beta / bA);
            pcons += vn * (double)f[d][i];
            v[d][i] = (float)vn;
        }
        if (a.dq) {   // P_diss = -g |v|^2, P_sto = vbar.(beta / b) / dt, P_cons = v.f (Langevin.jl:199-206)
            const double g = a.gamma;
            a.ekin[i] = (float)(0.5 * v2 / (double)im);
            a.dq[i] -= (float)(-g * v2 + psto / (double)a.dt);
            a.dU[i] += (float)pcons;
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) st[E_STEP] += 1;
}

}  // namespace pdb

struct pd_ell_md {
    pd_ell *e = nullptr;
    pd_md_state st;
    cudaStream_t body = nullptr;
    bool cond_nodes = true;
    // graphs: [mode (0 NVE, 1 Langevin BAOAB, 2 Langevin GJF)][energy]
    cudaGraphExec_t exec[3][2] = {{nullptr, nullptr}, {nullptr, nullptr}, {nullptr, nullptr}};
    EllStepArgs key[3][2];
    cudaStream_t exec_stream[3][2] = {{nullptr, nullptr}, {nullptr, nullptr}, {nullptr, nullptr}};
    float *f0 = nullptr;   // GJF old forces, 3 n
    float *dq = nullptr, *dU = nullptr, *ekin = nullptr;   // caller-owned Langevin bookkeeping, or null
};

namespace pdb {

static EllStepArgs ell_step_args(pd_ell_md *md, float dt, float gamma, float kT, unsigned long long seed,
                                 float kick) {
    EllStepArgs a;
    memset(&a, 0, sizeof a);
    pd_ell *e = md->e;
    a.n = e->n;
    a.x = md->st.x;
    a.y = md->st.y;
    a.z = md->st.z;
    a.vx = md->st.vx;
    a.vy = md->st.vy;
    a.vz = md->st.vz;
    a.fx = md->st.fx;
    a.fy = md->st.fy;
    a.fz = md->st.fz;
    a.inv_mass = md->st.inv_mass;
    a.inv_mass_uniform = md->st.inv_mass_uniform;
    for (int d = 0; d < 3; ++d) a.L[d] = e->L[d];
    a.dt = dt;
    a.gamma = gamma;
    a.noise = gamma > 0.f ? (float)std::sqrt(2.0 * (double)gamma * (double)kT * (double)dt) : 0.f;
    a.seed = seed;
    a.kick = kick;
    if (gamma > 0.f) {
        a.dq = md->dq;
        a.dU = md->dU;
        a.ekin = md->ekin;
    }
    a.xq = e->xq;
    a.ref = e->ref;
    a.threshold = e->threshold;
    if (md->f0) {
        a.f0x = md->f0;
        a.f0y = md->f0 + e->n;
        a.f0z = md->f0 + 2 * (size_t)e->n;
    }
    return a;
}

// One step: drift (+ decision), the flag-gated rebuild (an IF node when captured with cond), the
// pair kernel with the closing half kick and the step advance.
static int ell_enqueue_step(pd_ell_md *md, const EllStepArgs &a, int mode, int energy, cudaStream_t s, int cond) {
    pd_ell *e = md->e;
    const int blocks = (e->n + ELL_THREADS - 1) / ELL_THREADS;
    cudaGraphConditionalHandle h = 0;
    if (cond) {
        cudaStreamCaptureStatus status;
        cudaGraph_t g = nullptr;
        PD_CUDA(cudaStreamGetCaptureInfo(s, &status, nullptr, &g, nullptr, nullptr));
        PD_CUDA(cudaGraphConditionalHandleCreate(&h, g, 0, cudaGraphCondAssignDefault));
    }
#define PD_ELL_DRIFT(DD, MM, CC) k_ell_drift<DD, MM, CC><<<blocks, ELL_THREADS, 0, s>>>(a, e->st, h)
#define PD_ELL_DRIFT_D(DD)                                                        \
    if (mode == 0) { if (cond) PD_ELL_DRIFT(DD, 0, true); else PD_ELL_DRIFT(DD, 0, false); } \
    else if (mode == 1) { if (cond) PD_ELL_DRIFT(DD, 1, true); else PD_ELL_DRIFT(DD, 1, false); } \
    else { if (cond) PD_ELL_DRIFT(DD, 2, true); else PD_ELL_DRIFT(DD, 2, false); }
    if (e->dim == 3) {
        PD_ELL_DRIFT_D(3)
    } else {
        PD_ELL_DRIFT_D(2)
    }
#undef PD_ELL_DRIFT_D
#undef PD_ELL_DRIFT
    PD_LAUNCHED();
    int rc;
    if (cond) {
        if ((rc = capture_if_body(s, md->body, h, [&](cudaStream_t cs) {
                 return ell_rebuild_launch(e, md->st.x, md->st.y, md->st.z, cs);
             })))
            return rc;
    } else {
        if ((rc = ell_rebuild_launch(e, md->st.x, md->st.y, md->st.z, s))) return rc;
    }
    EllKick kick;
    memset(&kick, 0, sizeof kick);
    if (mode == 2) {
        // GJF: forces without a kick, then the velocity update (which advances the step)
        if ((rc = ell_pairs_launch(e, md->st.fx, md->st.fy, md->st.fz, md->st.epot, md->st.vir6, energy, kick, s)))
            return rc;
        if (e->dim == 3) k_ell_gjf_vel<3><<<blocks, ELL_THREADS, 0, s>>>(a, e->st);
        else k_ell_gjf_vel<2><<<blocks, ELL_THREADS, 0, s>>>(a, e->st);
        PD_LAUNCHED();
        return PD_OK;
    }
    kick.vx = md->st.vx;
    kick.vy = md->st.vy;
    kick.vz = md->st.vz;
    kick.inv_mass = md->st.inv_mass;
    kick.inv_mass_uniform = md->st.inv_mass_uniform;
    if (mode == 1) {
        kick.dU = a.dU;
        kick.ekin = a.ekin;
    }
    // the closing half kick: dt / 2 (NVE, BAOAB), none for BAOA (its B1 kicked the full 2 dt / 2)
    kick.half_dt = mode == 1 ? 0.5f * (2.f * a.dt - a.kick) : 0.5f * a.dt;
    kick.advance = 1;
    return ell_pairs_launch(e, md->st.fx, md->st.fy, md->st.fz, md->st.epot, md->st.vir6, energy, kick, s);
}

static int ell_run(pd_ell_md *md, int mode, int nsteps, float dt, float gamma, float kT, unsigned long long seed,
                   int energy_last, int use_graph, cudaStream_t s, float kick = 0.f) {
    const EllStepArgs a = ell_step_args(md, dt, gamma, kT, seed, kick > 0.f ? kick : dt);
    for (int k = 0; k < nsteps; ++k) {
        const int energy = (energy_last && k == nsteps - 1) ? 1 : 0;
        if (!use_graph) {
            int rc = ell_enqueue_step(md, a, mode, energy, s, 0);
            if (rc) return rc;
            continue;
        }
        cudaGraphExec_t &ex = md->exec[mode][energy];
        if (!ex || memcmp(&md->key[mode][energy], &a, sizeof a) != 0 || md->exec_stream[mode][energy] != s) {
            if (ex) {
                cudaGraphExecDestroy(ex);
                ex = nullptr;
            }
            PD_CHECK(s != nullptr, PD_EINVAL, "ELL step: graph replay needs a non-default stream");
            for (int attempt = 0; attempt < 2 && !ex; ++attempt) {
                const int cond = md->cond_nodes ? 1 : 0;
                cudaGraph_t g = nullptr;
                PD_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
                const int rc = ell_enqueue_step(md, a, mode, energy, s, cond);
                cudaError_t err = cudaStreamEndCapture(s, &g);
                if (rc == PD_OK && err == cudaSuccess) err = cudaGraphInstantiate(&ex, g, 0);
                if (g) cudaGraphDestroy(g);
                if (rc == PD_OK && err == cudaSuccess) break;
                ex = nullptr;
                cudaGetLastError();
                if (!cond) {
                    if (rc) return rc;
                    PD_CHECK(false, PD_ECUDA, "ELL step capture failed: %s", cudaGetErrorString(err));
                }
                md->cond_nodes = false;
            }
            md->key[mode][energy] = a;
            md->exec_stream[mode][energy] = s;
        }
        PD_CUDA(cudaGraphLaunch(ex, s));
    }
    return PD_OK;
}

}  // namespace pdb

extern "C" {

int pd_ell_md_create(pd_ell_md **out, pd_ell *e, const pd_md_state *st) {
    PD_CHECK(out && e && st, PD_EINVAL, "pd_ell_md_create: null argument");
    *out = nullptr;
    PD_CHECK(st->n == e->n, PD_EINVAL, "pd_ell_md_create: state has %d particles, the list %d", st->n, e->n);
    PD_CHECK(st->x && st->y && st->vx && st->vy && st->fx && st->fy, PD_EINVAL, "pd_ell_md_create: state arrays missing");
    PD_CHECK(e->dim == 2 || (st->z && st->vz && st->fz), PD_EINVAL, "pd_ell_md_create: 3D state needs z arrays");
    pd_ell_md *md = new pd_ell_md();
    md->e = e;
    md->st = *st;
    memset(md->key, 0, sizeof md->key);
    if (cudaStreamCreateWithFlags(&md->body, cudaStreamNonBlocking) != cudaSuccess) {
        delete md;
        set_error("pd_ell_md_create: stream creation failed");
        return PD_ECUDA;
    }
    *out = md;
    return PD_OK;
}

int pd_ell_md_destroy(pd_ell_md *md) {
    if (!md) return PD_OK;
    for (int m = 0; m < 3; ++m)
        for (int k = 0; k < 2; ++k)
            if (md->exec[m][k]) cudaGraphExecDestroy(md->exec[m][k]);
    if (md->body) cudaStreamDestroy(md->body);
    dfree(md->f0);
    delete md;
    return PD_OK;
}

// evaluate_forces_into_f! on the ELL route: decision + rebuild at the current coordinates, then
// the forces (no kick, no step advance).
int pd_ell_md_evaluate(pd_ell_md *md, int energy, pd_stream_t sp) {
    PD_CHECK(md, PD_EINVAL, "pd_ell_md_evaluate: null handle");
    PD_CHECK(!energy || (md->st.epot && md->st.vir6), PD_EINVAL, "pd_ell_md_evaluate: energy needs epot and vir6");
    pd_ell *e = md->e;
    cudaStream_t s = (cudaStream_t)sp;
    int rc;
    if ((rc = ell_decide_launch(e, md->st.x, md->st.y, md->st.z, s))) return rc;
    if ((rc = ell_rebuild_launch(e, md->st.x, md->st.y, md->st.z, s))) return rc;
    if ((rc = ell_pack_launch(e, md->st.x, md->st.y, md->st.z, s))) return rc;
    EllKick kick;
    memset(&kick, 0, sizeof kick);
    return ell_pairs_launch(e, md->st.fx, md->st.fy, md->st.fz, md->st.epot, md->st.vir6, energy, kick, s);
}

int pd_ell_md_step(pd_ell_md *md, int nsteps, float dt, int energy_last, int use_graph, pd_stream_t s) {
    PD_CHECK(md, PD_EINVAL, "pd_ell_md_step: null handle");
    PD_CHECK(nsteps >= 0, PD_EINVAL, "pd_ell_md_step: negative step count");
    PD_CHECK(!energy_last || (md->st.epot && md->st.vir6), PD_EINVAL, "pd_ell_md_step: energy needs epot and vir6");
    return ell_run(md, 0, nsteps, dt, 0.f, 0.f, 0ull, energy_last, use_graph, (cudaStream_t)s);
}

int pd_ell_md_langevin(pd_ell_md *md, int nsteps, float dt, float gamma, float kT, unsigned long long seed,
                       int energy_last, int use_graph, pd_stream_t s) {
    PD_CHECK(md, PD_EINVAL, "pd_ell_md_langevin: null handle");
    PD_CHECK(nsteps >= 0, PD_EINVAL, "pd_ell_md_langevin: negative step count");
    PD_CHECK(gamma > 0.f && std::isfinite(gamma), PD_EINVAL, "Langevin friction gamma must be positive");
    PD_CHECK(kT >= 0.f && std::isfinite(kT), PD_EINVAL, "Langevin temperature must be finite and nonnegative");
    PD_CHECK(!energy_last || (md->st.epot && md->st.vir6), PD_EINVAL,
             "pd_ell_md_langevin: energy needs epot and vir6");
    return ell_run(md, 1, nsteps, dt, gamma, kT, seed, energy_last, use_graph, (cudaStream_t)s);
}

int pd_ell_md_bookkeeping(pd_ell_md *md, float *dq, float *dU, float *ekin) {
    PD_CHECK(md, PD_EINVAL, "pd_ell_md_bookkeeping: null handle");
    PD_CHECK((dq && dU && ekin) || (!dq && !dU && !ekin), PD_EINVAL,
             "pd_ell_md_bookkeeping: give all three arrays or none");
    md->dq = dq;
    md->dU = dU;
    md->ekin = ekin;
    return PD_OK;
}

int pd_ell_md_baoa(pd_ell_md *md, int nsteps, float dt, float gamma, float kT, unsigned long long seed,
                   int energy_last, int use_graph, pd_stream_t s) {
    PD_CHECK(md, PD_EINVAL, "pd_ell_md_baoa: null handle");
    PD_CHECK(nsteps >= 0, PD_EINVAL, "pd_ell_md_baoa: negative step count");
    PD_CHECK(gamma > 0.f && std::isfinite(gamma), PD_EINVAL, "Langevin friction gamma must be positive");
    PD_CHECK(kT >= 0.f && std::isfinite(kT), PD_EINVAL, "Langevin temperature must be finite and nonnegative");
    PD_CHECK(!energy_last || (md->st.epot && md->st.vir6), PD_EINVAL, "pd_ell_md_baoa: energy needs epot and vir6");
    return ell_run(md, 1, nsteps, dt, gamma, kT, seed, energy_last, use_graph, (cudaStream_t)s, 2.f * dt);
}

int pd_ell_md_gjf(pd_ell_md *md, int nsteps, float dt, float gamma, float kT, unsigned long long seed,
                  int energy_last, int use_graph, pd_stream_t s) {
    PD_CHECK(md, PD_EINVAL, "pd_ell_md_gjf: null handle");
    PD_CHECK(nsteps >= 0, PD_EINVAL, "pd_ell_md_gjf: negative step count");
    PD_CHECK(gamma > 0.f && std::isfinite(gamma), PD_EINVAL, "Langevin friction gamma must be positive");
    PD_CHECK(kT >= 0.f && std::isfinite(kT), PD_EINVAL, "Langevin temperature must be finite and nonnegative");
    PD_CHECK(!energy_last || (md->st.epot && md->st.vir6), PD_EINVAL, "pd_ell_md_gjf: energy needs epot and vir6");
    if (!md->f0) {   // host boundary: the old-force storage is allocated on first use
        int rc = dalloc(&md->f0, 3 * (size_t)md->e->n);
        if (rc) return rc;
        PD_CUDA(cudaMemset(md->f0, 0, sizeof(float) * 3 * (size_t)md->e->n));
    }
    return ell_run(md, 2, nsteps, dt, gamma, kT, seed, energy_last, use_graph, (cudaStream_t)s);
}

}  // extern "C"
