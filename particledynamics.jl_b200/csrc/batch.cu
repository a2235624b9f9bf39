// Batched replicas of libpdb200: hundreds of independent LJ / WCA systems of uneven size (their
// own box, density and pair model) stepped together, one launch per stage over all replicas,
// the whole velocity-Verlet step captured into one CUDA graph.
//
// The replicas' particles are concatenated (replica r owns [first_r, first_r + N_r)); every
// replica has its own cell grid, and the grids are concatenated too (global cell = cell_base_r +
// local cell), so the counting sort of the ELL route (scan, scatter, id order per cell) serves
// all replicas in one pass.  Per-replica geometry and pair model sit in a small device table
// read through the read-only cache.  Stages per step:
//   1. k_batch_drift: half kick, drift, centred wrap in the replica's box, per-replica
//      displacement maxima since each replica's last build; the last block flags the replicas to
//      rebuild and sets the graph's IF condition when there is one;
//   2. the rebuild (IF node): k_batch_bin (flagged replicas re-binned, the others keep their
//      cells), the shared counting sort (which leaves the others' cell order unchanged),
//      k_batch_rows for the flagged replicas' cells only (one warp per cell, the replica's
//      stencil staged in shared memory, rows identical to the single-system kernels'), the
//      capacity commit by the last block;
//   3. k_batch_pack (coordinates in cell order) and k_batch_pairs<G>: G lanes per row (G chosen by
//      the caller's autotuner), the replica's LJ or WCA model, the closing half kick fused, the
//      device step advanced.
// Rows live in cell order (slot t of the particle at position k of the cell order at t * N + k,
// entries are cell-order positions), so row stores and loads are contiguous per warp and the
// neighbours' packed records of a row sit in nearby cells.
//
// Charged replicas (the batched ionic melts) add the real-space Coulomb polynomial to the pair kernel
// and a mesh per replica (batch_mesh.cu): the step's force pass packs coordinates and charges once,
// runs the pair kernel while the mesh branch (spread, batched transforms per mesh size, influence
// multiply) runs on a second stream, and the gather joins both and applies the closing half kick.
#include <cmath>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "ell_common.cuh"
#include "internal.hpp"

#include <algorithm>
#include <numeric>
#include <tuple>

using namespace pdb;

namespace pdb {

constexpr int B_THREADS = 256;
constexpr int BROWS_WARPS = 4, BROWS_CAP = 640;

struct BatchRep {
    float L[3];
    int nx, ny, nz, cell_base;
    int kind;
    float eps, sig2, rc2, eshift;
};

__device__ __forceinline__ float wrap_centred(float x, float L) {
    x -= (x >= 0.5f * L) ? L : 0.f;
    x += (x < -0.5f * L) ? L : 0.f;
    return x;
}

// Rebuild decision per replica, taken by the whole last block of the drift kernel: replica r is
// rebuilt when one of its particles moved more than skin / 2 since its last build, and every replica
// when the list is invalid or the rebuild interval is reached.  Sets the device request (and the
// graph's IF condition) when any replica is rebuilt.
template <bool COND>
__device__ void batch_decide(long long *st, unsigned *rep_dmax, int *rep_flag, int nrep, float threshold,
                             bool thread0, cudaGraphConditionalHandle h) {
    __shared__ int any, all, bad;
    if (thread0) {
        st[E_CHECKS] += 1;
        st[E_REQUEST] = 0;
        bad = !isfinite(__uint_as_float((unsigned)st[E_DMAX]));
        all = st[E_VALID] == 0 || st[E_STEP] - st[E_LAST_BUILD] >= st[E_INTERVAL];
        any = 0;
        st[E_DMAX] = 0;
    }
    __syncthreads();
    for (int r = threadIdx.x; r < nrep; r += blockDim.x) {
        const int f = (all || __uint_as_float(rep_dmax[r]) > threshold) ? 1 : 0;
        rep_flag[r] = f;
        rep_dmax[r] = 0u;
        if (f) any = 1;   // benign race: every writer stores 1
    }
    __syncthreads();
    if (thread0) {
        if (bad) {
            st[E_ERROR] = E_ERR_COORD;
            st[E_VALID] = 0;
        } else if (any) {
            st[E_REQUEST] = 1;
            st[E_VALID] = 0;
        }
        if (COND) cudaGraphSetConditional(h, ell_requested(st) ? 1u : 0u);
    }
}

// Half kick, drift, wrap and displacement (DRIFT), or the displacement of the current coordinates
// alone; per-replica displacement maxima, the decision by the last block.
template <bool DRIFT, bool COND>
__global__ void __launch_bounds__(B_THREADS) k_batch_drift(int n, float *__restrict__ x, float *__restrict__ y,
                                                           float *__restrict__ z, float *__restrict__ vx,
                                                           float *__restrict__ vy, float *__restrict__ vz,
                                                           const float *__restrict__ fx, const float *__restrict__ fy,
                                                           const float *__restrict__ fz,
                                                           const float *__restrict__ inv_mass, float dt,
                                                           const int *__restrict__ rep_of,
                                                           const BatchRep *__restrict__ reps,
                                                           const float4 *__restrict__ ref, float threshold,
                                                           unsigned *__restrict__ rep_dmax, int *__restrict__ rep_flag,
                                                           int nrep, long long *__restrict__ st,
                                                           cudaGraphConditionalHandle h) {
    if (st[E_ERROR] != 0) {
        if (COND && blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(h, 0u);
        return;
    }
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    float v = 0.f;
    int r = -1;
    if (i < n) {
        r = __ldg(rep_of + i);
        const BatchRep &R = reps[r];
        const float L[3] = {R.L[0], R.L[1], R.L[2]};
        float p[3] = {x[i], y[i], z[i]};
        if (DRIFT) {
            const float c = 0.5f * dt * inv_mass[i];
            const float u[3] = {fmaf(c, fx[i], vx[i]), fmaf(c, fy[i], vy[i]), fmaf(c, fz[i], vz[i])};
            vx[i] = u[0];
            vy[i] = u[1];
            vz[i] = u[2];
#pragma unroll
            for (int d = 0; d < 3; ++d) p[d] = wrap_centred(fmaf(dt, u[d], p[d]), L[d]);
            x[i] = p[0];
            y[i] = p[1];
            z[i] = p[2];
        }
        v = ell_displacement<3>(p, ref[i], L, st[E_VALID] != 0);
    }
    // per-replica maximum: one atomic per warp where the warp's particles share a replica
    const unsigned bits = __float_as_uint(v);
    const int r0 = __shfl_sync(0xffffffffu, r, 0);
    if (__all_sync(0xffffffffu, r == r0)) {
        const unsigned m = __reduce_max_sync(0xffffffffu, bits);
        if ((threadIdx.x & 31) == 0 && r0 >= 0) atomicMax(rep_dmax + r0, m);
    } else if (r >= 0) {
        atomicMax(rep_dmax + r, bits);
    }
    __threadfence();   // the per-replica maxima are visible before this block's ticket
    __shared__ bool last_block;
    const bool t0last = ell_block_max_last(bits, st, E_DMAX, E_TICKET_D);
    if (threadIdx.x == 0) last_block = t0last;
    __syncthreads();
    if (last_block) {
        __threadfence();
        if (threadIdx.x == 0) st[E_TICKET_D] = 0;
        batch_decide<COND>(st, rep_dmax, rep_flag, nrep, threshold, threadIdx.x == 0, h);
    }
}

// Global cell of every particle (its replica's grid) and the cell histogram.
// Particles of replicas that are not rebuilt keep their cells, so that their cell-order positions,
// and with them their rows, stay valid through the counting sort.
__global__ void k_batch_bin(const float *__restrict__ x, const float *__restrict__ y, const float *__restrict__ z,
                            int n, const int *__restrict__ rep_of, const BatchRep *__restrict__ reps,
                            const int *__restrict__ rep_flag, int *__restrict__ cell_of, int *__restrict__ cell_count,
                            const long long *__restrict__ st) {
    if (!ell_requested(st)) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int r = __ldg(rep_of + i);
    if (!rep_flag[r]) {
        atomicAdd(&cell_count[cell_of[i]], 1);
        return;
    }
    const BatchRep &R = reps[r];
    const float p[3] = {x[i], y[i], z[i]};
    const int ng[3] = {R.nx, R.ny, R.nz};
    int cc[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        float u = p[d] + 0.5f * R.L[d];
        u -= floorf(u / R.L[d]) * R.L[d];
        cc[d] = min(max((int)floorf(u * ((float)ng[d] / R.L[d])), 0), ng[d] - 1);
    }
    const int c = R.cell_base + (cc[2] * R.ny + cc[1]) * R.nx + cc[0];
    cell_of[i] = c;
    atomicAdd(&cell_count[c], 1);
}

// Rows, one warp per global cell: the replica's stencil (same visiting order as the single-system
// row kernels) staged in shared memory once per cell, each lane taking up to M particles of the cell
// (lane, lane + 32, ...), so a cell of up to 32 M particles stages its candidates once.
// The candidates come from the packed coordinates in cell order (xq, packed after the sort of this
// rebuild), so a stencil row's candidates are one contiguous, coalesced float4 run.  Rows, their
// lengths and their entries are in cell order (positions in `sorted`), so the row stores of a warp and
// the pair kernel's row loads are contiguous and neighbours' packed records sit close together; a
// particle's entries are appended in the candidates' visiting order, as in the single-system kernels.
template <int M>   // particles per lane (1, 2 or 4), from the batch's mean cell occupancy
__global__ void __launch_bounds__(32 * BROWS_WARPS) k_batch_rows(
    const float4 *__restrict__ xq, int n, int ncell, const int *__restrict__ cell_rep,
    const BatchRep *__restrict__ reps, const int *__restrict__ rep_flag, const int *__restrict__ sorted,
    const int *__restrict__ cell_off, float rl2, int cap, int *__restrict__ rows, int *__restrict__ counts,
    float4 *__restrict__ ref, long long *__restrict__ st) {
    if (!ell_requested(st)) return;
    extern __shared__ float4 batch_stage[];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int c = blockIdx.x * BROWS_WARPS + w;
    float4 *sw = batch_stage + w * BROWS_CAP;
    unsigned fmax = 0;
    if (c < ncell && rep_flag[__ldg(cell_rep + c)]) {   // warp-uniform; only replicas being rebuilt
        const BatchRep &R = reps[__ldg(cell_rep + c)];
        const float Lx = R.L[0], Ly = R.L[1], Lz = R.L[2];
        const int nx = R.nx, ny = R.ny, nz = R.nz, base = R.cell_base;
        const float hLx = 0.5f * Lx, hLy = 0.5f * Ly, hLz = 0.5f * Lz;
        const float rl = sqrtf(rl2);
        const float hx = Lx / (float)nx, hy = Ly / (float)ny, hz = Lz / (float)nz;
        const int Sx = ell_reach(rl, Lx, nx), Sy = ell_reach(rl, Ly, ny), Sz = ell_reach(rl, Lz, nz);
        const int lc = c - base;
        const int cx = lc % nx, tmp = lc / nx, cy = tmp % ny, cz = tmp / ny;
        const int p0 = cell_off[c], pn = cell_off[c + 1] - p0;
        for (int pg = 0; pg < pn; pg += 32 * M) {
            int kp[M], found[M];
            bool has[M];
            float xi[M], yi[M], zi[M];
#pragma unroll
            for (int m = 0; m < M; ++m) {
                has[m] = pg + lane + 32 * m < pn;
                kp[m] = p0 + pg + lane + 32 * m;   // this lane's m-th particle: its position in cell order
                const float4 v = has[m] ? xq[kp[m]] : make_float4(0.f, 0.f, 0.f, 0.f);
                xi[m] = v.x;
                yi[m] = v.y;
                zi[m] = v.z;
                found[m] = 0;
            }
            // bounding box of this group's particles: a candidate farther than the list radius from the
            // box is farther from every particle of the group, so it is not staged (a conservative
            // margin keeps rounding from dropping a candidate that the exact test would accept)
            float blo[3] = {INFINITY, INFINITY, INFINITY}, bhi[3] = {-INFINITY, -INFINITY, -INFINITY};
#pragma unroll
            for (int m = 0; m < M; ++m) {
                if (!has[m]) continue;
                blo[0] = fminf(blo[0], xi[m]);
                blo[1] = fminf(blo[1], yi[m]);
                blo[2] = fminf(blo[2], zi[m]);
                bhi[0] = fmaxf(bhi[0], xi[m]);
                bhi[1] = fmaxf(bhi[1], yi[m]);
                bhi[2] = fmaxf(bhi[2], zi[m]);
            }
#pragma unroll
            for (int d = 0; d < 3; ++d) {
#pragma unroll
                for (int off = 16; off > 0; off >>= 1) {
                    blo[d] = fminf(blo[d], __shfl_xor_sync(0xffffffffu, blo[d], off));
                    bhi[d] = fmaxf(bhi[d], __shfl_xor_sync(0xffffffffu, bhi[d], off));
                }
            }
            const float bcx = 0.5f * (blo[0] + bhi[0]), bcy = 0.5f * (blo[1] + bhi[1]), bcz = 0.5f * (blo[2] + bhi[2]);
            const float bhx = 0.5f * (bhi[0] - blo[0]), bhy = 0.5f * (bhi[1] - blo[1]), bhz = 0.5f * (bhi[2] - blo[2]);
            const float rbox = rl * 1.0001f + 1e-3f;
            const float rbox2 = rbox * rbox;
            int fill = 0;
            // scan of the staged candidates by every particle of the lane (one body, expanded where a
            // full stage buffer is flushed and at the end, so the per-particle counters stay in registers)
#define PD_BATCH_ROWS_SCAN                                                            \
    do {                                                                              \
        __syncwarp();                                                                 \
        for (int t = 0; t < fill; ++t) {                                              \
            const float4 cj = sw[t];                                                  \
            const int kc = __float_as_int(cj.w);                                      \
            _Pragma("unroll") for (int m = 0; m < M; ++m) {                           \
                if (!has[m] || kc == kp[m]) continue;                                 \
                const float dx = mic_fast(cj.x - xi[m], hLx, Lx);                     \
                const float dy = mic_fast(cj.y - yi[m], hLy, Ly);                     \
                const float dz = mic_fast(cj.z - zi[m], hLz, Lz);                     \
                const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));                 \
                if (r2 <= rl2) {                                                      \
                    if (found[m] < cap) rows[(size_t)found[m] * n + kp[m]] = kc;      \
                    ++found[m];                                                       \
                }                                                                     \
            }                                                                         \
        }                                                                             \
        __syncwarp();                                                                 \
        fill = 0;                                                                     \
    } while (0)
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
                    const int row = base + (cz2 * ny + cy2) * nx;
                    int a1, b1, a2, b2;
                    ell_row_ranges(cx, g2, rl2, hx, Sx, nx, a1, b1, a2, b2);
                    for (int part = 0; part < 2; ++part) {
                        if (part == 1 && a2 > b2) break;
                        const int ka = cell_off[row + (part ? a2 : a1)], kb = cell_off[row + (part ? b2 : b1) + 1];
                        for (int k0 = ka; k0 < kb; k0 += 32) {
                            const bool in = lane < kb - k0;
                            float4 v = in ? xq[k0 + lane] : make_float4(0.f, 0.f, 0.f, 0.f);
                            const float ex = fmaxf(fabsf(mic_fast(v.x - bcx, hLx, Lx)) - bhx, 0.f);
                            const float ey = fmaxf(fabsf(mic_fast(v.y - bcy, hLy, Ly)) - bhy, 0.f);
                            const float ez = fmaxf(fabsf(mic_fast(v.z - bcz, hLz, Lz)) - bhz, 0.f);
                            const bool keep = in && fmaf(ex, ex, fmaf(ey, ey, ez * ez)) <= rbox2;
                            const unsigned bal = __ballot_sync(0xffffffffu, keep);
                            const int nk = __popc(bal);
                            if (fill + nk > BROWS_CAP) PD_BATCH_ROWS_SCAN;
                            if (keep) {   // staged in the candidates' order
                                v.w = __int_as_float(k0 + lane);
                                sw[fill + __popc(bal & ((1u << lane) - 1u))] = v;
                            }
                            fill += nk;
                        }
                    }
                }
            }
            PD_BATCH_ROWS_SCAN;
#undef PD_BATCH_ROWS_SCAN
#pragma unroll
            for (int m = 0; m < M; ++m) {
                if (has[m]) {
                    counts[kp[m]] = found[m];
                    ref[sorted[kp[m]]] = make_float4(xi[m], yi[m], zi[m], 0.f);
                }
                fmax = max(fmax, (unsigned)found[m]);
            }
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

// Packed coordinates (and charges, when q is given) in cell order: xq[k] = (x, y, z, q) of particle
// sorted[k].  REBUILD: the pack that feeds the row build of a rebuild (runs while the rows are being
// rebuilt); otherwise the pack of the pair pass (skipped while the rows are invalid).
template <bool REBUILD>
__global__ void k_batch_pack(const float *__restrict__ x, const float *__restrict__ y, const float *__restrict__ z,
                             const float *__restrict__ q, const int *__restrict__ sorted, int n,
                             float4 *__restrict__ xq, const long long *__restrict__ st) {
    if (REBUILD ? !ell_requested(st) : st[E_VALID] == 0) return;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int i = sorted[k];
    xq[k] = make_float4(x[i], y[i], z[i], q ? q[i] : 0.f);
}

struct BatchKick {
    float *vx, *vy, *vz;
    const float *inv_mass;
    float half_dt;
    int on;
};

// Real-space Coulomb of charged replicas, shared by every replica (one split and cutoff): the
// cluster route's fitted polynomial (pair_force, PairFunctor.jl:127-156), f/r = C qq (r^-3 - P_f(x)),
// e = C qq (1/r + P_e(x) - eshift), x = r^2 sx - 1, inside rc2.  Monomial coefficients, constant term
// first, zero above the fitted degree.
constexpr int BATCH_NP = 16;
struct BatchCoul {
    float C, rc2, sx, eshift;
    float pf[BATCH_NP], pe[BATCH_NP];
};

// Row pair kernel over all replicas: the model of particle i's replica (LJ or WCA, the ELL route's
// UniformLJ / UniformWCA arithmetic), forces stored, optional energy (half of each pair), the
// closing half kick fused.  The packed coordinates are refreshed by the pack of the same stage.
// COUL: the packed records carry the charges (xq.w) and the pair adds the Coulomb polynomial term,
// evaluated with NP coefficients (the fitted ones, zeros above them); one reciprocal square root
// serves both terms.
template <int G, bool ENERGY, bool COUL, int NP = BATCH_NP>
__global__ void __launch_bounds__(B_THREADS) k_batch_pairs(const float4 *__restrict__ xq, int n,
                                                           const int *__restrict__ rows,
                                                           const int *__restrict__ counts,
                                                           const int *__restrict__ sorted,
                                                           const int *__restrict__ rep_of,
                                                           const BatchRep *__restrict__ reps, float *__restrict__ fx,
                                                           float *__restrict__ fy, float *__restrict__ fz,
                                                           float *__restrict__ epot, BatchKick kick,
                                                           long long *__restrict__ st, int advance,
                                                           const __grid_constant__ BatchCoul cp) {
    if (st[E_VALID] == 0) return;
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    const int k = tid / G, lane = tid % G;   // position in cell order
    const int i = k < n ? sorted[k] : -1;
    float a[3] = {0.f, 0.f, 0.f}, e = 0.f;
    if (k < n) {
        const BatchRep &R = reps[__ldg(rep_of + i)];
        const float Lx = R.L[0], Ly = R.L[1], Lz = R.L[2];
        const float hLx = 0.5f * Lx, hLy = 0.5f * Ly, hLz = 0.5f * Lz;
        const float eps = R.eps, sig2 = R.sig2, rc2 = R.rc2;
        const float eoff = R.kind == PD_PAIR_WCA ? R.eps : -R.eshift;
        const float4 pi = xq[k];
        const int cnt = counts[k];
        const float cqi = COUL ? cp.C * pi.w : 0.f;
        const float cut2 = COUL ? fmaxf(rc2, cp.rc2) : rc2;
        auto pair = [&](float4 pj) {
            const float dx = periodic_delta(pi.x, pj.x, hLx, Lx);
            const float dy = periodic_delta(pi.y, pj.y, hLy, Ly);
            const float dz = periodic_delta(pi.z, pj.z, hLz, Lz);
            const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
            if (COUL) {
                if (!(r2 > 0.f && r2 < cut2)) return;
                const float rinv = rsqrtf(r2);
                const float ir2 = rinv * rinv;
                float fr = 0.f;
                if (r2 < rc2) {
                    const float s2 = sig2 * ir2;
                    const float s6 = s2 * s2 * s2;
                    const float s12 = s6 * s6;
                    fr = 24.f * eps * (2.f * s12 - s6) * ir2;
                    if (ENERGY) e += 0.5f * (4.f * eps * (s12 - s6) + eoff);
                }
                if (r2 < cp.rc2) {
                    const float x = fmaf(r2, cp.sx, -1.f);
                    float pf = cp.pf[NP - 1];
#pragma unroll
                    for (int t = NP - 2; t >= 0; --t) pf = fmaf(pf, x, cp.pf[t]);
                    const float cq = cqi * pj.w;
                    fr = fmaf(cq, rinv * ir2 - pf, fr);
                    if (ENERGY) {
                        float pe = cp.pe[NP - 1];
#pragma unroll
                        for (int t = NP - 2; t >= 0; --t) pe = fmaf(pe, x, cp.pe[t]);
                        e = fmaf(0.5f * cq, rinv + pe - cp.eshift, e);
                    }
                }
                a[0] = fmaf(fr, dx, a[0]);
                a[1] = fmaf(fr, dy, a[1]);
                a[2] = fmaf(fr, dz, a[2]);
                return;
            }
            if (r2 > 0.f && r2 < rc2) {
                const float ir2 = 1.f / r2;
                const float s2 = sig2 * ir2;
                const float s6 = s2 * s2 * s2;
                const float s12 = s6 * s6;
                const float fr = 24.f * eps * (2.f * s12 - s6) * ir2;
                a[0] += fr * dx;
                a[1] += fr * dy;
                a[2] += fr * dz;
                if (ENERGY) e += 0.5f * (4.f * eps * (s12 - s6) + eoff);
            }
        };
        int slot = lane;
        for (; slot + G < cnt; slot += 2 * G) {
            const float4 p1 = xq[rows[(size_t)slot * n + k]];
            const float4 p2 = xq[rows[(size_t)(slot + G) * n + k]];
            pair(p1);
            pair(p2);
        }
        for (; slot < cnt; slot += G) pair(xq[rows[(size_t)slot * n + k]]);
    }
#pragma unroll
    for (int off = G / 2; off > 0; off >>= 1) {
#pragma unroll
        for (int d = 0; d < 3; ++d) a[d] += __shfl_down_sync(0xffffffffu, a[d], off, G);
        if (ENERGY) e += __shfl_down_sync(0xffffffffu, e, off, G);
    }
    if (lane == 0 && k < n) {
        fx[i] = a[0];
        fy[i] = a[1];
        fz[i] = a[2];
        if (ENERGY) epot[i] = e;
        if (kick.on) {
            const float c = kick.half_dt * kick.inv_mass[i];
            kick.vx[i] = fmaf(c, a[0], kick.vx[i]);
            kick.vy[i] = fmaf(c, a[1], kick.vy[i]);
            kick.vz[i] = fmaf(c, a[2], kick.vz[i]);
        }
    }
    if (advance && blockIdx.x == 0 && threadIdx.x == 0) st[E_STEP] += 1;
}

}  // namespace pdb

struct pd_batch {
    int nrep = 0, n = 0, ncell = 0, cap = 0, lanes = 4;
    float rl2 = 0.f, threshold = 0.f;
    std::vector<BatchRep> hreps;
    std::vector<int> first;
    BatchRep *reps = nullptr;
    int *rep_of = nullptr, *cell_rep = nullptr;
    int *rep_flag = nullptr;         // replicas rebuilt by the current decision
    unsigned *rep_dmax = nullptr;    // per-replica displacement maxima (float bits)
    long long *st = nullptr;
    int *cell_of = nullptr, *cell_count = nullptr, *cell_off = nullptr, *sorted = nullptr, *tmp = nullptr;
    int *rows = nullptr, *counts = nullptr;
    float4 *ref = nullptr, *xq = nullptr;
    // bound state (pd_batch_bind)
    pd_md_state state;
    bool bound = false;
    cudaStream_t body = nullptr;
    bool cond_nodes = true;
    cudaGraphExec_t exec = nullptr;
    float exec_dt = 0.f;
    int exec_lanes = 0;
    cudaStream_t exec_stream = nullptr;
    int exec_chunk = 0;
    std::vector<double> box;          // 3 per replica, as given
    // charged replicas: real-space Coulomb and the batched meshes
    bool coul = false;
    BatchCoul cp{};
    int coul_ne = 0, coul_nf = 0;
    float half_c_self = 0.f;
    bool mesh = false;
    int morder = 5, mchunk = 64, nchunk = 0, mtpi = 2;
    std::vector<BMeshRep> hmreps;
    BMeshRep *mreps = nullptr;
    int *chunk_rep = nullptr, *slot_src = nullptr, *mid = nullptr;
    float4 *mq = nullptr;
    float *gridA = nullptr, *gridB = nullptr, *G = nullptr;
    float2 *spec = nullptr;
    long long total_nodes = 0, total_modes = 0;
    struct FftGroup {
        int K1, K2, K3, count;
        long long grid, modes;
        cufftHandle fwd, bwd;
    };
    std::vector<FftGroup> groups;
    // the mesh sizes' transforms run on NFFT streams at once, group g on stream g % NFFT with that
    // stream's own cuFFT work area
    static constexpr int NFFT = 4;
    void *fft_work[NFFT] = {};
    cudaStream_t fft_stream[NFFT] = {};
    cudaEvent_t ev_fft[NFFT] = {};
    cudaEvent_t ev_fft_fork = nullptr;
    cudaStream_t mesh_stream = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
};

namespace pdb {

static void batch_free_chunks(pd_batch *b) {
    dfree(b->chunk_rep);
    dfree(b->slot_src);
    dfree(b->mid);
    dfree(b->mq);
    b->nchunk = 0;
}

static void batch_free_mesh(pd_batch *b) {
    for (auto &g : b->groups) {
        if (g.fwd) cufftDestroy(g.fwd);
        if (g.bwd) cufftDestroy(g.bwd);
    }
    b->groups.clear();
    batch_free_chunks(b);
    dfree(b->mreps);
    dfree(b->gridA);
    dfree(b->gridB);
    dfree(b->G);
    dfree(b->spec);
    for (int k = 0; k < pd_batch::NFFT; ++k) {
        if (b->fft_work[k]) cudaFree(b->fft_work[k]);
        if (b->fft_stream[k]) cudaStreamDestroy(b->fft_stream[k]);
        if (b->ev_fft[k]) cudaEventDestroy(b->ev_fft[k]);
        b->fft_work[k] = nullptr;
        b->fft_stream[k] = nullptr;
        b->ev_fft[k] = nullptr;
    }
    if (b->ev_fft_fork) cudaEventDestroy(b->ev_fft_fork);
    b->ev_fft_fork = nullptr;
    if (b->mesh_stream) cudaStreamDestroy(b->mesh_stream);
    if (b->ev_fork) cudaEventDestroy(b->ev_fork);
    if (b->ev_join) cudaEventDestroy(b->ev_join);
    b->mesh_stream = nullptr;
    b->ev_fork = b->ev_join = nullptr;
    b->mesh = false;
}

static void batch_free(pd_batch *b) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    b->exec = nullptr;
    batch_free_mesh(b);
    if (b->body) cudaStreamDestroy(b->body);
    b->body = nullptr;
    dfree(b->reps);
    dfree(b->rep_of);
    dfree(b->cell_rep);
    dfree(b->rep_flag);
    dfree(b->rep_dmax);
    dfree(b->st);
    dfree(b->cell_of);
    dfree(b->cell_count);
    dfree(b->cell_off);
    dfree(b->sorted);
    dfree(b->tmp);
    dfree(b->rows);
    dfree(b->counts);
    dfree(b->ref);
    dfree(b->xq);
}

static int batch_rebuild_launch(pd_batch *b, const float *x, const float *y, const float *z, cudaStream_t s) {
    const int blocks = (b->n + B_THREADS - 1) / B_THREADS;
    k_batch_bin<<<blocks, B_THREADS, 0, s>>>(x, y, z, b->n, b->rep_of, b->reps, b->rep_flag, b->cell_of,
                                             b->cell_count, b->st);
    PD_LAUNCHED();
    int rc;
    if ((rc = ell_sort_cells_launch(b->cell_of, b->n, b->ncell, b->cell_count, b->cell_off, b->sorted, b->tmp, b->st,
                                    s)))
        return rc;
    k_batch_pack<true><<<(b->n + B_THREADS - 1) / B_THREADS, B_THREADS, 0, s>>>(x, y, z, nullptr, b->sorted, b->n,
                                                                                b->xq, b->st);
    PD_LAUNCHED();
    // particles per lane: enough lanes for a cell of 1.3x the mean occupancy
    const double occ = 1.3 * (double)b->n / (double)std::max(b->ncell, 1);
    const dim3 grid((b->ncell + BROWS_WARPS - 1) / BROWS_WARPS), block(32 * BROWS_WARPS);
    const size_t shm = sizeof(float4) * BROWS_WARPS * BROWS_CAP;
    if (occ <= 32.0)
        k_batch_rows<1><<<grid, block, shm, s>>>(b->xq, b->n, b->ncell, b->cell_rep, b->reps, b->rep_flag, b->sorted,
                                                 b->cell_off, b->rl2, b->cap, b->rows, b->counts, b->ref, b->st);
    else if (occ <= 64.0)
        k_batch_rows<2><<<grid, block, shm, s>>>(b->xq, b->n, b->ncell, b->cell_rep, b->reps, b->rep_flag, b->sorted,
                                                 b->cell_off, b->rl2, b->cap, b->rows, b->counts, b->ref, b->st);
    else
        k_batch_rows<4><<<grid, block, shm, s>>>(b->xq, b->n, b->ncell, b->cell_rep, b->reps, b->rep_flag, b->sorted,
                                                 b->cell_off, b->rl2, b->cap, b->rows, b->counts, b->ref, b->st);
    PD_LAUNCHED();
    return PD_OK;
}

template <bool COUL, int NP = BATCH_NP>
static void launch_batch_pairs(pd_batch *b, float *fx, float *fy, float *fz, float *epot, int energy,
                               const BatchKick &kick, int advance, cudaStream_t s) {
    const int G = b->lanes;
    const int blocks = (int)(((long long)b->n * G + B_THREADS - 1) / B_THREADS);
#define PD_BP(GG)                                                                                                      \
    if (energy)                                                                                                        \
        k_batch_pairs<GG, true, COUL, NP><<<blocks, B_THREADS, 0, s>>>(b->xq, b->n, b->rows, b->counts, b->sorted,   \
                                                                        b->rep_of, b->reps, fx, fy, fz, epot, kick,    \
                                                                        b->st, advance, b->cp);                        \
    else                                                                                                               \
        k_batch_pairs<GG, false, COUL, NP><<<blocks, B_THREADS, 0, s>>>(b->xq, b->n, b->rows, b->counts, b->sorted,  \
                                                                         b->rep_of, b->reps, fx, fy, fz, epot, kick,   \
                                                                         b->st, advance, b->cp);
    switch (G) {
        case 1: PD_BP(1) break;
        case 2: PD_BP(2) break;
        case 4: PD_BP(4) break;
        default: PD_BP(8) break;
    }
#undef PD_BP
}

static BMeshView batch_mesh_view(const pd_batch *b) {
    BMeshView v;
    v.order = b->morder;
    v.chunk = b->mchunk;
    v.tpi = b->mtpi;
    v.nchunk = b->nchunk;
    v.nrep = b->nrep;
    v.reps = b->mreps;
    v.chunk_rep = b->chunk_rep;
    v.slot_src = b->slot_src;
    v.mq = b->mq;
    v.mid = b->mid;
    v.gridA = b->gridA;
    v.gridB = b->gridB;
    v.spec = b->spec;
    v.G = b->G;
    v.total_nodes = b->total_nodes;
    v.total_modes = b->total_modes;
    return v;
}

// The mesh branch of charged replicas: spread, the batched forward transforms (one per mesh size),
// the influence multiply, the batched inverse transforms.
// Transforms of every mesh size, forked from s onto the FFT streams and joined back into s.
static int batch_fft_all(pd_batch *b, bool forward, cudaStream_t s) {
    const int ns = std::min<int>(pd_batch::NFFT, (int)b->groups.size());
    PD_CUDA(cudaEventRecord(b->ev_fft_fork, s));
    for (int k = 0; k < ns; ++k) PD_CUDA(cudaStreamWaitEvent(b->fft_stream[k], b->ev_fft_fork, 0));
    for (size_t gi = 0; gi < b->groups.size(); ++gi) {
        auto &g = b->groups[gi];
        cudaStream_t fs = b->fft_stream[gi % pd_batch::NFFT];
        if (forward) {
            PD_CHECK(cufftSetStream(g.fwd, fs) == CUFFT_SUCCESS, PD_ECUFFT, "batched mesh: cufftSetStream failed");
            PD_CHECK(cufftExecR2C(g.fwd, b->gridA + g.grid, reinterpret_cast<cufftComplex *>(b->spec + g.modes)) ==
                         CUFFT_SUCCESS,
                     PD_ECUFFT, "batched mesh: forward transform failed");
        } else {
            PD_CHECK(cufftSetStream(g.bwd, fs) == CUFFT_SUCCESS, PD_ECUFFT, "batched mesh: cufftSetStream failed");
            PD_CHECK(cufftExecC2R(g.bwd, reinterpret_cast<cufftComplex *>(b->spec + g.modes), b->gridB + g.grid) ==
                         CUFFT_SUCCESS,
                     PD_ECUFFT, "batched mesh: inverse transform failed");
        }
    }
    for (int k = 0; k < ns; ++k) {
        PD_CUDA(cudaEventRecord(b->ev_fft[k], b->fft_stream[k]));
        PD_CUDA(cudaStreamWaitEvent(s, b->ev_fft[k], 0));
    }
    return PD_OK;
}

static int batch_mesh_transform(pd_batch *b, cudaStream_t s) {
    const BMeshView v = batch_mesh_view(b);
    int rc;
    if ((rc = bmesh_spread_launch(v, b->st, s))) return rc;
    if ((rc = batch_fft_all(b, true, s))) return rc;
    if ((rc = bmesh_solve_launch(v, b->st, s))) return rc;
    return batch_fft_all(b, false, s);
}

// The force pass: pack, then the row pair kernel; with charges and meshes the pair kernel runs on s
// while the mesh branch runs on the batch's mesh stream (forked and joined by events, so the same
// code is captured into the step graph), and the gather joins both and applies the closing kick.
static int batch_pairs_launch(pd_batch *b, const float *x, const float *y, const float *z, float *fx, float *fy,
                              float *fz, float *epot, int energy, BatchKick kick, int advance, cudaStream_t s) {
    if (!b->coul) {
        k_batch_pack<false><<<(b->n + B_THREADS - 1) / B_THREADS, B_THREADS, 0, s>>>(x, y, z, nullptr, b->sorted, b->n,
                                                                                     b->xq, b->st);
        PD_LAUNCHED();
        launch_batch_pairs<false>(b, fx, fy, fz, epot, energy, kick, advance, s);
        PD_LAUNCHED();
        return PD_OK;
    }
    PD_CHECK(b->mesh && b->bound && b->state.q, PD_ESTATE,
             "charged replicas need their meshes (pd_batch_set_mesh) and a bound state with charges");
    const BMeshView v = batch_mesh_view(b);
    int rc;
    if ((rc = bmesh_pack_launch(v, x, y, z, b->state.q, b->sorted, b->xq, b->st, s))) return rc;
    PD_CUDA(cudaEventRecord(b->ev_fork, s));
    PD_CUDA(cudaStreamWaitEvent(b->mesh_stream, b->ev_fork, 0));
    if ((rc = batch_mesh_transform(b, b->mesh_stream))) return rc;
    PD_CUDA(cudaEventRecord(b->ev_join, b->mesh_stream));
    BatchKick nokick = kick;
    nokick.on = 0;
    // the polynomial's coefficient bucket: the fitted force coefficients, and the energy's with energy
    if (std::max(b->coul_nf, energy ? b->coul_ne : 0) <= 14)
        launch_batch_pairs<true, 14>(b, fx, fy, fz, epot, energy, nokick, advance, s);
    else
        launch_batch_pairs<true, BATCH_NP>(b, fx, fy, fz, epot, energy, nokick, advance, s);
    PD_LAUNCHED();
    PD_CUDA(cudaStreamWaitEvent(s, b->ev_join, 0));
    BMeshKick mk;
    mk.vx = kick.vx;
    mk.vy = kick.vy;
    mk.vz = kick.vz;
    mk.inv_mass = kick.inv_mass;
    mk.half_dt = kick.half_dt;
    mk.on = kick.on;
    return bmesh_gather_launch(v, fx, fy, fz, epot, energy, mk, b->half_c_self, b->st, s);
}

static int batch_enqueue_step(pd_batch *b, float dt, cudaStream_t s, int cond) {
    const pd_md_state &S = b->state;
    const int blocks = (b->n + B_THREADS - 1) / B_THREADS;
    cudaGraphConditionalHandle h = 0;
    if (cond) {
        cudaStreamCaptureStatus status;
        cudaGraph_t g = nullptr;
        PD_CUDA(cudaStreamGetCaptureInfo(s, &status, nullptr, &g, nullptr, nullptr));
        PD_CUDA(cudaGraphConditionalHandleCreate(&h, g, 0, cudaGraphCondAssignDefault));
        k_batch_drift<true, true><<<blocks, B_THREADS, 0, s>>>(b->n, S.x, S.y, S.z, S.vx, S.vy, S.vz, S.fx, S.fy, S.fz,
                                                               S.inv_mass, dt, b->rep_of, b->reps, b->ref,
                                                               b->threshold, b->rep_dmax, b->rep_flag, b->nrep,
                                                               b->st, h);
    } else {
        k_batch_drift<true, false><<<blocks, B_THREADS, 0, s>>>(b->n, S.x, S.y, S.z, S.vx, S.vy, S.vz, S.fx, S.fy,
                                                                S.fz, S.inv_mass, dt, b->rep_of, b->reps, b->ref,
                                                                b->threshold, b->rep_dmax, b->rep_flag, b->nrep,
                                                                b->st, 0);
    }
    PD_LAUNCHED();
    int rc;
    if (cond) {
        if ((rc = capture_if_body(s, b->body, h, [&](cudaStream_t cs) {
                 return batch_rebuild_launch(b, S.x, S.y, S.z, cs);
             })))
            return rc;
    } else if ((rc = batch_rebuild_launch(b, S.x, S.y, S.z, s))) {
        return rc;
    }
    BatchKick kick;
    kick.vx = S.vx;
    kick.vy = S.vy;
    kick.vz = S.vz;
    kick.inv_mass = S.inv_mass;
    kick.half_dt = 0.5f * dt;
    kick.on = 1;
    return batch_pairs_launch(b, S.x, S.y, S.z, S.fx, S.fy, S.fz, S.epot, 0, kick, 1, s);
}

}  // namespace pdb

extern "C" {

int pd_batch_create(pd_batch **out, const pd_batch_replica *reps, int nrep, float skin, int cap, int lanes) {
    PD_CHECK(out && reps && nrep > 0, PD_EINVAL, "pd_batch_create: bad argument");
    PD_CHECK(cap > 0, PD_EINVAL, "pd_batch_create: row capacity must be positive");
    PD_CHECK(lanes == 1 || lanes == 2 || lanes == 4 || lanes == 8, PD_EINVAL, "pd_batch_create: lanes 1, 2, 4 or 8");
    PD_CHECK(std::isfinite(skin) && skin >= 0.f, PD_EINVAL, "pd_batch_create: skin must be finite and nonnegative");
    *out = nullptr;
    float rmax = 0.f;
    for (int r = 0; r < nrep; ++r) {
        const pd_batch_replica &R = reps[r];
        PD_CHECK(R.n > 0, PD_EINVAL, "pd_batch_create: replica %d is empty", r);
        PD_CHECK(R.kind == PD_PAIR_LJ || R.kind == PD_PAIR_WCA, PD_EINVAL, "pd_batch_create: replica %d pair model", r);
        PD_CHECK(R.rc2 > 0.f && R.eps >= 0.f && R.sigma > 0.f, PD_EINVAL, "pd_batch_create: replica %d parameters", r);
        rmax = fmaxf(rmax, sqrtf(R.rc2));
    }
    const float rl = rmax + skin;
    pd_batch *b = new pd_batch();
    b->nrep = nrep;
    b->cap = cap;
    b->lanes = lanes;
    b->rl2 = rl * rl;
    b->threshold = 0.25f * skin * skin;
    std::vector<int> rep_of, cell_rep;
    for (int r = 0; r < nrep; ++r) {
        const pd_batch_replica &R = reps[r];
        BatchRep h;
        memset(&h, 0, sizeof h);
        int ng[3];
        for (int d = 0; d < 3; ++d) {
            if (!(std::isfinite(R.box[d]) && R.box[d] > 2.0 * rl)) {
                delete b;
                set_error("pd_batch_create: replica %d box length %g is not above twice the list radius %g", r,
                          R.box[d], 2.0 * rl);
                return PD_EINVAL;
            }
            h.L[d] = (float)R.box[d];
            // cells at least r_list wide; at least three per dimension (then the stencil spans the box)
            ng[d] = std::max(3, (int)std::floor(h.L[d] / rl));
        }
        h.nx = ng[0];
        h.ny = ng[1];
        h.nz = ng[2];
        h.cell_base = b->ncell;
        h.kind = R.kind;
        h.eps = R.eps;
        h.sig2 = R.sigma * R.sigma;
        h.rc2 = R.rc2;
        h.eshift = R.eshift;
        b->hreps.push_back(h);
        b->box.insert(b->box.end(), R.box, R.box + 3);
        b->first.push_back(b->n);
        b->n += R.n;
        const int nc = ng[0] * ng[1] * ng[2];
        b->ncell += nc;
        rep_of.insert(rep_of.end(), R.n, r);
        cell_rep.insert(cell_rep.end(), nc, r);
    }
    int rc;
    const size_t n = (size_t)b->n;
    if ((rc = dalloc(&b->reps, (size_t)nrep)) || (rc = dalloc(&b->rep_of, n)) ||
        (rc = dalloc(&b->cell_rep, (size_t)b->ncell)) || (rc = dalloc(&b->st, (size_t)E_LEN)) ||
        (rc = dalloc(&b->rep_flag, (size_t)nrep)) || (rc = dalloc(&b->rep_dmax, (size_t)nrep)) ||
        (rc = dalloc(&b->cell_of, n)) || (rc = dalloc(&b->cell_count, (size_t)b->ncell)) ||
        (rc = dalloc(&b->cell_off, (size_t)b->ncell + 1)) || (rc = dalloc(&b->sorted, n)) ||
        (rc = dalloc(&b->tmp, n)) || (rc = dalloc(&b->rows, n * (size_t)cap)) || (rc = dalloc(&b->counts, n)) ||
        (rc = dalloc(&b->ref, n)) || (rc = dalloc(&b->xq, n))) {
        batch_free(b);
        delete b;
        return rc;
    }
    long long init[E_LEN] = {0};
    init[E_INTERVAL] = 100;
    std::vector<int> iota(n);
    for (size_t k = 0; k < n; ++k) iota[k] = (int)k;   // a valid cell order before the first build
    if (cudaMemcpy(b->reps, b->hreps.data(), sizeof(BatchRep) * nrep, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(b->sorted, iota.data(), sizeof(int) * n, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(b->rep_of, rep_of.data(), sizeof(int) * n, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(b->cell_rep, cell_rep.data(), sizeof(int) * b->ncell, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(b->st, init, sizeof init, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemset(b->cell_count, 0, sizeof(int) * (size_t)b->ncell) != cudaSuccess ||
        cudaMemset(b->rep_flag, 0, sizeof(int) * (size_t)nrep) != cudaSuccess ||
        cudaMemset(b->rep_dmax, 0, sizeof(unsigned) * (size_t)nrep) != cudaSuccess ||
        cudaMemset(b->cell_of, 0, sizeof(int) * n) != cudaSuccess ||
        cudaMemset(b->counts, 0, sizeof(int) * n) != cudaSuccess ||
        cudaMemset(b->ref, 0, sizeof(float4) * n) != cudaSuccess ||
        cudaStreamCreateWithFlags(&b->body, cudaStreamNonBlocking) != cudaSuccess) {
        batch_free(b);
        delete b;
        set_error("pd_batch_create: device initialisation failed");
        return PD_ECUDA;
    }
    *out = b;
    return PD_OK;
}

int pd_batch_destroy(pd_batch *b) {
    if (!b) return PD_OK;
    batch_free(b);
    delete b;
    return PD_OK;
}

int pd_batch_count(pd_batch *b, int *n, int *ncell) {
    PD_CHECK(b, PD_EINVAL, "pd_batch_count: null handle");
    if (n) *n = b->n;
    if (ncell) *ncell = b->ncell;
    return PD_OK;
}

int pd_batch_set_lanes(pd_batch *b, int lanes) {
    PD_CHECK(b, PD_EINVAL, "pd_batch_set_lanes: null handle");
    PD_CHECK(lanes == 1 || lanes == 2 || lanes == 4 || lanes == 8, PD_EINVAL, "pd_batch_set_lanes: lanes 1, 2, 4 or 8");
    b->lanes = lanes;
    return PD_OK;
}

int pd_batch_update(pd_batch *b, const float *x, const float *y, const float *z, pd_stream_t sp) {
    PD_CHECK(b && x && y && z, PD_EINVAL, "pd_batch_update: null argument");
    cudaStream_t s = (cudaStream_t)sp;
    k_batch_drift<false, false><<<(b->n + B_THREADS - 1) / B_THREADS, B_THREADS, 0, s>>>(
        b->n, const_cast<float *>(x), const_cast<float *>(y), const_cast<float *>(z), nullptr, nullptr, nullptr,
        nullptr, nullptr, nullptr, nullptr, 0.f, b->rep_of, b->reps, b->ref, b->threshold, b->rep_dmax, b->rep_flag,
        b->nrep, b->st, 0);
    PD_LAUNCHED();
    return batch_rebuild_launch(b, x, y, z, s);
}

int pd_batch_forces(pd_batch *b, const float *x, const float *y, const float *z, float *fx, float *fy, float *fz,
                    float *epot, int energy, pd_stream_t sp) {
    PD_CHECK(b && x && y && z && fx && fy && fz, PD_EINVAL, "pd_batch_forces: null argument");
    PD_CHECK(!energy || epot, PD_EINVAL, "pd_batch_forces: energy needs epot");
    BatchKick kick;
    memset(&kick, 0, sizeof kick);
    return batch_pairs_launch(b, x, y, z, fx, fy, fz, epot, energy, kick, 0, (cudaStream_t)sp);
}

int pd_batch_status(pd_batch *b, pd_ell_stats *out) {
    PD_CHECK(b && out, PD_EINVAL, "pd_batch_status: null argument");
    long long h[E_LEN];
    PD_CUDA(cudaMemcpy(h, b->st, sizeof h, cudaMemcpyDeviceToHost));
    memset(out, 0, sizeof *out);
    out->valid = h[E_VALID] != 0;
    out->error = (int)h[E_ERROR];
    out->requested = h[E_REQUEST] != 0;
    out->step = h[E_STEP];
    out->last_build = h[E_LAST_BUILD];
    out->interval = h[E_INTERVAL];
    out->checks = h[E_CHECKS];
    out->builds = h[E_BUILDS];
    out->required = h[E_REQUIRED];
    out->cap = b->cap;
    out->lanes = b->lanes;
    return PD_OK;
}

int pd_batch_bind(pd_batch *b, const pd_md_state *st) {
    PD_CHECK(b && st, PD_EINVAL, "pd_batch_bind: null argument");
    PD_CHECK(st->n == b->n, PD_EINVAL, "pd_batch_bind: state has %d particles, the batch %d", st->n, b->n);
    PD_CHECK(st->x && st->y && st->z && st->vx && st->vy && st->vz && st->fx && st->fy && st->fz && st->inv_mass,
             PD_EINVAL, "pd_batch_bind: state arrays missing (per-particle inverse masses required)");
    b->state = *st;
    b->bound = true;
    if (b->exec) cudaGraphExecDestroy(b->exec);
    b->exec = nullptr;
    return PD_OK;
}

int pd_batch_evaluate(pd_batch *b, int energy, pd_stream_t sp) {
    PD_CHECK(b && b->bound, PD_ESTATE, "pd_batch_evaluate: no state bound");
    const pd_md_state &S = b->state;
    int rc;
    if ((rc = pd_batch_update(b, S.x, S.y, S.z, sp))) return rc;
    PD_CHECK(!energy || S.epot, PD_EINVAL, "pd_batch_evaluate: energy needs epot in the state");
    return pd_batch_forces(b, S.x, S.y, S.z, S.fx, S.fy, S.fz, S.epot, energy, sp);
}

int pd_batch_step(pd_batch *b, int nsteps, float dt, int use_graph, pd_stream_t sp) {
    PD_CHECK(b && b->bound, PD_ESTATE, "pd_batch_step: no state bound");
    PD_CHECK(nsteps >= 0, PD_EINVAL, "pd_batch_step: negative step count");
    cudaStream_t s = (cudaStream_t)sp;
    for (int k = 0; k < nsteps; ++k) {
        if (!use_graph) {
            int rc = batch_enqueue_step(b, dt, s, 0);
            if (rc) return rc;
            continue;
        }
        if (!b->exec || b->exec_dt != dt || b->exec_stream != s || b->exec_lanes != b->lanes ||
            b->exec_chunk != b->mchunk * 8 + b->mtpi) {
            if (b->exec) {
                cudaGraphExecDestroy(b->exec);
                b->exec = nullptr;
            }
            PD_CHECK(s != nullptr, PD_EINVAL, "pd_batch_step: graph replay needs a non-default stream");
            for (int attempt = 0; attempt < 2 && !b->exec; ++attempt) {
                const int cond = b->cond_nodes ? 1 : 0;
                cudaGraph_t g = nullptr;
                PD_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
                const int rc = batch_enqueue_step(b, dt, s, cond);
                cudaError_t err = cudaStreamEndCapture(s, &g);
                // node priorities kept, so the charged batches' mesh branch keeps its streams' high priority
                if (rc == PD_OK && err == cudaSuccess)
                    err = cudaGraphInstantiateWithFlags(&b->exec, g, cudaGraphInstantiateFlagUseNodePriority);
                if (g) cudaGraphDestroy(g);
                if (rc == PD_OK && err == cudaSuccess) break;
                b->exec = nullptr;
                cudaGetLastError();
                if (!cond) {
                    if (rc) return rc;
                    PD_CHECK(false, PD_ECUDA, "batch step capture failed: %s", cudaGetErrorString(err));
                }
                b->cond_nodes = false;
            }
            b->exec_dt = dt;
            b->exec_stream = s;
            b->exec_lanes = b->lanes;
            b->exec_chunk = b->mchunk * 8 + b->mtpi;
        }
        PD_CUDA(cudaGraphLaunch(b->exec, s));
    }
    return PD_OK;
}

int pd_batch_set_coulomb(pd_batch *b, const pd_batch_coulomb *c) {
    PD_CHECK(b && c, PD_EINVAL, "pd_batch_set_coulomb: null argument");
    PD_CHECK(std::isfinite(c->C) && c->C > 0.f && c->rc2 > 0.f && std::isfinite(c->sx) && std::isfinite(c->selfc),
             PD_EINVAL, "pd_batch_set_coulomb: C, rc2, sx and selfc must be finite and C, rc2 positive");
    PD_CHECK(c->ne >= 1 && c->nf >= 1 && c->ne <= BATCH_NP && c->nf <= BATCH_NP, PD_EINVAL,
             "pd_batch_set_coulomb: the polynomials hold 1..%d coefficients", BATCH_NP);
    PD_CHECK(c->rc2 <= b->rl2, PD_EINVAL, "pd_batch_set_coulomb: the Coulomb cutoff exceeds the list radius %g "
             "(create the batch with a van der Waals cutoff covering it)", std::sqrt((double)b->rl2));
    BatchCoul cp{};
    cp.C = c->C;
    cp.rc2 = c->rc2;
    cp.sx = c->sx;
    cp.eshift = c->eshift;
    for (int k = 0; k < c->nf; ++k) cp.pf[k] = c->pf[k];
    for (int k = 0; k < c->ne; ++k) cp.pe[k] = c->pe[k];
    b->cp = cp;
    b->coul_ne = c->ne;
    b->coul_nf = c->nf;
    b->half_c_self = 0.5f * c->C * c->selfc;
    b->coul = true;
    if (b->exec) cudaGraphExecDestroy(b->exec);
    b->exec = nullptr;
    return PD_OK;
}

// Tiles of the batched meshes: replica r's cell-order positions are [first_r, first_r + N_r) (its
// cells are contiguous in the global cell order), cut into tiles of `chunk` positions; the last
// tile of a replica is padded (slot_src = -1).
static int batch_layout_chunks(pd_batch *b, int chunk) {
    batch_free_chunks(b);
    std::vector<int> crep, src;
    for (int r = 0; r < b->nrep; ++r) {
        const int first = b->first[(size_t)r];
        const int nr = (r + 1 < b->nrep ? b->first[(size_t)r + 1] : b->n) - first;
        const int nc = (nr + chunk - 1) / chunk;
        for (int c = 0; c < nc; ++c) {
            crep.push_back(r);
            for (int p = 0; p < chunk; ++p) {
                const int k = c * chunk + p;
                src.push_back(k < nr ? first + k : -1);
            }
        }
    }
    int rc;
    if ((rc = dalloc(&b->chunk_rep, crep.size())) || (rc = dalloc(&b->slot_src, src.size())) ||
        (rc = dalloc(&b->mid, src.size())) || (rc = dalloc(&b->mq, src.size())))
        return rc;
    PD_CUDA(cudaMemcpy(b->chunk_rep, crep.data(), sizeof(int) * crep.size(), cudaMemcpyHostToDevice));
    PD_CUDA(cudaMemcpy(b->slot_src, src.data(), sizeof(int) * src.size(), cudaMemcpyHostToDevice));
    PD_CUDA(cudaMemset(b->mid, 0xff, sizeof(int) * src.size()));
    PD_CUDA(cudaMemset(b->mq, 0, sizeof(float4) * src.size()));
    b->nchunk = (int)crep.size();   // only a complete layout is used
    b->mchunk = chunk;
    return PD_OK;
}

static int batch_set_mesh(pd_batch *b, int kind, int order, double alpha, double C, const int *meshes) {
    const int nrep = b->nrep;
    std::vector<int> idx((size_t)nrep);
    std::iota(idx.begin(), idx.end(), 0);
    auto key = [&](int r) { return std::make_tuple(meshes[3 * r + 2], meshes[3 * r + 1], meshes[3 * r]); };
    std::stable_sort(idx.begin(), idx.end(), [&](int a, int c) { return key(a) < key(c); });
    b->hmreps.assign((size_t)nrep, BMeshRep{});
    long long grid = 0, modes = 0;
    for (size_t a = 0; a < idx.size();) {
        size_t e = a;
        while (e < idx.size() && key(idx[e]) == key(idx[a])) ++e;
        const int r0 = idx[a];
        pd_batch::FftGroup g{};
        g.K1 = meshes[3 * r0];
        g.K2 = meshes[3 * r0 + 1];
        g.K3 = meshes[3 * r0 + 2];
        g.count = (int)(e - a);
        grid = (grid + 63) & ~63ll;     // each group starts on a 256-byte boundary
        modes = (modes + 31) & ~31ll;
        g.grid = grid;
        g.modes = modes;
        const int K1h = g.K1 / 2 + 1;
        const long long nn = (long long)g.K1 * g.K2 * g.K3, nm = (long long)K1h * g.K2 * g.K3;
        for (size_t j = a; j < e; ++j) {
            const int r = idx[j];
            BMeshRep &R = b->hmreps[(size_t)r];
            R.K1 = g.K1;
            R.K2 = g.K2;
            R.K3 = g.K3;
            R.K1h = K1h;
            R.Lx = b->hreps[(size_t)r].L[0];
            R.Ly = b->hreps[(size_t)r].L[1];
            R.Lz = b->hreps[(size_t)r].L[2];
            R.nmodes = (int)nm;
            R.grid = grid;
            R.modes = modes;
            grid += nn;
            modes += nm;
        }
        g.fwd = g.bwd = 0;
        b->groups.push_back(g);
        a = e;
    }
    b->total_nodes = grid;
    b->total_modes = modes;
    PD_CHECK(2 * modes >= grid, PD_EINVAL, "batched mesh: the modes do not cover the grids");
    int rc;
    if ((rc = dalloc(&b->gridA, (size_t)grid)) || (rc = dalloc(&b->gridB, (size_t)grid)) ||
        (rc = dalloc(&b->spec, (size_t)modes)) || (rc = dalloc(&b->G, (size_t)modes)) ||
        (rc = dalloc(&b->mreps, (size_t)nrep)))
        return rc;
    PD_CUDA(cudaMemset(b->gridA, 0, sizeof(float) * (size_t)grid));
    PD_CUDA(cudaMemset(b->gridB, 0, sizeof(float) * (size_t)grid));
    PD_CUDA(cudaMemset(b->spec, 0, sizeof(float2) * (size_t)modes));
    PD_CUDA(cudaMemset(b->G, 0, sizeof(float) * (size_t)modes));
    PD_CUDA(cudaMemcpy(b->mreps, b->hmreps.data(), sizeof(BMeshRep) * nrep, cudaMemcpyHostToDevice));
    // every replica's influence function from the single-system mesh setup (FP64, Influence.jl)
    for (int r = 0; r < nrep; ++r) {
        const BMeshRep &R = b->hmreps[(size_t)r];
        pd_mesh_params mp;
        memset(&mp, 0, sizeof mp);
        mp.kind = kind;
        mp.order = order;
        mp.alias_order = 2;
        mp.mesh[0] = R.K1;
        mp.mesh[1] = R.K2;
        mp.mesh[2] = R.K3;
        mp.alpha = alpha;
        mp.C = C;
        const int first = b->first[(size_t)r];
        mp.nmax = std::max(1, (r + 1 < nrep ? b->first[(size_t)r + 1] : b->n) - first);
        pd_mesh *m = nullptr;
        if ((rc = pd_mesh_create(&m, &mp, &b->box[3 * (size_t)r]))) return rc;
        cudaError_t err = cudaDeviceSynchronize();
        if (err == cudaSuccess)
            err = cudaMemcpy(b->G + R.modes, m->G, sizeof(float) * (size_t)R.nmodes, cudaMemcpyDeviceToDevice);
        pd_mesh_destroy(m);
        PD_CHECK(err == cudaSuccess, PD_ECUDA, "batched mesh: influence copy failed: %s", cudaGetErrorString(err));
    }
    size_t wmax = 0;
    for (auto &g : b->groups) {
        int n[3] = {g.K3, g.K2, g.K1};
        const int K1h = g.K1 / 2 + 1;
        const int nn = g.K1 * g.K2 * g.K3, nm = K1h * g.K2 * g.K3;
        size_t w1 = 0, w2 = 0;
        PD_CHECK(cufftCreate(&g.fwd) == CUFFT_SUCCESS && cufftCreate(&g.bwd) == CUFFT_SUCCESS, PD_ECUFFT,
                 "batched mesh: cufftCreate failed");
        PD_CHECK(cufftSetAutoAllocation(g.fwd, 0) == CUFFT_SUCCESS && cufftSetAutoAllocation(g.bwd, 0) == CUFFT_SUCCESS,
                 PD_ECUFFT, "batched mesh: cufftSetAutoAllocation failed");
        PD_CHECK(cufftMakePlanMany(g.fwd, 3, n, nullptr, 1, nn, nullptr, 1, nm, CUFFT_R2C, g.count, &w1) ==
                         CUFFT_SUCCESS &&
                     cufftMakePlanMany(g.bwd, 3, n, nullptr, 1, nm, nullptr, 1, nn, CUFFT_C2R, g.count, &w2) ==
                         CUFFT_SUCCESS,
                 PD_ECUFFT, "batched mesh: plan of %d meshes %dx%dx%d failed", g.count, g.K1, g.K2, g.K3);
        wmax = std::max(wmax, std::max(w1, w2));
    }
    // the mesh branch is the longer of the two branches of the force pass: its streams get the high
    // priority, so its kernels' blocks are scheduled ahead of the pair kernel's
    int prio_lo = 0, prio_hi = 0;
    cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi);
    for (int k = 0; k < pd_batch::NFFT; ++k) {
        PD_CUDA(cudaMalloc(&b->fft_work[k], std::max<size_t>(wmax, 256)));
        PD_CUDA(cudaStreamCreateWithPriority(&b->fft_stream[k], cudaStreamNonBlocking, prio_hi));
        PD_CUDA(cudaEventCreateWithFlags(&b->ev_fft[k], cudaEventDisableTiming));
    }
    PD_CUDA(cudaEventCreateWithFlags(&b->ev_fft_fork, cudaEventDisableTiming));
    for (size_t gi = 0; gi < b->groups.size(); ++gi) {
        auto &g = b->groups[gi];
        void *w = b->fft_work[gi % pd_batch::NFFT];
        PD_CHECK(cufftSetWorkArea(g.fwd, w) == CUFFT_SUCCESS && cufftSetWorkArea(g.bwd, w) == CUFFT_SUCCESS,
                 PD_ECUFFT, "batched mesh: cufftSetWorkArea failed");
    }
    PD_CUDA(cudaStreamCreateWithPriority(&b->mesh_stream, cudaStreamNonBlocking, prio_hi));
    PD_CUDA(cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming));
    PD_CUDA(cudaEventCreateWithFlags(&b->ev_join, cudaEventDisableTiming));
    if ((rc = batch_layout_chunks(b, b->mchunk))) return rc;
    b->morder = order;
    b->mesh = true;
    return PD_OK;
}

int pd_batch_set_mesh(pd_batch *b, int kind, int order, double alpha, double C, const int *meshes) {
    PD_CHECK(b && meshes, PD_EINVAL, "pd_batch_set_mesh: null argument");
    PD_CHECK(b->coul, PD_ESTATE, "pd_batch_set_mesh: set the real-space Coulomb terms first (pd_batch_set_coulomb)");
    PD_CHECK(kind == PD_MESH_SPME || kind == PD_MESH_P3M_AD, PD_ENOTSUP,
             "pd_batch_set_mesh: batched meshes take SPME or P3M-AD (analytic differentiation)");
    PD_CHECK(order >= 4 && order <= 6, PD_ENOTSUP, "pd_batch_set_mesh: batched meshes take orders 4, 5 and 6");
    PD_CHECK(std::isfinite(alpha) && alpha > 0 && std::isfinite(C) && C > 0, PD_EINVAL,
             "pd_batch_set_mesh: alpha and C must be finite and positive");
    for (int r = 0; r < b->nrep; ++r)
        for (int d = 0; d < 3; ++d)
            PD_CHECK(meshes[3 * r + d] >= order && meshes[3 * r + d] <= 1024, PD_EINVAL,
                     "pd_batch_set_mesh: replica %d mesh dimension %d is %d (order %d .. 1024)", r, d,
                     meshes[3 * r + d], order);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    b->exec = nullptr;
    batch_free_mesh(b);
    const int rc = batch_set_mesh(b, kind, order, alpha, C, meshes);
    if (rc != PD_OK) batch_free_mesh(b);
    return rc;
}

int pd_batch_set_spread_tile(pd_batch *b, int chunk, int threads_per_ion) {
    PD_CHECK(b, PD_EINVAL, "pd_batch_set_spread_tile: null handle");
    PD_CHECK(chunk == 32 || chunk == 64, PD_EINVAL, "pd_batch_set_spread_tile: 32 or 64 particles per tile");
    PD_CHECK(threads_per_ion == 2 || (threads_per_ion == 4 && chunk == 64), PD_EINVAL,
             "pd_batch_set_spread_tile: 2 threads per ion, or 4 with tiles of 64");
    b->mtpi = threads_per_ion;
    if (!b->mesh) {
        b->mchunk = chunk;
        return PD_OK;
    }
    if (chunk == b->mchunk) return PD_OK;
    const int rc = batch_layout_chunks(b, chunk);
    if (rc != PD_OK) batch_free_mesh(b);   // a batch without its tiles takes no charged step (PD_ESTATE)
    return rc;
}

int pd_batch_mesh_info(pd_batch *b, int *groups, long long *nodes, long long *modes, int *chunk, int *nchunk) {
    PD_CHECK(b, PD_EINVAL, "pd_batch_mesh_info: null handle");
    if (groups) *groups = (int)b->groups.size();
    if (nodes) *nodes = b->total_nodes;
    if (modes) *modes = b->total_modes;
    if (chunk) *chunk = b->mchunk;
    if (nchunk) *nchunk = b->nchunk;
    return PD_OK;
}

int pd_batch_rows(pd_batch *b, int **rows, int **counts, int **order) {
    PD_CHECK(b && rows && counts, PD_EINVAL, "pd_batch_rows: null argument");
    *rows = b->rows;
    *counts = b->counts;
    if (order) *order = b->sorted;
    return PD_OK;
}

}  // extern "C"
