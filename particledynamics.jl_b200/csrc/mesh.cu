// PME / P3M mesh engine of libpdb200.
//
// Semantics follow src/electrostatics of ParticleDynamics.jl: B-spline windows
// (Windows.jl:187-308), influence functions and virial coefficients in FP64
// (Influence.jl:24-227), the solve with the FP64 energy/virial reduction
// (MeshKernels.jl:34-81), the ik field (MeshKernels.jl:84-102) and the AD / ik
// gathers (MeshKernels.jl:105-147, 281-333); cuFFT does the transforms
// (Solver.jl:34-65, 305-347).
//
// Layout of this library: particles are processed in chunks of 64 consecutive
// entries of a spatially sorted sequence (a super-cluster of the cluster list).
// A chunk's stencils cover a small brick of the mesh; the spread accumulates
// the chunk into that brick in shared memory and adds the brick to the global
// grid once (one coalesced reduction per brick node instead of P^3 scattered
// atomics per particle), and the gather stages the brick of the potential in
// shared memory before every particle reads its P^3 nodes.  A chunk whose
// brick exceeds the shared-memory budget falls back to direct global
// accumulation.  The charge grid is kept zero between transforms: the solve
// clears it after the forward transform has consumed it, and the inverse
// transform writes the potential into a second grid.
#include <cufft.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "internal.hpp"

using namespace pdb;

#define PD_CUFFT(call)                                                      \
    do {                                                                    \
        cufftResult r_ = (call);                                            \
        if (r_ != CUFFT_SUCCESS) {                                          \
            ::pdb::set_error("%s failed: cufftResult %d", #call, (int)r_);  \
            return PD_ECUFFT;                                               \
        }                                                                   \
    } while (0)

namespace pdb {

constexpr int MESH_CHUNK = 64;        // particles per CTA
constexpr int MESH_THREADS = 128;     // two threads per particle (halves of the z stencil)
constexpr int TILE_MAX = 6144;        // floats of the shared brick (24 KiB)
constexpr int MESH_CTAS_PER_SM = 8;   // resident spread / gather CTAs per SM (one wave at ~1200 chunks)

// _grid_coordinate (MeshKernels.jl:9-15)
__device__ __forceinline__ float grid_coordinate(float x, float L, int K) {
    float s = x / L;
    s -= floorf(s);
    float u = s * (float)K;
    if (!isfinite(u)) return 0.f;
    return u >= (float)K ? u - (float)K : u;
}

// window_stencil(::BSplineStencil{P}, u) (Windows.jl:209-223): first node k0 =
// floor(u) - P + 1, weights M_P(u - k) in ascending node order and their
// derivatives dM_P/du = M_{P-1}(u-k) - M_{P-1}(u-k-1), by the order recursion
// of _bspline_step (Windows.jl:188-196).
template <int P>
__device__ __forceinline__ int bspline(float u, float *w, float *dw) {
    const float fl = floorf(u);
    const float t = u - fl;
    float a[P];
    a[0] = t;
    a[1] = 1.f - t;
#pragma unroll
    for (int n = 2; n < P - 1; ++n) {
        const float inv = 1.f / (float)n;
#pragma unroll
        for (int j = n; j >= 0; --j) {
            const float left = j < n ? a[j] : 0.f;
            const float right = j >= 1 ? a[j - 1] : 0.f;
            a[j] = ((t + (float)j) * left + (((float)(n + 1) - t) - (float)j) * right) * inv;
        }
    }
    {
        const int n = P - 1;
        const float inv = 1.f / (float)n;
#pragma unroll
        for (int j = 0; j < P; ++j) {
            const float left = j < n ? a[j] : 0.f;
            const float right = j >= 1 ? a[j - 1] : 0.f;
            w[P - 1 - j] = ((t + (float)j) * left + (((float)(n + 1) - t) - (float)j) * right) * inv;
        }
    }
    if (dw) {
#pragma unroll
        for (int i = 0; i < P; ++i) {
            const int j = P - 1 - i;
            const float left = j <= P - 2 ? a[j] : 0.f;
            const float right = j >= 1 ? a[j - 1] : 0.f;
            dw[i] = left - right;
        }
    }
    return (int)fl - (P - 1);
}

__device__ __forceinline__ int wrap_node(int n, int K) {
    n %= K;
    return n < 0 ? n + K : n;
}

// Signed offset of node k from the reference node r on a periodic axis of K nodes, in [-K/2, K/2).
__device__ __forceinline__ int signed_offset(int k, int r, int K) {
    int d = (k - r) % K;
    if (d < 0) d += K;
    if (d >= (K + 1) / 2) d -= K;
    return d;
}

// Brick of one chunk: first valid particle's stencil base is the reference;
// every particle's base is expressed as an offset from it, and the brick is
// the bounding box of the stencils.
//
// With vec (K1 a multiple of 4) the brick's x origin is aligned down to a
// multiple of 4 nodes and its x extent rounded up to a multiple of 4, so every
// brick row moves to and from the global grid as 16-byte vectors (a row of a
// multiple-of-4 mesh never splits a vector across its periodic end).  The
// wrapped global base of every brick row is tabulated once in shared memory.
struct Brick {
    int o1, o2, o3;   // global origin node (not wrapped)
    int e1, e2, e3;   // extents
    int fits;
    int vec;
};

constexpr int ROWS_MAX = 512;   // brick rows tabulated in shared memory

template <int P>
__device__ __forceinline__ void chunk_brick(bool valid, int k1, int k2, int k3, int K1, int K2, int K3, int &d1,
                                            int &d2, int &d3, Brick &b, int *sm /* >= 10 ints */,
                                            unsigned *rowbase) {
    // sm[0] first valid, sm[1..3] ref, sm[4..6] min, sm[7..9] max
    const int t = threadIdx.x;
    if (t == 0) {
        sm[0] = 1 << 30;
        sm[4] = sm[5] = sm[6] = 1 << 30;
        sm[7] = sm[8] = sm[9] = -(1 << 30);
    }
    __syncthreads();
    if (valid) atomicMin(&sm[0], t);
    __syncthreads();
    if (valid && sm[0] == t) {
        sm[1] = k1;
        sm[2] = k2;
        sm[3] = k3;
    }
    __syncthreads();
    const bool any = sm[0] < (1 << 30);
    if (valid) {
        d1 = signed_offset(k1, sm[1], K1);
        d2 = signed_offset(k2, sm[2], K2);
        d3 = signed_offset(k3, sm[3], K3);
        atomicMin(&sm[4], d1);
        atomicMin(&sm[5], d2);
        atomicMin(&sm[6], d3);
        atomicMax(&sm[7], d1);
        atomicMax(&sm[8], d2);
        atomicMax(&sm[9], d3);
    }
    __syncthreads();
    b.vec = (K1 & 3) == 0;
    if (any) {
        int o1 = sm[1] + sm[4], e1 = sm[7] - sm[4] + P;
        int shift = 0;
        if (b.vec) {
            shift = ((o1 % 4) + 4) % 4;
            o1 -= shift;
            e1 = (e1 + shift + 3) & ~3;
        }
        b.o1 = o1;
        b.o2 = sm[2] + sm[5];
        b.o3 = sm[3] + sm[6];
        b.e1 = e1;
        b.e2 = sm[8] - sm[5] + P;
        b.e3 = sm[9] - sm[6] + P;
        const long long nodes = (long long)b.e1 * b.e2 * b.e3;
        b.fits = nodes <= TILE_MAX && b.e1 <= MESH_THREADS && (!b.vec || b.e1 <= K1) &&
                 (long long)b.e2 * b.e3 <= ROWS_MAX;
        if (valid) {
            d1 += shift - sm[4];
            d2 -= sm[5];
            d3 -= sm[6];
        }
    } else {
        b.o1 = b.o2 = b.o3 = 0;
        b.e1 = b.e2 = b.e3 = 0;
        b.fits = 1;
    }
    if (b.fits) {
        const int nrows = b.e2 * b.e3;
        for (int r = threadIdx.x; r < nrows; r += blockDim.x) {
            const int l2 = r % b.e2, l3 = r / b.e2;
            rowbase[r] = (unsigned)(((size_t)wrap_node(b.o3 + l3, K3) * K2 + wrap_node(b.o2 + l2, K2)) * K1);
        }
    }
    __syncthreads();
}

// Move a brick between shared memory and the global grid: lanes are laid out as
// (row, x vector) with MESH_THREADS / nv rows in flight, nv = vectors (or nodes)
// per row; visit(tile_element, global_node) gets the first node of each
// 4-node vector (vec) or single node.
template <typename F>
__device__ __forceinline__ void for_brick(const Brick &b, const unsigned *rowbase, int K1, F &&visit) {
    const int per = b.vec ? 4 : 1;
    const int nv = b.e1 / per;
    if (nv == 0) return;
    const int rpi = MESH_THREADS / nv;
    const int t = threadIdx.x;
    const int r0 = t / nv, v = t - r0 * nv;
    if (r0 >= rpi) return;
    const int x0 = wrap_node(b.o1 + per * v, K1);
    const int nrows = b.e2 * b.e3;
    for (int r = r0; r < nrows; r += rpi) visit(r * nv + v, (size_t)rowbase[r] + x0);
}

// Spread of chunks of packed (x, y, z, q) particles (the charge assignment of
// _spread_lines_kernel!, MeshKernels.jl:247-276).  nchunk_dev (optional) holds
// the number of active chunks (the cluster list's super-cluster count).
template <int P>
__global__ void __launch_bounds__(MESH_THREADS, MESH_CTAS_PER_SM) k_spread(const float4 *__restrict__ xq, int nchunks,
                                                         const int *__restrict__ nchunk_dev, float *__restrict__ grid,
                                                         int K1, int K2, int K3, float Lx, float Ly, float Lz) {
    const int c = blockIdx.x;
    if (nchunk_dev && c >= *nchunk_dev) return;
    if (c >= nchunks) return;
    __shared__ __align__(16) float tile[TILE_MAX];
    __shared__ unsigned rowbase[ROWS_MAX];
    __shared__ int sm[10];
    const int t = threadIdx.x, p = t & (MESH_CHUNK - 1), h = t >> 6;
    const float4 v = xq[c * MESH_CHUNK + p];
    const bool valid = v.w != 0.f && isfinite(v.x) && isfinite(v.y) && isfinite(v.z);
    float w1[P], w2[P], w3[P];
    int k1 = 0, k2 = 0, k3 = 0;
    if (valid) {
        k1 = bspline<P>(grid_coordinate(v.x, Lx, K1), w1, nullptr);
        k2 = bspline<P>(grid_coordinate(v.y, Ly, K2), w2, nullptr);
        k3 = bspline<P>(grid_coordinate(v.z, Lz, K3), w3, nullptr);
    }
    int d1 = 0, d2 = 0, d3 = 0;
    Brick b;
    // both halves of a particle take part (their min/max contributions are identical)
    chunk_brick<P>(valid, k1, k2, k3, K1, K2, K3, d1, d2, d3, b, sm, rowbase);
    constexpr int PH = (P + 1) / 2;

    if (b.fits) {
        const int nb4 = (b.e1 * b.e2 * b.e3 + 3) >> 2;
        float4 *tile4 = reinterpret_cast<float4 *>(tile);
        for (int k = t; k < nb4; k += MESH_THREADS) tile4[k] = make_float4(0.f, 0.f, 0.f, 0.f);
        __syncthreads();
        if (valid) {
#pragma unroll
            for (int j3 = 0; j3 < P; ++j3) {   // this half's z nodes only (warp-uniform test)
            if ((j3 < PH) != (h == 0)) continue;
                const float q3 = v.w * w3[j3];
#pragma unroll
                for (int j2 = 0; j2 < P; ++j2) {
                    const float q23 = q3 * w2[j2];
                    float *row = tile + ((d3 + j3) * b.e2 + (d2 + j2)) * b.e1 + d1;
#pragma unroll
                    for (int j1 = 0; j1 < P; ++j1) red_add_shared(row + j1, q23 * w1[j1]);
                }
            }
        }
        __syncthreads();
        if (b.vec) {
            for_brick(b, rowbase, K1, [&](int kt, size_t kg) {
                const float4 val = tile4[kt];
                if (val.x != 0.f || val.y != 0.f || val.z != 0.f || val.w != 0.f)
                    red_add_v4(grid + kg, val.x, val.y, val.z, val.w);
            });
        } else {
            for_brick(b, rowbase, K1, [&](int kt, size_t kg) {
                const float val = tile[kt];
                if (val != 0.f) red_add(grid + kg, val);
            });
        }
    } else if (valid) {
#pragma unroll
        for (int j3 = 0; j3 < P; ++j3) {   // this half's z nodes only (warp-uniform test)
            if ((j3 < PH) != (h == 0)) continue;
            const int n3 = wrap_node(k3 + j3, K3);
            const float q3 = v.w * w3[j3];
#pragma unroll
            for (int j2 = 0; j2 < P; ++j2) {
                const int n2 = wrap_node(k2 + j2, K2);
                const float q23 = q3 * w2[j2];
#pragma unroll
                for (int j1 = 0; j1 < P; ++j1)
                    red_add(grid + ((size_t)n3 * K2 + n2) * K1 + wrap_node(k1 + j1, K1), q23 * w1[j1]);
            }
        }
    }
}

// Solve (_solve_kernel!, MeshKernels.jl:57-81): spec *= G; with energy the FP64
// mesh energy 1/2 sum w |b|^2 G and the six virial sums; the consumed charge grid
// is cleared for the next spread (two nodes per mode).
template <bool ENERGY>
__global__ void __launch_bounds__(256) k_solve(float2 *__restrict__ spec, const float *__restrict__ G,
                                               const float *__restrict__ Vc, double *__restrict__ acc, int K1, int K1h,
                                               int nmodes, float *__restrict__ gridA, int nnodes) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    double e = 0, v[6] = {0, 0, 0, 0, 0, 0};
    if (idx < nmodes) {
        const float2 z = spec[idx];
        const float Gm = G[idx];
        if (ENERGY) {
            const int m1 = idx % K1h;
            const double wgt = (m1 == 0 || ((K1 & 1) == 0 && m1 == K1 / 2)) ? 0.5 : 1.0;
            const double a = wgt * ((double)z.x * z.x + (double)z.y * z.y);
            e = a * (double)Gm;
#pragma unroll
            for (int k = 0; k < 6; ++k) v[k] = a * (double)Vc[(size_t)k * nmodes + idx];
        }
        spec[idx] = make_float2(z.x * Gm, z.y * Gm);
    }
    if (gridA) {
        const int n0 = 2 * idx;
        if (n0 + 1 < nnodes) {
            reinterpret_cast<float2 *>(gridA)[idx] = make_float2(0.f, 0.f);
        } else if (n0 < nnodes) {
            gridA[n0] = 0.f;
        }
    }
    if (ENERGY) {
        __shared__ double sh[7][8];
        const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
        double vals[7] = {e, v[0], v[1], v[2], v[3], v[4], v[5]};
#pragma unroll
        for (int k = 0; k < 7; ++k) {
            double s = warp_sum_d(vals[k]);
            if (lane == 0) sh[k][w] = s;
        }
        __syncthreads();
        if (w == 0) {
            const int nwp = blockDim.x >> 5;
#pragma unroll
            for (int k = 0; k < 7; ++k) {
                double s = lane < nwp ? sh[k][lane] : 0.0;
                s = warp_sum_d(s);
                if (lane == 0 && s != 0.0) red_add_d(&acc[k], s);
            }
        }
    }
}

// ik: out = -i k_d spec, Nyquist component of the operator zeroed (_ik_field_kernel!, MeshKernels.jl:84-102).
__global__ void k_ik_field(float2 *__restrict__ out, const float2 *__restrict__ spec, int K1, int K2, int K3, float L,
                           int dim) {
    const int K1h = K1 / 2 + 1;
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= K1h * K2 * K3) return;
    const int m1 = idx % K1h, rest = idx / K1h, m2 = rest % K2, m3 = rest / K2;
    const int m = dim == 0 ? m1 : (dim == 1 ? m2 : m3);
    const int K = dim == 0 ? K1 : (dim == 1 ? K2 : K3);
    const int s = ((K & 1) == 0 && m == K / 2) ? 0 : (m <= K / 2 ? m : m - K);
    const float kd = 6.283185307179586f * (float)s / L;
    const float2 z = spec[idx];
    out[idx] = make_float2(z.y * kd, -z.x * kd);
}

// AD gather of chunks (the sums of _gather_ad_lines_sums, MeshKernels.jl:281-311,
// and _gather_ad_lines_kernel!, :313-333) with the potential brick staged in
// shared memory.  JOIN adds the chunk's slot pair forces (and energies), writes
// the total force in storage order and applies the closing half kick; without
// JOIN the mesh force is stored (SET) or added to fx/fy/fz.
struct GatherOut {
    float *fx, *fy, *fz, *epot, *vir6;
    float *vx, *vy, *vz;
    const float *inv_mass;
    float inv_mass_uniform, half_dt;
    const int *ids;          // chunk entry -> particle (perm for the cluster slots, the order otherwise)
    int n_entries;           // entries with an id (SoA path); slots use perm < 0 for padding
    float4 *fc;              // JOIN: slot pair force + energy (cleared here)
    float *vc;               // JOIN energy: slot pair virial (cleared here)
    int nslot;
    float half_c_self;       // JOIN energy: 0.5 C selfc
    float bg;                // background potential per unit charge
    const float4 *extra;     // JOIN: per-particle force added before the kick (learned correction), or null
    const float4 *self_tab;  // self-force table of the mesh (T^3), or null: no self-force removal
    int self_T;
};

// Spurious self force of a unit charge at grid coordinates (u1, u2, u3): trilinear interpolation of
// the table sampled at the fractional positions t / T (t = 0 .. T-1) on each axis; the self force is
// periodic with period one node on every axis.
__device__ __forceinline__ float4 self_force(const float4 *__restrict__ tab, int T, float u1, float u2, float u3) {
    int i[3], j[3];
    float t[3];
    const float u[3] = {u1, u2, u3};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const float f = (u[d] - floorf(u[d])) * (float)T;
        int a = (int)f;
        a = a < 0 ? 0 : (a >= T ? T - 1 : a);
        i[d] = a;
        j[d] = a + 1 == T ? 0 : a + 1;
        t[d] = f - (float)a;
    }
    float4 r = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        const int a1 = (c & 1) ? j[0] : i[0], a2 = (c & 2) ? j[1] : i[1], a3 = (c & 4) ? j[2] : i[2];
        const float w = ((c & 1) ? t[0] : 1.f - t[0]) * ((c & 2) ? t[1] : 1.f - t[1]) * ((c & 4) ? t[2] : 1.f - t[2]);
        const float4 v = __ldg(tab + ((size_t)a3 * T + a2) * T + a1);
        r.x = fmaf(w, v.x, r.x);
        r.y = fmaf(w, v.y, r.y);
        r.z = fmaf(w, v.z, r.z);
    }
    return r;
}

// Grids a gather reads: AD the potential (g[0]); ik the three field components (g[0..2]) and, with
// energy, the potential (g[3]).
struct GatherGrids {
    const float *g[4];
};

// IK: the ik gather (_gather_ik_kernel!, MeshKernels.jl:105-147), F_i = q_i sum W E, with the three
// field grids staged through the same brick one after another.
template <int P, int MODE, bool ENERGY, bool IK>   // MODE 0: add, 1: set, 2: join (+ kick)
__global__ void __launch_bounds__(MESH_THREADS, MESH_CTAS_PER_SM) k_gather(const float4 *__restrict__ xq, int nchunks,
                                                         const int *__restrict__ nchunk_dev, GatherGrids grids,
                                                         int K1, int K2, int K3, float Lx, float Ly, float Lz,
                                                         GatherOut o) {
    const int c = blockIdx.x;
    if (nchunk_dev && c >= *nchunk_dev) return;
    if (c >= nchunks) return;
    __shared__ __align__(16) float tile[TILE_MAX];
    __shared__ unsigned rowbase[ROWS_MAX];
    __shared__ int sm[10];
    __shared__ float part[MESH_CHUNK][4];
    const int t = threadIdx.x, p = t & (MESH_CHUNK - 1), h = t >> 6;
    const int e = c * MESH_CHUNK + p;
    const float4 v = xq[e];
    const int id = (MODE == 2) ? o.ids[e] : (e < o.n_entries ? (o.ids ? o.ids[e] : e) : -1);
    const bool charged = v.w != 0.f && isfinite(v.x) && isfinite(v.y) && isfinite(v.z) && id >= 0;
    // join: fetch the slot pair force and the particle's velocity now, so that their latency
    // overlaps the brick set-up and the potential load below
    float4 fpair = make_float4(0.f, 0.f, 0.f, 0.f);
    float pvx = 0.f, pvy = 0.f, pvz = 0.f, pim = 0.f;
    float4 fextra = make_float4(0.f, 0.f, 0.f, 0.f);
    if (MODE == 2 && h == 0 && id >= 0) {
        fpair = o.fc[e];
        if (o.extra) fextra = o.extra[id];
        pvx = o.vx[id];
        pvy = o.vy[id];
        pvz = o.vz[id];
        pim = o.inv_mass ? o.inv_mass[id] : o.inv_mass_uniform;
    }
    float w1[P], w2[P], w3[P], g1[P], g2[P], g3[P];
    int k1 = 0, k2 = 0, k3 = 0;
    float u1 = 0.f, u2 = 0.f, u3 = 0.f;
    if (charged) {
        u1 = grid_coordinate(v.x, Lx, K1);
        u2 = grid_coordinate(v.y, Ly, K2);
        u3 = grid_coordinate(v.z, Lz, K3);
        k1 = bspline<P>(u1, w1, IK ? nullptr : g1);
        k2 = bspline<P>(u2, w2, IK ? nullptr : g2);
        k3 = bspline<P>(u3, w3, IK ? nullptr : g3);
    }
    int d1 = 0, d2 = 0, d3 = 0;
    Brick b;
    chunk_brick<P>(charged, k1, k2, k3, K1, K2, K3, d1, d2, d3, b, sm, rowbase);
    constexpr int PH = (P + 1) / 2;
    constexpr int NG = IK ? (ENERGY ? 4 : 3) : 1;   // grids read one after another

    float phi = 0.f, gx = 0.f, gy = 0.f, gz = 0.f;
    if (IK && b.fits) {
#pragma unroll 1
        for (int gi = 0; gi < NG; ++gi) {
            const float *grid = grids.g[gi];
            if (gi > 0) __syncthreads();   // every thread is done with the previous grid's brick
            if (b.vec) {
                float4 *tile4 = reinterpret_cast<float4 *>(tile);
                for_brick(b, rowbase, K1, [&](int kt, size_t kg) {
                    tile4[kt] = __ldg(reinterpret_cast<const float4 *>(grid + kg));
                });
            } else {
                for_brick(b, rowbase, K1, [&](int kt, size_t kg) { tile[kt] = __ldg(grid + kg); });
            }
            __syncthreads();
            if (charged) {
                float acc = 0.f;
#pragma unroll
                for (int j3 = 0; j3 < P; ++j3) {   // this half's z nodes only (warp-uniform test)
                    if ((j3 < PH) != (h == 0)) continue;
                    float s0 = 0.f;
#pragma unroll
                    for (int j2 = 0; j2 < P; ++j2) {
                        const float *row = tile + ((d3 + j3) * b.e2 + (d2 + j2)) * b.e1 + d1;
                        float a0 = 0.f;
#pragma unroll
                        for (int j1 = 0; j1 < P; ++j1) a0 = fmaf(w1[j1], row[j1], a0);
                        s0 = fmaf(w2[j2], a0, s0);
                    }
                    acc = fmaf(w3[j3], s0, acc);
                }
                if (gi == 0) gx = acc;
                else if (gi == 1) gy = acc;
                else if (gi == 2) gz = acc;
                else phi = acc;
            }
        }
    } else if (IK && charged) {
#pragma unroll 1
        for (int gi = 0; gi < NG; ++gi) {
            const float *grid = grids.g[gi];
            float acc = 0.f;
#pragma unroll
            for (int j3 = 0; j3 < P; ++j3) {   // this half's z nodes only (warp-uniform test)
                if ((j3 < PH) != (h == 0)) continue;
                const int n3 = wrap_node(k3 + j3, K3);
                float s0 = 0.f;
#pragma unroll
                for (int j2 = 0; j2 < P; ++j2) {
                    const int n2 = wrap_node(k2 + j2, K2);
                    float a0 = 0.f;
#pragma unroll
                    for (int j1 = 0; j1 < P; ++j1)
                        a0 = fmaf(w1[j1], grid[((size_t)n3 * K2 + n2) * K1 + wrap_node(k1 + j1, K1)], a0);
                    s0 = fmaf(w2[j2], a0, s0);
                }
                acc = fmaf(w3[j3], s0, acc);
            }
            if (gi == 0) gx = acc;
            else if (gi == 1) gy = acc;
            else if (gi == 2) gz = acc;
            else phi = acc;
        }
    } else if (b.fits) {
        const float *grid = grids.g[0];
        if (b.vec) {
            float4 *tile4 = reinterpret_cast<float4 *>(tile);
            for_brick(b, rowbase, K1, [&](int kt, size_t kg) {
                tile4[kt] = __ldg(reinterpret_cast<const float4 *>(grid + kg));
            });
        } else {
            for_brick(b, rowbase, K1, [&](int kt, size_t kg) { tile[kt] = __ldg(grid + kg); });
        }
        __syncthreads();
        if (charged) {
#pragma unroll
            for (int j3 = 0; j3 < P; ++j3) {   // this half's z nodes only (warp-uniform test)
            if ((j3 < PH) != (h == 0)) continue;
                float s0 = 0.f, s1 = 0.f, s2 = 0.f;   // sum w1 w2 c, sum dw1 w2 c, sum w1 dw2 c over a z-plane
#pragma unroll
                for (int j2 = 0; j2 < P; ++j2) {
                    const float *row = tile + ((d3 + j3) * b.e2 + (d2 + j2)) * b.e1 + d1;
                    float a0 = 0.f, a1 = 0.f;
#pragma unroll
                    for (int j1 = 0; j1 < P; ++j1) {
                        const float cval = row[j1];
                        a0 = fmaf(w1[j1], cval, a0);
                        a1 = fmaf(g1[j1], cval, a1);
                    }
                    s0 = fmaf(w2[j2], a0, s0);
                    s1 = fmaf(w2[j2], a1, s1);
                    s2 = fmaf(g2[j2], a0, s2);
                }
                phi = fmaf(w3[j3], s0, phi);
                gz = fmaf(g3[j3], s0, gz);
                gx = fmaf(w3[j3], s1, gx);
                gy = fmaf(w3[j3], s2, gy);
            }
        }
    } else if (charged) {
        const float *grid = grids.g[0];
#pragma unroll
        for (int j3 = 0; j3 < P; ++j3) {   // this half's z nodes only (warp-uniform test)
            if ((j3 < PH) != (h == 0)) continue;
            const int n3 = wrap_node(k3 + j3, K3);
            float s0 = 0.f, s1 = 0.f, s2 = 0.f;
#pragma unroll
            for (int j2 = 0; j2 < P; ++j2) {
                const int n2 = wrap_node(k2 + j2, K2);
                float a0 = 0.f, a1 = 0.f;
#pragma unroll
                for (int j1 = 0; j1 < P; ++j1) {
                    const float cval = grid[((size_t)n3 * K2 + n2) * K1 + wrap_node(k1 + j1, K1)];
                    a0 = fmaf(w1[j1], cval, a0);
                    a1 = fmaf(g1[j1], cval, a1);
                }
                s0 = fmaf(w2[j2], a0, s0);
                s1 = fmaf(w2[j2], a1, s1);
                s2 = fmaf(g2[j2], a0, s2);
            }
            phi = fmaf(w3[j3], s0, phi);
            gz = fmaf(g3[j3], s0, gz);
            gx = fmaf(w3[j3], s1, gx);
            gy = fmaf(w3[j3], s2, gy);
        }
    }
    // combine the two z halves
    if (h == 1) {
        part[p][0] = phi;
        part[p][1] = gx;
        part[p][2] = gy;
        part[p][3] = gz;
    }
    __syncthreads();
    if (h == 1) return;
    phi += part[p][0];
    gx += part[p][1];
    gy += part[p][2];
    gz += part[p][3];
    const float qi = v.w;
    float Fx = 0.f, Fy = 0.f, Fz = 0.f, Ei = 0.f;
    if (charged) {
        if (IK) {
            Fx = qi * gx;
            Fy = qi * gy;
            Fz = qi * gz;
        } else {
            Fx = -(qi * gx * ((float)K1 / Lx));
            Fy = -(qi * gy * ((float)K2 / Ly));
            Fz = -(qi * gz * ((float)K3 / Lz));
        }
        if (ENERGY) Ei = 0.5f * qi * phi + o.bg * qi;
        if (!IK && o.self_tab) {   // remove the charge's own force through the mesh: F -= q^2 S(u)
            const float4 sf = self_force(o.self_tab, o.self_T, u1, u2, u3);
            const float q2 = qi * qi;
            Fx = fmaf(-q2, sf.x, Fx);
            Fy = fmaf(-q2, sf.y, Fy);
            Fz = fmaf(-q2, sf.z, Fz);
        }
    }
    if (MODE == 2) {
        if (id < 0) return;
        const float4 f = fpair;
        o.fc[e] = make_float4(0.f, 0.f, 0.f, 0.f);
        Fx += f.x + fextra.x;
        Fy += f.y + fextra.y;
        Fz += f.z + fextra.z;
        o.fx[id] = Fx;
        o.fy[id] = Fy;
        o.fz[id] = Fz;
        const float cm = o.half_dt * pim;
        o.vx[id] = fmaf(cm, Fx, pvx);
        o.vy[id] = fmaf(cm, Fy, pvy);
        o.vz[id] = fmaf(cm, Fz, pvz);
        if (ENERGY) {
            o.epot[id] = Ei + f.w - o.half_c_self * qi * qi;
#pragma unroll
            for (int k = 0; k < 6; ++k) {
                o.vir6[(size_t)id * 6 + k] = o.vc[(size_t)k * o.nslot + e];
                o.vc[(size_t)k * o.nslot + e] = 0.f;
            }
        }
    } else {
        if (id < 0) return;
        if (MODE == 1) {
            o.fx[id] = Fx;
            o.fy[id] = Fy;
            o.fz[id] = Fz;
            if (ENERGY) o.epot[id] = Ei;
        } else if (charged) {
            o.fx[id] += Fx;
            o.fy[id] += Fy;
            o.fz[id] += Fz;
            if (ENERGY) o.epot[id] += Ei;
        }
    }
}

// Particles of `order` packed as (x, y, z, q) in chunks of 64 (zero-charge padding).
// Self-force table: a unit charge at grid coordinate t / T (t = 0 .. T-1 per axis) spreads the
// weights W_b (b in the P^3 stencil) and gathers -grad W_a . phi_a with phi_a = sum_b Ghat(a - b) W_b,
// where Ghat is the potential grid that the solve and the inverse transform make from a unit grid
// charge at node 0 (the mesh's own discrete kernel, translation invariant).  The result is the force
// that the AD gather gives a particle from its own charge (zero for the exact reciprocal sum);
// Ballenegger, Cerda and Holm, Comput. Phys. Commun. 182 (2011) 1919, remove it the same way.
template <int P>
__global__ void k_self_table(const float *__restrict__ ghat, int K1, int K2, int K3, float s1, float s2, float s3,
                             int T, float4 *__restrict__ tab) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= T * T * T) return;
    const int t1 = idx % T, t2 = (idx / T) % T, t3 = idx / (T * T);
    float w1[P], w2[P], w3[P], g1[P], g2[P], g3[P];
    bspline<P>((float)t1 / (float)T, w1, g1);
    bspline<P>((float)t2 / (float)T, w2, g2);
    bspline<P>((float)t3 / (float)T, w3, g3);
    double fx = 0, fy = 0, fz = 0;
    for (int a3 = 0; a3 < P; ++a3)
        for (int a2 = 0; a2 < P; ++a2)
            for (int a1 = 0; a1 < P; ++a1) {
                double phi = 0;
                for (int b3 = 0; b3 < P; ++b3)
                    for (int b2 = 0; b2 < P; ++b2) {
                        const size_t row = ((size_t)wrap_node(a3 - b3, K3) * K2 + wrap_node(a2 - b2, K2)) * K1;
                        const double wb = (double)w3[b3] * w2[b2];
                        for (int b1 = 0; b1 < P; ++b1)
                            phi += wb * w1[b1] * (double)ghat[row + wrap_node(a1 - b1, K1)];
                    }
                fx += (double)g1[a1] * w2[a2] * w3[a3] * phi;
                fy += (double)w1[a1] * g2[a2] * w3[a3] * phi;
                fz += (double)w1[a1] * w2[a2] * g3[a3] * phi;
            }
    tab[idx] = make_float4((float)(-fx * s1), (float)(-fy * s2), (float)(-fz * s3), 0.f);
}

__global__ void k_unit_node(float *grid) { grid[0] = 1.f; }

__global__ void k_pack_order(const float *__restrict__ x, const float *__restrict__ y, const float *__restrict__ z,
                             const float *__restrict__ q, const int *__restrict__ order, int n, int ntot,
                             float4 *__restrict__ out) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ntot) return;
    if (t < n) {
        const int i = order ? order[t] : t;
        out[t] = make_float4(x[i], y[i], z[i], q[i]);
    } else {
        out[t] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
}

// Global virial plus background (_store_global_virial_kernel!, Solver.jl:382-388).
__global__ void k_store_virial(float *vg, const double *acc, double ubg) {
    const int i = threadIdx.x;
    if (i < 6) vg[i] = (float)(acc[i + 1] + (i < 3 ? ubg : 0.0));
}

// ------------------------------------------------------------ influence (FP64)

__device__ __forceinline__ int signed_mode(int m, int K) { return m <= K / 2 ? m : m - K; }
__device__ __forceinline__ bool is_nyquist(int m, int K) { return (K % 2 == 0) && m == K / 2; }

// spectral_g(::GaussianSpectral, k) (Splits.jl:220-224): g(k) and g'(k)/k
__device__ __forceinline__ void spectral_g(double alpha, double k, double &g, double &gpk) {
    const double k2 = k * k;
    g = 4.0 * M_PI * exp(-k2 / (4.0 * alpha * alpha)) / k2;
    gpk = g * (-2.0 / k2 - 1.0 / (2.0 * alpha * alpha));
}

// _influence_ewald_kernel! (Influence.jl:35-67)
__global__ void k_influence_spme(float *__restrict__ G, float *__restrict__ Vc, const double *__restrict__ D1,
                                 const double *__restrict__ D2, const double *__restrict__ D3, int K1, int K2, int K3,
                                 double L1, double L2, double L3, double C, double alpha) {
    const int K1h = K1 / 2 + 1;
    const int nmodes = K1h * K2 * K3;
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= nmodes) return;
    const int m1 = idx % K1h, rest = idx / K1h, m2 = rest % K2, m3 = rest / K2;
    const int s1 = m1, s2 = signed_mode(m2, K2), s3 = signed_mode(m3, K3);
    if (s1 == 0 && s2 == 0 && s3 == 0) {
        G[idx] = 0.f;
        for (int c = 0; c < 6; ++c) Vc[(size_t)c * nmodes + idx] = 0.f;
        return;
    }
    const double CoverV = C / (L1 * L2 * L3);
    const double kx = 2.0 * M_PI * s1 / L1, ky = 2.0 * M_PI * s2 / L2, kz = 2.0 * M_PI * s3 / L3;
    const double k = sqrt(kx * kx + ky * ky + kz * kz);
    double g, gpk;
    spectral_g(alpha, k, g, gpk);
    const double D = D1[m1] * D2[m2] * D3[m3];
    const double Gm = CoverV * g * D;
    const double c = CoverV * D * gpk;
    const bool n1 = is_nyquist(m1, K1), n2 = is_nyquist(m2, K2), n3 = is_nyquist(m3, K3);
    G[idx] = (float)Gm;
    Vc[(size_t)0 * nmodes + idx] = (float)(Gm + c * kx * kx);
    Vc[(size_t)1 * nmodes + idx] = (float)(Gm + c * ky * ky);
    Vc[(size_t)2 * nmodes + idx] = (float)(Gm + c * kz * kz);
    Vc[(size_t)3 * nmodes + idx] = (n1 || n2) ? 0.f : (float)(c * kx * ky);
    Vc[(size_t)4 * nmodes + idx] = (n1 || n3) ? 0.f : (float)(c * kx * kz);
    Vc[(size_t)5 * nmodes + idx] = (n2 || n3) ? 0.f : (float)(c * ky * kz);
}

// _influence_alias_kernel! (Influence.jl:77-181): optimal P3M influence for AD or ik.
__global__ void k_influence_alias(float *__restrict__ G, float *__restrict__ Vc, const double *__restrict__ U1,
                                  const double *__restrict__ U2, const double *__restrict__ U3, int K1, int K2, int K3,
                                  double L1, double L2, double L3, double C, double alpha, int nmax, int ik) {
    const int K1h = K1 / 2 + 1;
    const int nmodes = K1h * K2 * K3;
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= nmodes) return;
    const int na = 2 * nmax + 1;
    const int m1 = idx % K1h, rest = idx / K1h, m2 = rest % K2, m3 = rest / K2;
    const int s1 = m1, s2 = signed_mode(m2, K2), s3 = signed_mode(m3, K3);
    const bool ny1 = is_nyquist(m1, K1), ny2 = is_nyquist(m2, K2), ny3 = is_nyquist(m3, K3);
    const double kx = 2.0 * M_PI * s1 / L1, ky = 2.0 * M_PI * s2 / L2, kz = 2.0 * M_PI * s3 / L3;
    const double dx = ny1 ? 0.0 : kx, dy = ny2 ? 0.0 : ky, dz = ny3 ? 0.0 : kz;
    const double d2 = dx * dx + dy * dy + dz * dz;
    const bool zero_mode = s1 == 0 && s2 == 0 && s3 == 0;
    if (zero_mode || (ik && d2 == 0.0)) {
        G[idx] = 0.f;
        for (int c = 0; c < 6; ++c) Vc[(size_t)c * nmodes + idx] = 0.f;
        return;
    }
    const double CoverV = C / (L1 * L2 * L3);
    double A = 0, B = 0, Cc = 0;
    double a1 = 0, a2 = 0, a3 = 0, a4 = 0, a5 = 0, a6 = 0;
    double c1 = 0, c2 = 0, c3 = 0, c4 = 0, c5 = 0, c6 = 0;
    for (int n1 = -nmax; n1 <= nmax; ++n1) {
        const double u1 = U1[(size_t)m1 * na + (n1 + nmax)];
        const double q1 = 2.0 * M_PI * (s1 + (double)K1 * n1) / L1;
        for (int n2 = -nmax; n2 <= nmax; ++n2) {
            const double u2 = U2[(size_t)m2 * na + (n2 + nmax)];
            const double q2 = 2.0 * M_PI * (s2 + (double)K2 * n2) / L2;
            for (int n3 = -nmax; n3 <= nmax; ++n3) {
                const double u3 = U3[(size_t)m3 * na + (n3 + nmax)];
                const double q3 = 2.0 * M_PI * (s3 + (double)K3 * n3) / L3;
                const double uu = u1 * u2 * u3;
                const double U2tot = uu * uu;
                B += U2tot;
                const double qq = q1 * q1 + q2 * q2 + q3 * q3;
                if (qq == 0.0) continue;
                double g, gpk;
                spectral_g(alpha, sqrt(qq), g, gpk);
                if (ik) {
                    const double dq = dx * q1 + dy * q2 + dz * q3;
                    A += U2tot * g * dq;
                    const double hh = U2tot * gpk * dq;
                    a1 += hh * q1 * q1 + U2tot * g * 2.0 * dx * q1;
                    a2 += hh * q2 * q2 + U2tot * g * 2.0 * dy * q2;
                    a3 += hh * q3 * q3 + U2tot * g * 2.0 * dz * q3;
                    a4 += hh * q1 * q2 + U2tot * g * (dx * q2 + q1 * dy);
                    a5 += hh * q1 * q3 + U2tot * g * (dx * q3 + q1 * dz);
                    a6 += hh * q2 * q3 + U2tot * g * (dy * q3 + q2 * dz);
                } else {
                    A += U2tot * g * qq;
                    Cc += U2tot * qq;
                    const double hh = U2tot * (gpk * qq + 2.0 * g);
                    a1 += hh * q1 * q1;
                    a2 += hh * q2 * q2;
                    a3 += hh * q3 * q3;
                    a4 += hh * q1 * q2;
                    a5 += hh * q1 * q3;
                    a6 += hh * q2 * q3;
                    const double h2 = 2.0 * U2tot;
                    c1 += h2 * q1 * q1;
                    c2 += h2 * q2 * q2;
                    c3 += h2 * q3 * q3;
                    c4 += h2 * q1 * q2;
                    c5 += h2 * q1 * q3;
                    c6 += h2 * q2 * q3;
                }
            }
        }
    }
    double Gm, v1, v2, v3, v4, v5, v6;
    if (ik) {
        const double den = d2 * B * B;
        Gm = CoverV * A / den;
        const double f = CoverV / den;
        const double r = CoverV * A / (B * B) * 2.0 / (d2 * d2);
        v1 = Gm + f * a1 - r * dx * dx;
        v2 = Gm + f * a2 - r * dy * dy;
        v3 = Gm + f * a3 - r * dz * dz;
        v4 = f * a4 - r * dx * dy;
        v5 = f * a5 - r * dx * dz;
        v6 = f * a6 - r * dy * dz;
    } else {
        Gm = CoverV * A / (B * Cc);
        const double f = CoverV / (B * Cc);
        const double r = CoverV * A / (B * Cc * Cc);
        v1 = Gm + f * a1 - r * c1;
        v2 = Gm + f * a2 - r * c2;
        v3 = Gm + f * a3 - r * c3;
        v4 = f * a4 - r * c4;
        v5 = f * a5 - r * c5;
        v6 = f * a6 - r * c6;
    }
    G[idx] = (float)Gm;
    Vc[(size_t)0 * nmodes + idx] = (float)v1;
    Vc[(size_t)1 * nmodes + idx] = (float)v2;
    Vc[(size_t)2 * nmodes + idx] = (float)v3;
    Vc[(size_t)3 * nmodes + idx] = (ny1 || ny2) ? 0.f : (float)v4;
    Vc[(size_t)4 * nmodes + idx] = (ny1 || ny3) ? 0.f : (float)v5;
    Vc[(size_t)5 * nmodes + idx] = (ny2 || ny3) ? 0.f : (float)v6;
}

// ---------------------------------------------------------------- host side

// M_P at the integers 0..P-1 (_bspline_integer_values, Windows.jl:265-271).
static std::vector<double> bspline_integer_values(int P) {
    std::vector<double> a = {0.0, 1.0};
    while ((int)a.size() < P) {
        const int N = (int)a.size();
        std::vector<double> b(N + 1);
        for (int jj = 0; jj <= N; ++jj) {
            const double left = jj < N ? a[jj] : 0.0;
            const double right = jj >= 1 ? a[jj - 1] : 0.0;
            b[jj] = ((0.0 + jj) * left + ((double)(N + 1) - 0.0 - jj) * right) / (double)N;
        }
        a = b;
    }
    return a;
}

// window_deconvolution(::BSplineWindow, K) (Windows.jl:283-308)
static std::vector<double> bspline_deconvolution(int P, int K) {
    std::vector<double> M = bspline_integer_values(P);
    std::vector<double> D(K);
    for (int m = 0; m < K; ++m) {
        double re = 0, im = 0;
        for (int j = 0; j < P; ++j) {
            const double ang = 2.0 * M_PI * m * j / K;
            re += M[j] * cos(ang);
            im += M[j] * sin(ang);
        }
        const double den = re * re + im * im;
        D[m] = den > 1e-12 ? 1.0 / den : NAN;
    }
    for (int m = 0; m < K; ++m) {
        if (std::isnan(D[m])) {
            const double l = D[(m - 1 + K) % K], r = D[(m + 1) % K];
            D[m] = 0.5 * (l + r);
        }
    }
    return D;
}

// window_alias_table(::BSplineWindow, K, nmax) (Windows.jl:391-399), stored [m][n + nmax].
static std::vector<double> bspline_alias_table(int P, int K, int nmax) {
    const int na = 2 * nmax + 1;
    std::vector<double> U((size_t)K * na);
    for (int m = 0; m < K; ++m) {
        const int sm = m <= K / 2 ? m : m - K;
        for (int n = -nmax; n <= nmax; ++n) {
            const double x = M_PI * (sm + (double)K * n) / K;
            const double s = fabs(x) < 1e-12 ? 1.0 : sin(x) / x;
            U[(size_t)m * na + (n + nmax)] = pow(s, P);
        }
    }
    return U;
}

static int compute_influence(pd_mesh *m) {
    const int K1 = m->K1, K2 = m->K2, K3 = m->K3, P = m->p.order;
    std::vector<double> t1, t2, t3;
    if (m->p.kind == PD_MESH_SPME) {
        t1 = bspline_deconvolution(P, K1);
        t2 = bspline_deconvolution(P, K2);
        t3 = bspline_deconvolution(P, K3);
    } else {
        t1 = bspline_alias_table(P, K1, m->p.alias_order);
        t2 = bspline_alias_table(P, K2, m->p.alias_order);
        t3 = bspline_alias_table(P, K3, m->p.alias_order);
    }
    double *d1 = nullptr, *d2 = nullptr, *d3 = nullptr;
    int rc;
    if ((rc = dalloc(&d1, t1.size())) || (rc = dalloc(&d2, t2.size())) || (rc = dalloc(&d3, t3.size()))) {
        dfree(d1);
        dfree(d2);
        dfree(d3);
        return rc;
    }
    cudaMemcpy(d1, t1.data(), t1.size() * sizeof(double), cudaMemcpyHostToDevice);
    cudaMemcpy(d2, t2.data(), t2.size() * sizeof(double), cudaMemcpyHostToDevice);
    cudaMemcpy(d3, t3.data(), t3.size() * sizeof(double), cudaMemcpyHostToDevice);
    const int threads = 128, blocks = (m->nmodes + threads - 1) / threads;
    if (m->p.kind == PD_MESH_SPME) {
        k_influence_spme<<<blocks, threads>>>(m->G, m->Vc, d1, d2, d3, K1, K2, K3, m->box[0], m->box[1], m->box[2],
                                              m->p.C, m->p.alpha);
    } else {
        k_influence_alias<<<blocks, threads>>>(m->G, m->Vc, d1, d2, d3, K1, K2, K3, m->box[0], m->box[1], m->box[2],
                                               m->p.C, m->p.alpha, m->p.alias_order, m->p.kind == PD_MESH_P3M_IK);
    }
    count_launch();
    cudaError_t e = cudaGetLastError();
    cudaError_t e2 = cudaDeviceSynchronize();
    dfree(d1);
    dfree(d2);
    dfree(d3);
    PD_CHECK(e == cudaSuccess && e2 == cudaSuccess, PD_ECUDA, "influence kernel failed: %s",
             cudaGetErrorString(e != cudaSuccess ? e : e2));
    return PD_OK;
}

static void refresh_background(pd_mesh *m) {
    const double V = m->box[0] * m->box[1] * m->box[2];
    const double bgcoef = M_PI / (2.0 * m->p.alpha * m->p.alpha);   // background_coefficient (Splits.jl:85)
    m->bg = m->p.background ? (float)(-m->p.C * bgcoef * m->p.qtotal / V) : 0.f;
    m->ubg = m->p.background ? -m->p.C * bgcoef * m->p.qtotal * m->p.qtotal / V : 0.0;
}

#define PD_SPREAD_CASE(PP)                                                                                         \
    case PP:                                                                                                       \
        k_spread<PP><<<nchunks, MESH_THREADS, 0, s>>>(xq, nchunks, ns_dev, m->gridA, m->K1, m->K2, m->K3, Lx, Ly, Lz); \
        break;

// Fill m->self_tab (T = m->self_T) for the current box and influence function (host boundary: runs on
// the legacy stream and waits for it).  Leaves the charge grid zero, as every transform does.
static int compute_self_table(pd_mesh *m) {
    if (!m->self_tab || m->self_T <= 0) return PD_OK;
    cudaStream_t s = 0;
    k_unit_node<<<1, 1, 0, s>>>(m->gridA);
    PD_LAUNCHED();
    PD_CUFFT(cufftSetStream(m->fwd, s));
    PD_CUFFT(cufftExecR2C(m->fwd, m->gridA, m->spec));
    k_solve<false><<<(m->nmodes + 255) / 256, 256, 0, s>>>((float2 *)m->spec, m->G, m->Vc, m->acc, m->K1, m->K1h,
                                                            m->nmodes, m->gridA, m->nnodes);
    PD_LAUNCHED();
    PD_CUFFT(cufftSetStream(m->bwd, s));
    PD_CUFFT(cufftExecC2R(m->bwd, m->spec, m->gridB));
    const int T = m->self_T, cells = T * T * T;
    const float s1 = (float)(m->K1 / m->box[0]), s2 = (float)(m->K2 / m->box[1]), s3 = (float)(m->K3 / m->box[2]);
#define PD_ST(PP)                                                                                             \
    case PP:                                                                                                  \
        k_self_table<PP><<<(cells + 127) / 128, 128, 0, s>>>(m->gridB, m->K1, m->K2, m->K3, s1, s2, s3, T,     \
                                                             m->self_tab);                                    \
        break;
    switch (m->p.order) {
        PD_ST(3) PD_ST(4) PD_ST(5) PD_ST(6) PD_ST(7) PD_ST(8) PD_ST(9) PD_ST(10) PD_ST(11) PD_ST(12)
        default: break;
    }
#undef PD_ST
    PD_LAUNCHED();
    PD_CUDA(cudaStreamSynchronize(s));
    return PD_OK;
}

int mesh_transform_packed(pd_mesh *m, const float4 *xq, int nchunks, const int *ns_dev, int energy, cudaStream_t s) {
    const float Lx = (float)m->box[0], Ly = (float)m->box[1], Lz = (float)m->box[2];
    switch (m->p.order) {
        PD_SPREAD_CASE(3)
        PD_SPREAD_CASE(4)
        PD_SPREAD_CASE(5)
        PD_SPREAD_CASE(6)
        PD_SPREAD_CASE(7)
        PD_SPREAD_CASE(8)
        PD_SPREAD_CASE(9)
        PD_SPREAD_CASE(10)
        PD_SPREAD_CASE(11)
        PD_SPREAD_CASE(12)
        default: set_error("unsupported order %d", m->p.order); return PD_EINVAL;
    }
    PD_LAUNCHED();
    PD_CUFFT(cufftSetStream(m->fwd, s));
    PD_CUFFT(cufftExecR2C(m->fwd, m->gridA, m->spec));
    if (energy) PD_CUDA(cudaMemsetAsync(m->acc, 0, 7 * sizeof(double), s));
    const int blocks = (m->nmodes + 255) / 256;
    if (energy)
        k_solve<true><<<blocks, 256, 0, s>>>((float2 *)m->spec, m->G, m->Vc, m->acc, m->K1, m->K1h, m->nmodes, m->gridA,
                                             m->nnodes);
    else
        k_solve<false><<<blocks, 256, 0, s>>>((float2 *)m->spec, m->G, m->Vc, m->acc, m->K1, m->K1h, m->nmodes,
                                              m->gridA, m->nnodes);
    PD_LAUNCHED();
    PD_CUFFT(cufftSetStream(m->bwd, s));
    if (m->p.kind == PD_MESH_P3M_IK) {
        const float L[3] = {Lx, Ly, Lz};
        for (int d = 0; d < 3; ++d) {
            k_ik_field<<<blocks, 256, 0, s>>>((float2 *)m->scratch, (const float2 *)m->spec, m->K1, m->K2, m->K3, L[d], d);
            PD_LAUNCHED();
            PD_CUFFT(cufftExecC2R(m->bwd, m->scratch, m->field[d]));
        }
        if (energy) {
            PD_CUFFT(cufftExecC2R(m->bwd, m->spec, m->gridB));
        }
    } else {
        PD_CUFFT(cufftExecC2R(m->bwd, m->spec, m->gridB));
    }
    return PD_OK;
}
#undef PD_SPREAD_CASE

int mesh_store_virial(pd_mesh *m, float *vglobal6, cudaStream_t s) {
    if (!vglobal6) return PD_OK;
    k_store_virial<<<1, 32, 0, s>>>(vglobal6, m->acc, m->ubg);
    PD_LAUNCHED();
    return PD_OK;
}

template <int MODE, bool ENERGY>
static void launch_gather(pd_mesh *m, const float4 *xq, int nchunks, const int *ns_dev, const GatherOut &o,
                          cudaStream_t s) {
    const float Lx = (float)m->box[0], Ly = (float)m->box[1], Lz = (float)m->box[2];
    const int K1 = m->K1, K2 = m->K2, K3 = m->K3;
    const bool ik = m->p.kind == PD_MESH_P3M_IK;
    GatherGrids g = {{m->gridB, nullptr, nullptr, nullptr}};
    if (ik) g = GatherGrids{{m->field[0], m->field[1], m->field[2], m->gridB}};
#define PD_G(PP)                                                                                                       \
    case PP:                                                                                                           \
        if (ik)                                                                                                        \
            k_gather<PP, MODE, ENERGY, true><<<nchunks, MESH_THREADS, 0, s>>>(xq, nchunks, ns_dev, g, K1, K2, K3, Lx,  \
                                                                              Ly, Lz, o);                              \
        else                                                                                                           \
            k_gather<PP, MODE, ENERGY, false><<<nchunks, MESH_THREADS, 0, s>>>(xq, nchunks, ns_dev, g, K1, K2, K3, Lx, \
                                                                               Ly, Lz, o);                             \
        break;
    switch (m->p.order) {
        PD_G(3) PD_G(4) PD_G(5) PD_G(6) PD_G(7) PD_G(8) PD_G(9) PD_G(10) PD_G(11) PD_G(12)
        default: break;
    }
#undef PD_G
}

int mesh_gather_join(pd_mesh *m, pd_cluster *c, const float4 *xq, const int *perm, const int *ns_dev, int nchunks,
                     float *fx, float *fy, float *fz, float *vx, float *vy, float *vz, const float *inv_mass,
                     float inv_mass_uniform, float half_dt, float *epot, float *vir6, float *vglobal6, const float *q,
                     float half_c_self, const float4 *extra, int energy, cudaStream_t s) {
    (void)q;
    GatherOut o;
    memset(&o, 0, sizeof o);
    o.fx = fx;
    o.fy = fy;
    o.fz = fz;
    o.epot = epot;
    o.vir6 = vir6;
    o.vx = vx;
    o.vy = vy;
    o.vz = vz;
    o.inv_mass = inv_mass;
    o.inv_mass_uniform = inv_mass_uniform;
    o.half_dt = half_dt;
    o.ids = perm;
    o.n_entries = nchunks * MESH_CHUNK;
    o.fc = c->fc;
    o.vc = c->vc;
    o.nslot = c->nslot;
    o.half_c_self = half_c_self;
    o.bg = m->bg;
    o.extra = extra;
    o.self_tab = m->self_tab;
    o.self_T = m->self_T;
    if (energy)
        launch_gather<2, true>(m, xq, nchunks, ns_dev, o, s);
    else
        launch_gather<2, false>(m, xq, nchunks, ns_dev, o, s);
    PD_LAUNCHED();
    if (energy) return mesh_store_virial(m, vglobal6, s);
    return PD_OK;
}

static void free_mesh(pd_mesh *m) {
    dfree(m->gridA);
    dfree(m->gridB);
    for (int d = 0; d < 3; ++d) dfree(m->field[d]);
    dfree(m->spec);
    dfree(m->scratch);
    dfree(m->G);
    dfree(m->Vc);
    dfree(m->acc);
    dfree(m->packed);
    dfree(m->self_tab);
    m->self_T = 0;
    if (m->plans) {
        cufftDestroy(m->fwd);
        cufftDestroy(m->bwd);
        m->plans = false;
    }
    if (m->work) cudaFree(m->work);
    m->work = nullptr;
}

}  // namespace pdb

extern "C" {

int pd_mesh_create(pd_mesh **out, const pd_mesh_params *p, const double box[3]) {
    PD_CHECK(out && p && box, PD_EINVAL, "pd_mesh_create: null argument");
    *out = nullptr;
    PD_CHECK(p->kind >= PD_MESH_SPME && p->kind <= PD_MESH_P3M_IK, PD_EINVAL, "Unknown influence kind %d.", p->kind);
    PD_CHECK(p->order >= 3 && p->order <= 12, PD_EINVAL,
             "B-spline assignment order must be between 3 and 12; got %d.", p->order);
    PD_CHECK(p->alias_order >= 0 && p->alias_order <= 6, PD_EINVAL, "alias_order must be between 0 and 6.");
    PD_CHECK(p->C > 0 && std::isfinite(p->C), PD_EINVAL, "coulomb constant must be finite and positive");
    PD_CHECK(p->alpha > 0 && std::isfinite(p->alpha), PD_EINVAL, "Ewald alpha must be finite and positive.");
    for (int d = 0; d < 3; ++d)
        PD_CHECK(p->mesh[d] >= p->order, PD_EINVAL, "Every mesh dimension must be at least the assignment order.");
    const long long nnodes = (long long)p->mesh[0] * p->mesh[1] * p->mesh[2];
    const long long nmodes = (long long)(p->mesh[0] / 2 + 1) * p->mesh[1] * p->mesh[2];
    PD_CHECK(nnodes < (1LL << 31) && nmodes < (1LL << 31), PD_EINVAL, "Mesh is too large for 32-bit grid indexing.");
    pd_mesh *m = new pd_mesh();
    m->p = *p;
    m->K1 = p->mesh[0];
    m->K2 = p->mesh[1];
    m->K3 = p->mesh[2];
    m->K1h = m->K1 / 2 + 1;
    m->nnodes = (int)nnodes;
    m->nmodes = (int)nmodes;
    const bool ik = p->kind == PD_MESH_P3M_IK;
    int rc;
    if ((rc = dalloc(&m->gridA, (size_t)nnodes)) || (rc = dalloc(&m->gridB, (size_t)nnodes)) ||
        (rc = dalloc(&m->spec, (size_t)nmodes)) || (rc = dalloc(&m->G, (size_t)nmodes)) ||
        (rc = dalloc(&m->Vc, (size_t)6 * nmodes)) || (rc = dalloc(&m->acc, 8))) {
        free_mesh(m);
        delete m;
        return rc;
    }
    if (ik) {
        if ((rc = dalloc(&m->field[0], (size_t)nnodes)) || (rc = dalloc(&m->field[1], (size_t)nnodes)) ||
            (rc = dalloc(&m->field[2], (size_t)nnodes)) || (rc = dalloc(&m->scratch, (size_t)nmodes))) {
            free_mesh(m);
            delete m;
            return rc;
        }
    }
    m->nmax_packed = ((std::max(p->nmax, 1) + MESH_CHUNK - 1) / MESH_CHUNK) * MESH_CHUNK;
    if ((rc = dalloc(&m->packed, (size_t)m->nmax_packed))) {
        free_mesh(m);
        delete m;
        return rc;
    }
    cudaMemset(m->gridA, 0, sizeof(float) * (size_t)nnodes);
    cudaMemset(m->gridB, 0, sizeof(float) * (size_t)nnodes);
    cudaMemset(m->acc, 0, 8 * sizeof(double));
    // cuFFT plans with a library-owned work area (Solver.jl:48-49: plan_rfft / plan_brfft)
    size_t ws1 = 0, ws2 = 0;
    bool ok = cufftCreate(&m->fwd) == CUFFT_SUCCESS && cufftCreate(&m->bwd) == CUFFT_SUCCESS;
    if (ok) {
        m->plans = true;
        ok = cufftSetAutoAllocation(m->fwd, 0) == CUFFT_SUCCESS && cufftSetAutoAllocation(m->bwd, 0) == CUFFT_SUCCESS &&
             cufftMakePlan3d(m->fwd, m->K3, m->K2, m->K1, CUFFT_R2C, &ws1) == CUFFT_SUCCESS &&
             cufftMakePlan3d(m->bwd, m->K3, m->K2, m->K1, CUFFT_C2R, &ws2) == CUFFT_SUCCESS;
    }
    if (!ok) {
        set_error("cuFFT plan creation failed for mesh %d x %d x %d", m->K1, m->K2, m->K3);
        free_mesh(m);
        delete m;
        return PD_ECUFFT;
    }
    m->work_size = std::max(ws1, ws2);
    if (m->work_size > 0 && cudaMalloc(&m->work, m->work_size) != cudaSuccess) {
        set_error("cuFFT work area allocation failed");
        free_mesh(m);
        delete m;
        return PD_ENOMEM;
    }
    cufftSetWorkArea(m->fwd, m->work);
    cufftSetWorkArea(m->bwd, m->work);
    if ((rc = pd_mesh_set_box(m, box))) {
        free_mesh(m);
        delete m;
        return rc;
    }
    *out = m;
    return PD_OK;
}

int pd_mesh_destroy(pd_mesh *m) {
    if (!m) return PD_OK;
    free_mesh(m);
    delete m;
    return PD_OK;
}

int pd_mesh_set_box(pd_mesh *m, const double box[3]) {
    PD_CHECK(m && box, PD_EINVAL, "pd_mesh_set_box: null argument");
    for (int d = 0; d < 3; ++d)
        PD_CHECK(std::isfinite(box[d]) && box[d] > 0, PD_EINVAL, "box lengths must be finite and positive");
    for (int d = 0; d < 3; ++d) m->box[d] = box[d];
    int rc = compute_influence(m);
    if (rc) return rc;
    refresh_background(m);
    return compute_self_table(m);
}

int pd_mesh_set_self_force_removal(pd_mesh *m, int table_size) {
    PD_CHECK(m, PD_EINVAL, "pd_mesh_set_self_force_removal: null handle");
    PD_CHECK(table_size == 0 || (table_size >= 4 && table_size <= 64), PD_EINVAL,
             "self-force table size must be 0 (off) or 4..64; got %d", table_size);
    PD_CHECK(table_size == 0 || m->p.kind != PD_MESH_P3M_IK, PD_ENOTSUP,
             "self-force removal needs analytic differentiation (SPME or P3M-AD)");
    dfree(m->self_tab);
    m->self_T = 0;
    ++m->epoch;   // captured steps hold the old table pointer
    if (table_size == 0) return PD_OK;
    int rc = dalloc(&m->self_tab, (size_t)table_size * table_size * table_size);
    if (rc) return rc;
    m->self_T = table_size;
    return compute_self_table(m);
}

int pd_mesh_self_force_table(pd_mesh *m, float *out4, int *table_size) {
    PD_CHECK(m, PD_EINVAL, "pd_mesh_self_force_table: null handle");
    if (table_size) *table_size = m->self_T;
    if (out4 && m->self_tab)
        PD_CUDA(cudaMemcpy(out4, m->self_tab, sizeof(float4) * (size_t)m->self_T * m->self_T * m->self_T,
                           cudaMemcpyDeviceToHost));
    return PD_OK;
}

int pd_mesh_transform(pd_mesh *m, const float *x, const float *y, const float *z, const float *q, const int *order,
                      int n, int energy, pd_stream_t s) {
    PD_CHECK(m && x && y && z && q, PD_EINVAL, "pd_mesh_transform: null argument");
    PD_CHECK(n >= 0, PD_EINVAL, "pd_mesh_transform: negative particle count");
    cudaStream_t st = (cudaStream_t)s;
    const int nchunks = (n + MESH_CHUNK - 1) / MESH_CHUNK;
    const int ntot = nchunks * MESH_CHUNK;
    PD_CHECK(ntot <= m->nmax_packed, PD_EINVAL, "pd_mesh_transform: %d particles exceed nmax = %d of this solver", n,
             m->p.nmax);
    if (ntot > 0) {
        k_pack_order<<<(ntot + 255) / 256, 256, 0, st>>>(x, y, z, q, order, n, ntot, m->packed);
        PD_LAUNCHED();
    }
    return mesh_transform_packed(m, m->packed, nchunks, nullptr, energy, st);
}

int pd_mesh_gather(pd_mesh *m, const float *x, const float *y, const float *z, const float *q, const int *order, int n,
                   float *fx, float *fy, float *fz, float *epot, float *vglobal6, int energy, int set, pd_stream_t s) {
    PD_CHECK(m && x && y && z && q && fx && fy && fz, PD_EINVAL, "pd_mesh_gather: null argument");
    PD_CHECK(!energy || epot, PD_EINVAL, "pd_mesh_gather: energy needs epot");
    cudaStream_t st = (cudaStream_t)s;
    const int nchunks = (n + MESH_CHUNK - 1) / MESH_CHUNK;
    PD_CHECK(m->nmax_packed >= nchunks * MESH_CHUNK, PD_ESTATE, "pd_mesh_gather: no transform of %d particles", n);
    // the packed staging buffer holds the particles of the last transform; refresh it (positions may differ)
    if (n > 0) {
        k_pack_order<<<(nchunks * MESH_CHUNK + 255) / 256, 256, 0, st>>>(x, y, z, q, order, n, nchunks * MESH_CHUNK,
                                                                         m->packed);
        PD_LAUNCHED();
    }
    if (n > 0) {
        GatherOut o;
        memset(&o, 0, sizeof o);
        o.fx = fx;
        o.fy = fy;
        o.fz = fz;
        o.epot = epot;
        o.ids = order;
        o.n_entries = n;
        o.bg = m->bg;
        o.self_tab = m->self_tab;
        o.self_T = m->self_T;
        if (set) {
            if (energy) launch_gather<1, true>(m, m->packed, nchunks, nullptr, o, st);
            else launch_gather<1, false>(m, m->packed, nchunks, nullptr, o, st);
        } else {
            if (energy) launch_gather<0, true>(m, m->packed, nchunks, nullptr, o, st);
            else launch_gather<0, false>(m, m->packed, nchunks, nullptr, o, st);
        }
        PD_LAUNCHED();
    }
    if (energy) return mesh_store_virial(m, vglobal6, st);
    return PD_OK;
}

int pd_mesh_energy(pd_mesh *m, double out7[7], pd_stream_t s) {
    PD_CHECK(m && out7, PD_EINVAL, "pd_mesh_energy: null argument");
    PD_CUDA(cudaMemcpyAsync(out7, m->acc, 7 * sizeof(double), cudaMemcpyDeviceToHost, (cudaStream_t)s));
    PD_CUDA(cudaStreamSynchronize((cudaStream_t)s));
    return PD_OK;
}

int pd_mesh_influence(pd_mesh *m, float *G, float *Vc) {
    PD_CHECK(m, PD_EINVAL, "pd_mesh_influence: null handle");
    if (G) PD_CUDA(cudaMemcpy(G, m->G, sizeof(float) * m->nmodes, cudaMemcpyDeviceToHost));
    if (Vc) PD_CUDA(cudaMemcpy(Vc, m->Vc, sizeof(float) * 6 * (size_t)m->nmodes, cudaMemcpyDeviceToHost));
    return PD_OK;
}

int pd_mesh_dims(pd_mesh *m, int mesh[3], int *nmodes) {
    PD_CHECK(m, PD_EINVAL, "pd_mesh_dims: null handle");
    if (mesh) {
        mesh[0] = m->K1;
        mesh[1] = m->K2;
        mesh[2] = m->K3;
    }
    if (nmodes) *nmodes = m->nmodes;
    return PD_OK;
}

}  // extern "C"
