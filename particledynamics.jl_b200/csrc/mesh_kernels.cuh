// Device code of the mesh engine shared by its translation units: the window stencils, the chunk
// bricks, the spread and gather kernels and their launchers.  The launchers are instantiated in
// separate translation units (mesh_spread.cu, mesh_gather_*.cu) so that the many (order, mode,
// window) variants compile in parallel.
//
// Layout: particles are processed in chunks of 64 consecutive entries of a spatially sorted
// sequence (a super-cluster of the cluster list).  A chunk's stencils cover a small brick of the
// mesh; the spread accumulates the chunk into that brick in shared memory and adds the brick to
// the global grid once (one coalesced reduction per brick node instead of P^3 scattered atomics
// per particle), and the gather stages the brick of the potential in shared memory before every
// particle reads its P^3 nodes.  A chunk whose brick exceeds the shared-memory budget falls back
// to direct global accumulation.
#pragma once

#include <cuda_runtime.h>

#include "common.cuh"
#include "internal.hpp"

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

// Window of a mesh: the B-spline of order P (WIN_BSPLINE) or the prolate window of width P
// (WIN_PROLATE), W(x) = psi(2x/P) - psi(1) centred on the particle (ProlateWindow, Windows.jl:26-54),
// evaluated as one polynomial per stencil node.
enum { WIN_BSPLINE = 0, WIN_PROLATE = 1 };

// Node polynomials of a prolate window (ProlatePolyStencil, Windows.jl:63-72): node h < H = ceil(P/2)
// carries W_h(tau) = sum_k c[k * H + h] tau^k, tau the offset of the particle from the centre of its
// cell; the other nodes are the mirror images, W_{P-1-h}(tau) = W_h(-tau).  The host fits the
// coefficients to the round-off of FP32 (prolate_node_polynomials, Windows.jl:99-135).
struct WindowPoly {
    const float *c;   // (deg + 1) x H, device
    int deg;
};

// First node and the weights (and du-derivatives) of the prolate stencil at grid coordinate u:
// _prolate_cell (Windows.jl:158-167) for the base node and tau, then one Horner pass per node
// giving the value and the tau-derivative of its polynomial (window_stencil(::ProlatePolyStencil),
// Windows.jl:224-243).
template <int P>
__device__ __forceinline__ int prolate_stencil(float u, float *w, float *dw, const WindowPoly &wp) {
    constexpr int H = (P + 1) / 2;
    int k0;
    float tau;
    if (P % 2 == 0) {
        const float fl = floorf(u);
        k0 = (int)fl - (P / 2 - 1);
        tau = (u - fl) - 0.5f;
    } else {
        const float fl = floorf(u + 0.5f);
        k0 = (int)fl - (P - 1) / 2;
        tau = u - fl;
    }
    const int D = wp.deg;
#pragma unroll
    for (int j = 0; j < P; ++j) {
        const int hh = j < H ? j : P - 1 - j;
        const float t = j < H ? tau : -tau;
        float p = __ldg(wp.c + D * H + hh), d = 0.f;
        for (int k = D - 1; k >= 0; --k) {
            d = fmaf(d, t, p);
            p = fmaf(p, t, __ldg(wp.c + k * H + hh));
        }
        w[j] = p;
        if (dw) dw[j] = j < H ? d : -d;
    }
    return k0;
}

template <int P, int WIN>
__device__ __forceinline__ int window_stencil(float u, float *w, float *dw, const WindowPoly &wp) {
    if (WIN == WIN_PROLATE) return prolate_stencil<P>(u, w, dw, wp);
    return bspline<P>(u, w, dw);
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

// NT: threads of the CTA that moves the brick (two per particle of the chunk); TILE: floats of the
// shared brick.
template <int P, int NT = MESH_THREADS, int TILE = TILE_MAX>
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
        b.fits = nodes <= TILE && b.e1 <= NT && (!b.vec || b.e1 <= K1) &&
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
template <int NT = MESH_THREADS, typename F>
__device__ __forceinline__ void for_brick(const Brick &b, const unsigned *rowbase, int K1, F &&visit) {
    const int per = b.vec ? 4 : 1;
    const int nv = b.e1 / per;
    if (nv == 0) return;
    const int rpi = NT / nv;
    const int t = threadIdx.x;
    const int r0 = t / nv, v = t - r0 * nv;
    if (r0 >= rpi) return;
    const int x0 = wrap_node(b.o1 + per * v, K1);
    const int nrows = b.e2 * b.e3;
    for (int r = r0; r < nrows; r += rpi) visit(r * nv + v, (size_t)rowbase[r] + x0);
}

// z planes of a particle's stencil taken by its thread h of TP: the two halves of the stencil (TP = 2),
// or every TP-th plane (TP = 4).
template <int P, int TP>
__device__ __forceinline__ bool my_plane(int j3, int h) {
    return TP == 2 ? ((j3 < (P + 1) / 2) == (h == 0)) : (j3 % TP == h);
}

// Spread of one chunk of CH packed (x, y, z, q) particles into `grid` (the charge assignment of
// _spread_lines_kernel!, MeshKernels.jl:247-276), by a CTA of TP CH threads: each particle's TP
// threads share the z planes of its stencil.
template <int P, int WIN, int CH, int TILE = TILE_MAX, int TP = 2>
__device__ __forceinline__ void spread_chunk(const float4 *__restrict__ chunk, float *__restrict__ grid, int K1,
                                             int K2, int K3, float Lx, float Ly, float Lz, const WindowPoly &wp) {
    constexpr int NT = TP * CH;
    __shared__ __align__(16) float tile[TILE];
    __shared__ unsigned rowbase[ROWS_MAX];
    __shared__ int sm[10];
    const int t = threadIdx.x, p = t & (CH - 1), h = t / CH;
    const float4 v = chunk[p];
    const bool valid = v.w != 0.f && isfinite(v.x) && isfinite(v.y) && isfinite(v.z);
    float w1[P], w2[P], w3[P];
    int k1 = 0, k2 = 0, k3 = 0;
    if (valid) {
        k1 = window_stencil<P, WIN>(grid_coordinate(v.x, Lx, K1), w1, nullptr, wp);
        k2 = window_stencil<P, WIN>(grid_coordinate(v.y, Ly, K2), w2, nullptr, wp);
        k3 = window_stencil<P, WIN>(grid_coordinate(v.z, Lz, K3), w3, nullptr, wp);
    }
    int d1 = 0, d2 = 0, d3 = 0;
    Brick b;
    // both halves of a particle take part (their min/max contributions are identical)
    chunk_brick<P, NT, TILE>(valid, k1, k2, k3, K1, K2, K3, d1, d2, d3, b, sm, rowbase);

    if (b.fits) {
        // The brick accumulates in 32-bit fixed point: integer shared-memory reductions are native
        // (a float reduction is not), and integer sums are exact, so a chunk's brick does not depend
        // on the order of its atomics.  The window weights lie in [0, 1], so no node of the brick
        // exceeds the chunk's sum of |q| in magnitude; the scale is the largest power of two that
        // keeps that sum below 2^30.  Each contribution rounds to a step of at most sum|q| / 2^30.
        __shared__ float s_qabs[NT / 32];
        float qa = (valid && h == 0) ? fabsf(v.w) : 0.f;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) qa += __shfl_xor_sync(0xffffffffu, qa, off);
        if ((t & 31) == 0) s_qabs[t >> 5] = qa;
        const int nb4 = (b.e1 * b.e2 * b.e3 + 3) >> 2;
        int4 *itile4 = reinterpret_cast<int4 *>(tile);
        int *itile = reinterpret_cast<int *>(tile);
        for (int k = t; k < nb4; k += NT) itile4[k] = make_int4(0, 0, 0, 0);
        __syncthreads();
        float qsum = 0.f;
#pragma unroll
        for (int k = 0; k < NT / 32; ++k) qsum += s_qabs[k];
        qsum = fmaxf(qsum, 1e-30f);
        const int ex = min(30 - (int)ceilf(log2f(qsum)), 126);   // qsum * 2^ex <= 2^30, 2^ex finite
        const float scale = ldexpf(1.f, ex), inv_scale = ldexpf(1.f, -ex);
        if (valid) {
            const float qs = v.w * scale;
#pragma unroll
            for (int j3 = 0; j3 < P; ++j3) {   // this half's z nodes only (warp-uniform test)
            if (!my_plane<P, TP>(j3, h)) continue;
                const float q3 = qs * w3[j3];
#pragma unroll
                for (int j2 = 0; j2 < P; ++j2) {
                    const float q23 = q3 * w2[j2];
                    int *row = itile + ((d3 + j3) * b.e2 + (d2 + j2)) * b.e1 + d1;
#pragma unroll
                    for (int j1 = 0; j1 < P; ++j1) atomicAdd(row + j1, __float2int_rn(q23 * w1[j1]));
                }
            }
        }
        __syncthreads();
        if (b.vec) {
            for_brick<NT>(b, rowbase, K1, [&](int kt, size_t kg) {
                const int4 iv = itile4[kt];
                if (iv.x != 0 || iv.y != 0 || iv.z != 0 || iv.w != 0)
                    red_add_v4(grid + kg, (float)iv.x * inv_scale, (float)iv.y * inv_scale, (float)iv.z * inv_scale,
                               (float)iv.w * inv_scale);
            });
        } else {
            for_brick<NT>(b, rowbase, K1, [&](int kt, size_t kg) {
                const int iv = itile[kt];
                if (iv != 0) red_add(grid + kg, (float)iv * inv_scale);
            });
        }
    } else if (valid) {
#pragma unroll
        for (int j3 = 0; j3 < P; ++j3) {   // this half's z nodes only (warp-uniform test)
            if (!my_plane<P, TP>(j3, h)) continue;
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

// Spread of chunks of packed (x, y, z, q) particles.  nchunk_dev (optional) holds the number of
// active chunks (the cluster list's super-cluster count).
template <int P, int WIN>
__global__ void __launch_bounds__(MESH_THREADS, MESH_CTAS_PER_SM) k_spread(const float4 *__restrict__ xq, int nchunks,
                                                         const int *__restrict__ nchunk_dev, float *__restrict__ grid,
                                                         int K1, int K2, int K3, float Lx, float Ly, float Lz,
                                                         WindowPoly wp) {
    const int c = blockIdx.x;
    if (nchunk_dev && c >= *nchunk_dev) return;
    if (c >= nchunks) return;
    spread_chunk<P, WIN, MESH_CHUNK>(xq + (size_t)c * MESH_CHUNK, grid, K1, K2, K3, Lx, Ly, Lz, wp);
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
    WindowPoly wp;           // prolate window: node polynomials
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
template <int P, int MODE, bool ENERGY, bool IK, int WIN>   // MODE 0: add, 1: set, 2: join (+ kick)
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
        k1 = window_stencil<P, WIN>(u1, w1, IK ? nullptr : g1, o.wp);
        k2 = window_stencil<P, WIN>(u2, w2, IK ? nullptr : g2, o.wp);
        k3 = window_stencil<P, WIN>(u3, w3, IK ? nullptr : g3, o.wp);
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

// ------------------------------------------------------------------ launchers
// Mesh orders 3..12 for both windows.  Each (window, differentiation, mode) launcher is instantiated
// once, in its own translation unit (extern templates below).

constexpr int MESH_ORDER_MIN = 3, MESH_ORDER_MAX = 12;

#define PD_MESH_ORDER_CASES(X) X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10) X(11) X(12)

template <int WIN>
void launch_spread_t(int P, const float4 *xq, int nchunks, const int *ns_dev, float *grid, int K1, int K2, int K3,
                     float Lx, float Ly, float Lz, const WindowPoly &wp, cudaStream_t s) {
    switch (P) {
#define PD_SPREAD_CASE(PP)                                                                                         \
    case PP:                                                                                                       \
        k_spread<PP, WIN><<<nchunks, MESH_THREADS, 0, s>>>(xq, nchunks, ns_dev, grid, K1, K2, K3, Lx, Ly, Lz, wp); \
        break;
        PD_MESH_ORDER_CASES(PD_SPREAD_CASE)
#undef PD_SPREAD_CASE
        default: break;
    }
}

// MODE 0 (add), 1 (set) or 2 (the join of the step).
template <int WIN, bool IK, int MODE>
void launch_gather_t(int P, bool energy, const float4 *xq, int nchunks, const int *ns_dev, const GatherGrids &g,
                     int K1, int K2, int K3, float Lx, float Ly, float Lz, const GatherOut &o, cudaStream_t s) {
    switch (P) {
#define PD_GATHER_CASE(PP)                                                                                          \
    case PP:                                                                                                        \
        if (energy)                                                                                                 \
            k_gather<PP, MODE, true, IK, WIN><<<nchunks, MESH_THREADS, 0, s>>>(xq, nchunks, ns_dev, g, K1, K2, K3, Lx, \
                                                                               Ly, Lz, o);                          \
        else                                                                                                        \
            k_gather<PP, MODE, false, IK, WIN><<<nchunks, MESH_THREADS, 0, s>>>(xq, nchunks, ns_dev, g, K1, K2, K3,    \
                                                                                Lx, Ly, Lz, o);                     \
        break;
        PD_MESH_ORDER_CASES(PD_GATHER_CASE)
#undef PD_GATHER_CASE
        default: break;
    }
}

#define PD_GATHER_LAUNCHER(WIN, IK, MODE)                                                                          \
    template void launch_gather_t<WIN, IK, MODE>(int, bool, const float4 *, int, const int *, const GatherGrids &, \
                                                 int, int, int, float, float, float, const GatherOut &, cudaStream_t)
#define PD_SPREAD_LAUNCHER(WIN)                                                                                 \
    template void launch_spread_t<WIN>(int, const float4 *, int, const int *, float *, int, int, int, float, float, \
                                       float, const WindowPoly &, cudaStream_t)

extern PD_SPREAD_LAUNCHER(WIN_BSPLINE);
extern PD_SPREAD_LAUNCHER(WIN_PROLATE);
extern PD_GATHER_LAUNCHER(WIN_BSPLINE, false, 0);
extern PD_GATHER_LAUNCHER(WIN_BSPLINE, false, 1);
extern PD_GATHER_LAUNCHER(WIN_BSPLINE, false, 2);
extern PD_GATHER_LAUNCHER(WIN_BSPLINE, true, 0);
extern PD_GATHER_LAUNCHER(WIN_BSPLINE, true, 1);
extern PD_GATHER_LAUNCHER(WIN_BSPLINE, true, 2);
extern PD_GATHER_LAUNCHER(WIN_PROLATE, false, 0);
extern PD_GATHER_LAUNCHER(WIN_PROLATE, false, 1);
extern PD_GATHER_LAUNCHER(WIN_PROLATE, false, 2);

}  // namespace pdb
