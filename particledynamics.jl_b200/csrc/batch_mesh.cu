// Mesh of batched charged replicas: one launch per stage over every replica's particles and
// grids (the reference runs one ElectrostaticsSolver per system, src/electrostatics/Solver.jl:305-393,
// through mesh_transform! and mesh_gather!).
//
// Every replica has its own mesh (its box at the shared mesh spacing), its own influence function
// (computed in FP64 by the single-system mesh setup) and its own slice of the concatenated grids.
// The replicas' particles are taken in the batched cell order (the ELL route's counting sort by
// cell, replica by replica), cut into chunks of `chunk` consecutive positions of one replica; a
// chunk of cell-sorted particles lies in about two cells, so its B-spline stencils cover a small
// brick that the spread accumulates in shared memory (32-bit fixed point, as the single-system
// spread) and the gather stages before every particle reads its P^3 nodes.  The tile (32 or 64
// particles, with 2 or 4 threads per particle sharing its z planes) is the autotuner's spread tile.  The transforms of the mesh sizes
// run on several streams at once (each size's batched plan is small; one after another they would
// leave most of the GPU idle).
//
// Stages: k_bmesh_pack (coordinates and charges of the step, for the pair kernel and the chunks),
// k_bspread, the batched R2C transforms (one cuFFT plan per mesh size, outside this file), k_bsolve
// (spec *= G over all modes; the charge grids are cleared for the next step), the batched C2R
// transforms, k_bgather (the AD gather joined with the pair forces, the closing half kick).
#include "ell_common.cuh"
#include "internal.hpp"
#include "mesh_kernels.cuh"

namespace pdb {

// Shared brick of the batched spread and gather (45 KB of static shared memory): a tile of cell-sorted
// ions spans one or two cells of at least the list radius, a larger brick than a single system's
// super-cluster, so the batched kernels trade occupancy (4 CTAs per SM) for bricks that fit.
constexpr int BTILE = 11264;
constexpr int BMESH_CTAS_PER_SM = 4;

__global__ void k_bmesh_pack(const float *__restrict__ x, const float *__restrict__ y, const float *__restrict__ z,
                             const float *__restrict__ q, const int *__restrict__ sorted,
                             const int *__restrict__ slot_src, int nslots, float4 *__restrict__ xq,
                             float4 *__restrict__ mq, int *__restrict__ mid, const long long *__restrict__ st) {
    if (st[E_VALID] == 0) return;
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nslots) return;
    const int k = slot_src[s];
    if (k < 0) {
        mq[s] = make_float4(0.f, 0.f, 0.f, 0.f);
        mid[s] = -1;
        return;
    }
    const int i = sorted[k];
    const float4 v = make_float4(x[i], y[i], z[i], q[i]);
    xq[k] = v;
    mq[s] = v;
    mid[s] = i;
}

template <int P, int CH, int TP>
__global__ void __launch_bounds__(TP * CH, BMESH_CTAS_PER_SM) k_bspread(const float4 *__restrict__ mq,
                                                                      const int *__restrict__ chunk_rep,
                                                                      const BMeshRep *__restrict__ reps,
                                                                      float *__restrict__ gridA,
                                                                      const long long *__restrict__ st) {
    if (st[E_VALID] == 0) return;
    const int c = blockIdx.x;
    const BMeshRep R = reps[chunk_rep[c]];
    spread_chunk<P, WIN_BSPLINE, CH, BTILE, TP>(mq + (size_t)c * CH, gridA + R.grid, R.K1, R.K2, R.K3, R.Lx, R.Ly, R.Lz,
                                     WindowPoly{nullptr, 0});
}

// spec *= G (the influence multiply of _solve_kernel!, MeshKernels.jl:57-81) over the concatenated
// spectra; two nodes of the concatenated charge grids are cleared per mode (the host checks that
// the modes cover the grids).
__global__ void __launch_bounds__(256) k_bsolve(float2 *__restrict__ spec, const float *__restrict__ G,
                                                long long nmodes, float *__restrict__ gridA, long long nnodes,
                                                const long long *__restrict__ st) {
    if (st[E_VALID] == 0) return;
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx < nmodes) {
        const float2 zz = spec[idx];
        const float g = G[idx];
        spec[idx] = make_float2(zz.x * g, zz.y * g);
    }
    const long long n0 = 2 * idx;
    if (n0 + 1 < nnodes) {
        reinterpret_cast<float2 *>(gridA)[idx] = make_float2(0.f, 0.f);
    } else if (n0 < nnodes) {
        gridA[n0] = 0.f;
    }
}

// AD gather of one chunk (the sums of _gather_ad_lines_sums, MeshKernels.jl:281-311, and
// _gather_ad_lines_kernel!, :313-333) from the replica's potential grid, joined with the pair force
// already stored for the particle: F = F_pair - q grad(phi) K / L, then the closing half kick.  Each
// particle's TP threads share the z planes of its stencil.
template <int P, int CH, int TP, bool ENERGY>
__global__ void __launch_bounds__(TP * CH, BMESH_CTAS_PER_SM) k_bgather(const float4 *__restrict__ mq,
                                                                      const int *__restrict__ mid,
                                                                      const int *__restrict__ chunk_rep,
                                                                      const BMeshRep *__restrict__ reps,
                                                                      const float *__restrict__ gridB,
                                                                      float *__restrict__ fx, float *__restrict__ fy,
                                                                      float *__restrict__ fz,
                                                                      float *__restrict__ epot, BMeshKick kick,
                                                                      float half_c_self,
                                                                      const long long *__restrict__ st) {
    if (st[E_VALID] == 0) return;
    constexpr int NT = TP * CH;
    const int c = blockIdx.x;
    const BMeshRep R = reps[chunk_rep[c]];
    const float *grid = gridB + R.grid;
    const int K1 = R.K1, K2 = R.K2, K3 = R.K3;
    __shared__ __align__(16) float tile[BTILE];
    __shared__ unsigned rowbase[ROWS_MAX];
    __shared__ int sm[10];
    const int t = threadIdx.x, p = t & (CH - 1), h = t / CH;
    const int e = c * CH + p;
    const float4 v = mq[e];
    const int id = mid[e];
    const bool charged = id >= 0 && v.w != 0.f && isfinite(v.x) && isfinite(v.y) && isfinite(v.z);
    // the pair force and the velocity are fetched now, so that their latency overlaps the brick
    float fpx = 0.f, fpy = 0.f, fpz = 0.f, pvx = 0.f, pvy = 0.f, pvz = 0.f, pim = 0.f, ep = 0.f;
    if (h == 0 && id >= 0) {
        fpx = fx[id];
        fpy = fy[id];
        fpz = fz[id];
        if (ENERGY) ep = epot[id];
        if (kick.on) {
            pvx = kick.vx[id];
            pvy = kick.vy[id];
            pvz = kick.vz[id];
            pim = kick.inv_mass[id];
        }
    }
    float w1[P], w2[P], w3[P], g1[P], g2[P], g3[P];
    int k1 = 0, k2 = 0, k3 = 0;
    if (charged) {
        k1 = bspline<P>(grid_coordinate(v.x, R.Lx, K1), w1, g1);
        k2 = bspline<P>(grid_coordinate(v.y, R.Ly, K2), w2, g2);
        k3 = bspline<P>(grid_coordinate(v.z, R.Lz, K3), w3, g3);
    }
    int d1 = 0, d2 = 0, d3 = 0;
    Brick b;
    chunk_brick<P, NT, BTILE>(charged, k1, k2, k3, K1, K2, K3, d1, d2, d3, b, sm, rowbase);
    float phi = 0.f, gx = 0.f, gy = 0.f, gz = 0.f;
    if (b.fits) {
        if (b.vec) {
            float4 *tile4 = reinterpret_cast<float4 *>(tile);
            for_brick<NT>(b, rowbase, K1, [&](int kt, size_t kg) {
                tile4[kt] = __ldg(reinterpret_cast<const float4 *>(grid + kg));
            });
        } else {
            for_brick<NT>(b, rowbase, K1, [&](int kt, size_t kg) { tile[kt] = __ldg(grid + kg); });
        }
        __syncthreads();
        if (charged) {
#pragma unroll
            for (int j3 = 0; j3 < P; ++j3) {   // this thread's z planes only (warp-uniform test)
                if (!my_plane<P, TP>(j3, h)) continue;
                float s0 = 0.f, s1 = 0.f, s2 = 0.f;
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
#pragma unroll
        for (int j3 = 0; j3 < P; ++j3) {
            if (!my_plane<P, TP>(j3, h)) continue;
            const int n3 = wrap_node(k3 + j3, K3);
            float s0 = 0.f, s1 = 0.f, s2 = 0.f;
#pragma unroll
            for (int j2 = 0; j2 < P; ++j2) {
                const int n2 = wrap_node(k2 + j2, K2);
                float a0 = 0.f, a1 = 0.f;
#pragma unroll
                for (int j1 = 0; j1 < P; ++j1) {
                    const float cval = __ldg(grid + ((size_t)n3 * K2 + n2) * K1 + wrap_node(k1 + j1, K1));
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
    // the partial sums of threads h > 0 meet in the brick's shared memory once every thread is done with it
    __syncthreads();
    float4 *part = reinterpret_cast<float4 *>(tile);   // (TP - 1) x CH, far below the brick's size
    if (h > 0) part[(h - 1) * CH + p] = make_float4(phi, gx, gy, gz);
    __syncthreads();
    if (h > 0 || id < 0) return;
#pragma unroll
    for (int k = 0; k < TP - 1; ++k) {
        const float4 o = part[k * CH + p];
        phi += o.x;
        gx += o.y;
        gy += o.z;
        gz += o.w;
    }
    const float qi = v.w;
    float Fx = fpx, Fy = fpy, Fz = fpz;
    if (charged) {
        Fx -= qi * gx * ((float)K1 / R.Lx);
        Fy -= qi * gy * ((float)K2 / R.Ly);
        Fz -= qi * gz * ((float)K3 / R.Lz);
    }
    fx[id] = Fx;
    fy[id] = Fy;
    fz[id] = Fz;
    if (kick.on) {
        const float cm = kick.half_dt * pim;
        kick.vx[id] = fmaf(cm, Fx, pvx);
        kick.vy[id] = fmaf(cm, Fy, pvy);
        kick.vz[id] = fmaf(cm, Fz, pvz);
    }
    if (ENERGY) epot[id] = ep + (charged ? 0.5f * qi * phi : 0.f) - half_c_self * qi * qi;
}

int bmesh_pack_launch(const BMeshView &v, const float *x, const float *y, const float *z, const float *q,
                      const int *sorted, float4 *xq, const long long *st, cudaStream_t s) {
    const int nslots = v.nchunk * v.chunk;
    k_bmesh_pack<<<(nslots + 255) / 256, 256, 0, s>>>(x, y, z, q, sorted, v.slot_src, nslots, xq, v.mq, v.mid, st);
    PD_LAUNCHED();
    return PD_OK;
}

template <int P>
static void spread_p(const BMeshView &v, const long long *st, cudaStream_t s) {
    if (v.chunk == 32)
        k_bspread<P, 32, 2><<<v.nchunk, 64, 0, s>>>(v.mq, v.chunk_rep, v.reps, v.gridA, st);
    else if (v.tpi == 4)
        k_bspread<P, 64, 4><<<v.nchunk, 256, 0, s>>>(v.mq, v.chunk_rep, v.reps, v.gridA, st);
    else
        k_bspread<P, 64, 2><<<v.nchunk, 128, 0, s>>>(v.mq, v.chunk_rep, v.reps, v.gridA, st);
}

int bmesh_spread_launch(const BMeshView &v, const long long *st, cudaStream_t s) {
    PD_CHECK(v.chunk == 32 || v.chunk == 64, PD_EINVAL, "batched spread: chunk must be 32 or 64");
    switch (v.order) {
        case 4: spread_p<4>(v, st, s); break;
        case 5: spread_p<5>(v, st, s); break;
        case 6: spread_p<6>(v, st, s); break;
        default: PD_CHECK(false, PD_EINVAL, "batched mesh: order %d (4, 5 or 6)", v.order);
    }
    PD_LAUNCHED();
    return PD_OK;
}

int bmesh_solve_launch(const BMeshView &v, const long long *st, cudaStream_t s) {
    const long long blocks = (v.total_modes + 255) / 256;
    k_bsolve<<<(unsigned)blocks, 256, 0, s>>>(v.spec, v.G, v.total_modes, v.gridA, v.total_nodes, st);
    PD_LAUNCHED();
    return PD_OK;
}

template <int P, int CH, int TP>
static void gather_pc(const BMeshView &v, float *fx, float *fy, float *fz, float *epot, int energy,
                      const BMeshKick &kick, float half_c_self, const long long *st, cudaStream_t s) {
    if (energy)
        k_bgather<P, CH, TP, true><<<v.nchunk, TP * CH, 0, s>>>(v.mq, v.mid, v.chunk_rep, v.reps, v.gridB, fx, fy,
                                                                fz, epot, kick, half_c_self, st);
    else
        k_bgather<P, CH, TP, false><<<v.nchunk, TP * CH, 0, s>>>(v.mq, v.mid, v.chunk_rep, v.reps, v.gridB, fx, fy,
                                                                 fz, epot, kick, half_c_self, st);
}

template <int P>
static void gather_p(const BMeshView &v, float *fx, float *fy, float *fz, float *epot, int energy,
                     const BMeshKick &kick, float half_c_self, const long long *st, cudaStream_t s) {
    if (v.chunk == 32)
        gather_pc<P, 32, 2>(v, fx, fy, fz, epot, energy, kick, half_c_self, st, s);
    else if (v.tpi == 4)
        gather_pc<P, 64, 4>(v, fx, fy, fz, epot, energy, kick, half_c_self, st, s);
    else
        gather_pc<P, 64, 2>(v, fx, fy, fz, epot, energy, kick, half_c_self, st, s);
}

int bmesh_gather_launch(const BMeshView &v, float *fx, float *fy, float *fz, float *epot, int energy,
                        const BMeshKick &kick, float half_c_self, const long long *st, cudaStream_t s) {
    PD_CHECK(v.chunk == 32 || v.chunk == 64, PD_EINVAL, "batched gather: chunk must be 32 or 64");
    switch (v.order) {
        case 4: gather_p<4>(v, fx, fy, fz, epot, energy, kick, half_c_self, st, s); break;
        case 5: gather_p<5>(v, fx, fy, fz, epot, energy, kick, half_c_self, st, s); break;
        case 6: gather_p<6>(v, fx, fy, fz, epot, energy, kick, half_c_self, st, s); break;
        default: PD_CHECK(false, PD_EINVAL, "batched mesh: order %d (4, 5 or 6)", v.order);
    }
    PD_LAUNCHED();
    return PD_OK;
}

}  // namespace pdb
