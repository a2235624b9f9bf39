// Fused cluster-pair force kernel of libpdb200 (included by the units that instantiate it: the
// plain pass and the pass with exclusion masks compile in parallel).
//
// Semantics: _cluster_pair_kernel! of
// src/clusterpairs/Kernels.jl (ParticleDynamics.jl) with the pair physics of
// pair_force (src/clusterpairs/PairFunctor.jl:127-156).  Layout of this
// library: one CTA of 1, 2 or 4 warps (two by default; the tuned shape) per super-cluster part; thread
// (ti, tj) = (tid & 7, tid >> 3) pairs i-atom ti of each of the 8 i-clusters
// with j-atom tj of the current j-cluster.  The 64 i-atoms live in shared
// memory as packed float4 (x, y, z, C q); j-atoms are read as one float4 each,
// with the next entry's j-atom prefetched into registers while the current
// entry is evaluated.  j-forces are reduced over the 8 ti lanes by shuffles and
// added with three fence-free reductions; i-forces stay in registers and are
// reduced once per CTA.
#pragma once
#include "common.cuh"
#include "internal.hpp"

namespace pdb {

// (x, y, z) summed over the 8 lanes of a ti group; lanes ti = 0, 1, 2 return the
// x, y, z totals (_reduce3, Kernels.jl:20-30).
__device__ __forceinline__ float reduce3(float fx, float fy, float fz, int ti) {
    fx += __shfl_down_sync(0xffffffffu, fx, 1);
    fy += __shfl_up_sync(0xffffffffu, fy, 1);
    fz += __shfl_down_sync(0xffffffffu, fz, 1);
    fx = (ti & 1) ? fy : fx;
    fx += __shfl_down_sync(0xffffffffu, fx, 2);
    fz += __shfl_up_sync(0xffffffffu, fz, 2);
    fx = (ti & 2) ? fz : fx;
    fx += __shfl_down_sync(0xffffffffu, fx, 4);
    return fx;
}

__device__ __forceinline__ float sum8(float v) {
    v += __shfl_down_sync(0xffffffffu, v, 4);
    v += __shfl_down_sync(0xffffffffu, v, 2);
    v += __shfl_down_sync(0xffffffffu, v, 1);
    return v;
}

__device__ __forceinline__ float reduce_i(float v) {
    v += __shfl_down_sync(0xffffffffu, v, 16);
    v += __shfl_down_sync(0xffffffffu, v, 8);
    return v;
}

// Horner evaluation of a polynomial held in registers; the coefficient count is a
// compile-time bucket and the coefficients above the fitted degree are zero, which
// leaves the value unchanged (fma(0, x, 0) = 0 until the leading coefficient).
template <int NP>
__device__ __forceinline__ float horner(const float (&c)[NP], float x) {
    float acc = c[NP - 1];
#pragma unroll
    for (int k = NP - 2; k >= 0; --k) acc = fmaf(acc, x, c[k]);
    return acc;
}

// EXCL: working entries flagged by the prune (bit 17) carry 8 pair masks (one per i-cluster,
// bit ti * 8 + tj) at xmask[8 (wxid[e] - 1)]; a masked pair takes the excluded branch of pair_force.
template <int LJK, bool COUL, bool ENERGY, int NP, bool EXCL>
__global__ void __launch_bounds__(128) k_pairs(const float4 *__restrict__ xq, const int *__restrict__ ts,
                                              const uint2 *__restrict__ cjw, const int *__restrict__ scio,
                                              const int *__restrict__ nw, const int *__restrict__ counts,
                                              const float *__restrict__ lj_table, float4 *__restrict__ fc,
                                              float *__restrict__ vc, int nslot, int nsplit, const PairParams pp,
                                              const int *__restrict__ wxid,
                                              const unsigned long long *__restrict__ xmask) {
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int nwarp = blockDim.x >> 5;   // warps per super-cluster part (1, 2 or 4: the tuned shape)
    const int ti = lane & 7, q = lane >> 3;
    const int S = blockIdx.x / nsplit, part = blockIdx.x % nsplit;
    if (S >= counts[W_NS] || counts[W_ERR] != 0) return;
    __shared__ float4 sxq[SUPER];
    __shared__ int sty[SUPER];
    __shared__ float4 stab[LJK == PD_LJ_TABLE ? PD_MAX_TYPES * PD_MAX_TYPES : 1];
    for (int k = tid; k < SUPER; k += blockDim.x) {
        float4 v = xq[S * SUPER + k];
        if (COUL) v.w *= pp.C;
        sxq[k] = v;
        if (LJK == PD_LJ_TABLE) sty[k] = (ts[S * SUPER + k] - 1) * pp.ntypes;
    }
    if (LJK == PD_LJ_TABLE) {
        for (int k = tid; k < pp.ntypes * pp.ntypes; k += blockDim.x)
            stab[k] = reinterpret_cast<const float4 *>(lj_table)[k];
    }
    __syncthreads();
    const float Lx = pp.Lx, Ly = pp.Ly, Lz = pp.Lz;
    const float hx = 0.5f * Lx, hy = 0.5f * Ly, hz = 0.5f * Lz;
    float cpf[NP], cpe[NP];
#pragma unroll
    for (int k = 0; k < NP; ++k) {
        cpf[k] = COUL ? pp.pf[k] : 0.f;
        cpe[k] = (COUL && ENERGY) ? pp.pe[k] : 0.f;
    }
    float fxi[8], fyi[8], fzi[8];
    float ei[8], w1i[8], w2i[8], w3i[8], w4i[8], w5i[8], w6i[8];
#pragma unroll
    for (int a = 0; a < 8; ++a) {
        fxi[a] = fyi[a] = fzi[a] = 0.f;
        if (ENERGY) ei[a] = w1i[a] = w2i[a] = w3i[a] = w4i[a] = w5i[a] = w6i[a] = 0.f;
    }
    // One pair: i-atom pi of i-cluster a against j-atom pj; J accumulates the j-atom's
    // force (and with ENERGY its half energy and half virial).  `masked` drops the self
    // and double-counted pairs of the tile that holds the i-cluster itself; marked
    // (pbc) tiles take the compensated periodic difference (PeriodicDisplacement.jl:4-14).
    // Padding atoms sit far away with zero charge and contribute exact zeros.  `excl` (EXCL only):
    // the pair is an exception; its Coulomb term becomes minus the mesh part (the scaled term is
    // added outside the tiles) and, with bond exclusions, its LJ term is dropped.
    auto pair = [&](const int a, const float4 &pi, const float4 &pj, int tyi, int tyj, bool masked, bool pbc,
                    bool excl, float (&J)[10]) {
        float dx, dy, dz;
        if (pbc) {
            dx = periodic_delta(pi.x, pj.x, hx, Lx);
            dy = periodic_delta(pi.y, pj.y, hy, Ly);
            dz = periodic_delta(pi.z, pj.z, hz, Lz);
        } else {
            dx = pi.x - pj.x;
            dy = pi.y - pj.y;
            dz = pi.z - pj.z;
        }
        const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
        const float rinv = rsqrtf(r2);
        const float rinv2 = rinv * rinv;
        float f = 0.f, en = 0.f;
        if (LJK != PD_LJ_NONE) {
            float c6, c12, lrc2, esh;
            if (LJK == PD_LJ_TABLE) {
                const float4 tb = stab[tyi + (tyj - 1)];
                c6 = tb.x;
                c12 = tb.y;
                lrc2 = tb.z;
                esh = tb.w;
            } else {
                c6 = pp.c6;
                c12 = pp.c12;
                lrc2 = pp.lrc2;
                esh = pp.esh;
            }
            const bool use = r2 < lrc2 && !(EXCL && pp.lj_excl && excl);
            const float ir6 = rinv2 * rinv2 * rinv2;
            f += use ? (12.f * c12 * ir6 - 6.f * c6) * ir6 * rinv2 : 0.f;
            if (ENERGY) en += use ? (c12 * ir6 - c6) * ir6 - esh : 0.f;
        }
        if (COUL) {
            // pi.w holds C q_i (premultiplied when the i-atoms were staged)
            const bool inr = r2 < pp.rc2;
            const float x = fmaf(r2, pp.sx, -1.f);
            const float pf = horner(cpf, x);
            const float rinv3 = rinv * rinv2;
            const float cq = pi.w * pj.w;
            float fq = inr ? rinv3 - pf : 0.f;
            if (EXCL) fq = excl ? (inr ? -pf : (pp.has_mesh ? -rinv3 : 0.f)) : fq;
            f = fmaf(cq, fq, f);
            if (ENERGY) {
                const float pe = horner(cpe, x);
                float eq = inr ? rinv + pe - pp.eshift : 0.f;
                if (EXCL) eq = excl ? (inr ? pe : (pp.has_mesh ? -rinv : 0.f)) : eq;
                en = fmaf(cq, eq, en);
            }
        }
        f = masked ? 0.f : f;
        fxi[a] = fmaf(f, dx, fxi[a]);
        fyi[a] = fmaf(f, dy, fyi[a]);
        fzi[a] = fmaf(f, dz, fzi[a]);
        J[0] = fmaf(-f, dx, J[0]);
        J[1] = fmaf(-f, dy, J[1]);
        J[2] = fmaf(-f, dz, J[2]);
        if (ENERGY) {
            en = masked ? 0.f : 0.5f * en;
            const float hf = 0.5f * f;
            const float hfx = hf * dx, hfy = hf * dy;
            const float w1 = hfx * dx, w2 = hfy * dy, w3 = hf * dz * dz;
            const float w4 = hfx * dy, w5 = hfx * dz, w6 = hfy * dz;
            ei[a] += en;
            w1i[a] += w1;
            w2i[a] += w2;
            w3i[a] += w3;
            w4i[a] += w4;
            w5i[a] += w5;
            w6i[a] += w6;
            J[3] += en;
            J[4] += w1;
            J[5] += w2;
            J[6] += w3;
            J[7] += w4;
            J[8] += w5;
            J[9] += w6;
        }
    };
    // j-atom results of one entry: reduced over the 8 ti lanes and added to the slot
    auto flush = [&](const float (&J)[10], int js) {
        const float r = reduce3(J[0], J[1], J[2], ti);
        if (ti < 3) red_add(reinterpret_cast<float *>(&fc[js]) + ti, r);
        if (ENERGY) {
            const float rv1 = reduce3(J[4], J[5], J[6], ti);
            const float rv2 = reduce3(J[7], J[8], J[9], ti);
            const float ej = sum8(J[3]);
            if (ti < 3) {
                red_add(&vc[(size_t)ti * nslot + js], rv1);
                red_add(&vc[(size_t)(ti + 3) * nslot + js], rv2);
            }
            if (ti == 0) red_add(reinterpret_cast<float *>(&fc[js]) + 3, ej);
        }
    };
    const int e0 = scio[S], ne = nw[S];
    const int ea = e0 + (int)(((long long)ne * part) / nsplit);
    const int eb = e0 + (int)(((long long)ne * (part + 1)) / nsplit);
    // The warps take entries in turn.  Lane (ti, q) pairs i-atom ti of every
    // i-cluster in the mask with j-atoms q (j half 0) and q + 4 (j half 1); the next
    // entry's word and j-atoms are loaded while the current one is evaluated.
    const bool gtA = q > ti, gtB = q + 4 > ti;
    int e = ea + w;
    uint2 ent = e < eb ? cjw[e] : make_uint2(0u, 0u);
    float4 pa = e < eb ? xq[(int)ent.x * 8 + q] : make_float4(0.f, 0.f, 0.f, 0.f);
    float4 pb = e < eb ? xq[(int)ent.x * 8 + q + 4] : make_float4(0.f, 0.f, 0.f, 0.f);
    int ta = 1, tb = 1;
    if (LJK == PD_LJ_TABLE && e < eb) {
        ta = ts[(int)ent.x * 8 + q];
        tb = ts[(int)ent.x * 8 + q + 4];
    }
    for (; e < eb; e += nwarp) {
        const uint2 cur = ent;
        const float4 ja = pa, jb = pb;
        const int cta = ta, ctb = tb;
        if (e + nwarp < eb) {
            ent = cjw[e + nwarp];
            pa = xq[(int)ent.x * 8 + q];
            pb = xq[(int)ent.x * 8 + q + 4];
            if (LJK == PD_LJ_TABLE) {
                ta = ts[(int)ent.x * 8 + q];
                tb = ts[(int)ent.x * 8 + q + 4];
            }
        }
        // the entry is the same for every lane; the warp reduction makes that visible to the
        // compiler, so the branches on its bits below are uniform
        const uint32_t word = __reduce_or_sync(0xffffffffu, cur.y);
        const uint32_t lo = word & 0xffu, hi = (word >> 8) & 0xffu;
        const bool pbc = (word >> 16) & 1u;   // tile may cross a box face before the next prune
        const int cj = (int)__reduce_or_sync(0xffffffffu, cur.x);
        const int da = cj - S * 8;   // index of the i-cluster that is the j-cluster itself, if in [0, 8)
        const bool hasx = EXCL && ((word >> 17) & 1u);
        size_t xb = 0;
        if (EXCL && hasx) xb = (size_t)(__reduce_or_sync(0xffffffffu, (uint32_t)wxid[e]) - 1) * 8;
        float A[10], B[10];
#pragma unroll
        for (int k = 0; k < 10; ++k) A[k] = B[k] = 0.f;
#pragma unroll
        for (int a = 0; a < 8; ++a) {
            if (((lo | hi) >> a) & 1u) {
                const float4 pi = sxq[a * 8 + ti];
                const int tyi = LJK == PD_LJ_TABLE ? sty[a * 8 + ti] : 0;
                const bool self = da == a;
                const unsigned long long mk = (EXCL && hasx) ? xmask[xb + a] : 0ull;
                const bool xa = (mk >> (ti * 8 + q)) & 1ull, xbb = (mk >> (ti * 8 + q + 4)) & 1ull;
                if ((lo >> a) & 1u) pair(a, pi, ja, tyi, cta, self && !gtA, pbc, xa, A);
                if ((hi >> a) & 1u) pair(a, pi, jb, tyi, ctb, self && !gtB, pbc, xbb, B);
            }
        }
        flush(A, cj * 8 + q);
        flush(B, cj * 8 + q + 4);
    }
#pragma unroll
    for (int a = 0; a < 8; ++a) {
        fxi[a] = reduce_i(fxi[a]);
        fyi[a] = reduce_i(fyi[a]);
        fzi[a] = reduce_i(fzi[a]);
        if (ENERGY) {
            ei[a] = reduce_i(ei[a]);
            w1i[a] = reduce_i(w1i[a]);
            w2i[a] = reduce_i(w2i[a]);
            w3i[a] = reduce_i(w3i[a]);
            w4i[a] = reduce_i(w4i[a]);
            w5i[a] = reduce_i(w5i[a]);
            w6i[a] = reduce_i(w6i[a]);
        }
    }
    if (lane < 8) {
#pragma unroll
        for (int a = 0; a < 8; ++a) {
            const int ai = S * SUPER + a * 8 + lane;
            if (ENERGY) {
                red_add_v4(reinterpret_cast<float *>(&fc[ai]), fxi[a], fyi[a], fzi[a], ei[a]);
                red_add(&vc[(size_t)0 * nslot + ai], w1i[a]);
                red_add(&vc[(size_t)1 * nslot + ai], w2i[a]);
                red_add(&vc[(size_t)2 * nslot + ai], w3i[a]);
                red_add(&vc[(size_t)3 * nslot + ai], w4i[a]);
                red_add(&vc[(size_t)4 * nslot + ai], w5i[a]);
                red_add(&vc[(size_t)5 * nslot + ai], w6i[a]);
            } else {
                red_add_v4(reinterpret_cast<float *>(&fc[ai]), fxi[a], fyi[a], fzi[a], 0.f);
            }
        }
    }
}

template <int LJK, bool COUL, bool EN, int NP, bool EXCL>
static void launch_pairs(pd_cluster *c, cudaStream_t s) {
    k_pairs<LJK, COUL, EN, NP, EXCL><<<c->nsmax * c->nsplit, 32 * c->pair_warps, 0, s>>>(
        c->xq, c->ts, c->cjw, c->scio, c->nw, c->counts, c->lj_table, c->fc, c->vc, c->nslot, c->nsplit, c->pp,
        c->wxid, c->xmask);
}

template <int LJK, bool EN, bool EXCL>
static void launch_pairs_poly(pd_cluster *c, cudaStream_t s) {
    const PairParams &pp = c->pp;
    if (!pp.coulomb) {
        launch_pairs<LJK, false, EN, 1, EXCL>(c, s);
        return;
    }
    const int n = EN ? (pp.nf > pp.ne ? pp.nf : pp.ne) : pp.nf;
    if (n <= 8) launch_pairs<LJK, true, EN, 8, EXCL>(c, s);
    else if (n <= 10) launch_pairs<LJK, true, EN, 10, EXCL>(c, s);
    else if (n <= 12) launch_pairs<LJK, true, EN, 12, EXCL>(c, s);
    else if (n <= 14) launch_pairs<LJK, true, EN, 14, EXCL>(c, s);
    else if (n <= 16) launch_pairs<LJK, true, EN, 16, EXCL>(c, s);
    else if (n <= 20) launch_pairs<LJK, true, EN, 20, EXCL>(c, s);
    else launch_pairs<LJK, true, EN, 32, EXCL>(c, s);
}

// The pair pass for the engine's LJ kind and energy flag.
template <bool EXCL>
static void pairs_dispatch(pd_cluster *c, int energy, cudaStream_t s) {
    switch (c->pp.lj_kind) {
        case PD_LJ_NONE:
            energy ? launch_pairs_poly<PD_LJ_NONE, true, EXCL>(c, s) : launch_pairs_poly<PD_LJ_NONE, false, EXCL>(c, s);
            break;
        case PD_LJ_UNIFORM:
            energy ? launch_pairs_poly<PD_LJ_UNIFORM, true, EXCL>(c, s)
                   : launch_pairs_poly<PD_LJ_UNIFORM, false, EXCL>(c, s);
            break;
        default:
            energy ? launch_pairs_poly<PD_LJ_TABLE, true, EXCL>(c, s) : launch_pairs_poly<PD_LJ_TABLE, false, EXCL>(c, s);
            break;
    }
}

}  // namespace pdb
