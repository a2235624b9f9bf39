// Shared device helpers of libpdb200 (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <math.h>

#include "../../include/pdb200.h"

namespace pdb {

constexpr int CLUSTER = 8;   // particles per cluster (List.jl:29)
constexpr int SUPER = 64;    // particles per super-cluster (List.jl:30)
constexpr int SEARCH_MAX_COLS = 1024;   // neighbouring columns one super-cluster may search

// Device count words of one cluster list (indices into pd_cluster::counts).
enum CountWord {
    W_NS = 0,        // super-clusters in use
    W_NE = 1,        // outer entries
    W_ERR = 2,       // latched error (PD_ECAPACITY / PD_ENONFINITE)
    W_REQ = 3,       // outer entries required on overflow
    W_BUILD = 4,     // this step's decision: rebuild
    W_PRUNE = 5,     // this step's decision: prune
    W_REQUEST = 6,   // forced rebuild on the next decision (setup, growth)
    W_NBUILD = 7,    // device-decided builds
    W_NPRUNE = 8,    // device-decided prunes
    W_DSTEP = 9,     // decisions so far (fixed intervals)
    W_FLAG_ANY = 10, // max displacement ratio (build or prune) as float bits
    W_FLAG_BUILD = 11, // max displacement ratio since the build as float bits
    W_NWORK = 12,    // working entries (sum over super-clusters, diagnostics)
    W_TICKET = 13,   // blocks of the step's kick kernel that have reported (last one decides)
    W_NX = 14,       // outer entries holding an excluded pair (exceptions)
    W_NP = 15,       // exception pairs computed outside the tiles (scaled in-list, or out of the list)
    W_LEN = 16
};

// The list geometry below is written with explicit round-to-nearest intrinsics
// (no multiply-add contraction) so that a build is reproducible operation by
// operation by a plain C restatement.

__device__ __forceinline__ float wrap_positive(float x, float L) {
    // _wrapc, List.jl:190: x - L floor(x / L)
    return __fsub_rn(x, __fmul_rn(L, floorf(__fdiv_rn(x, L))));
}

// force_coordinate (src/geometry/PeriodicDisplacement.jl:21-25): keep centred
// coordinates unchanged, otherwise translate into [-L/2, L/2).
__device__ __forceinline__ float force_coordinate(float x, float L) {
    float h = 0.5f * L;
    if (-h <= x && x <= h) return x;
    return __fsub_rn(x, __fmul_rn(L, floorf(__fadd_rn(__fdiv_rn(x, L), 0.5f))));
}

// periodic_delta (PeriodicDisplacement.jl:4-14): error-free TwoDiff followed by
// the exact subtraction of L.  Compiled without fast-math; the operations below
// must not be reassociated.
// Branch-free: both results are formed and one is selected, so lanes of a warp
// never diverge on it.
__device__ __forceinline__ float periodic_delta(float xi, float xj, float halfL, float L) {
    const float d = __fsub_rn(xi, xj);
    const float bv = __fsub_rn(xi, d);
    const float res = __fadd_rn(__fsub_rn(xi, __fadd_rn(d, bv)), __fsub_rn(bv, xj));
    const float w = __fadd_rn(__fsub_rn(d, copysignf(L, d)), res);
    return fabsf(d) > halfL ? w : d;
}

// _mic (List.jl:192-197)
__device__ __forceinline__ float mic(float d, float L) {
    float h = 0.5f * L;
    d -= (d > h) ? L : 0.0f;
    d += (d < -h) ? L : 0.0f;
    return d;
}

// Padding slots of the packed coordinates hold far-away, pairwise distinct points and
// zero charge: component k is 1e7 + 1000 * (k-th 10-bit digit of the slot index), so
// two slots differ by at least 1000 in some component (all values below 1.3e7 are
// exact in FP32).  Every pair with a padding atom then lies far beyond any cutoff on
// the plain (non-wrapping) difference and its LJ and Coulomb terms are exact zeros
// without masking.  Real coordinates stay far below PAD_LIMIT.
constexpr float PAD_BASE = 1.0e7f;
constexpr float PAD_STEP = 1000.0f;
constexpr float PAD_LIMIT = 1.0e6f;
__device__ __forceinline__ float4 pad_point(int slot) {
    return make_float4(PAD_BASE + PAD_STEP * (float)(slot & 1023), PAD_BASE + PAD_STEP * (float)((slot >> 10) & 1023),
                       PAD_BASE + PAD_STEP * (float)(slot >> 20), 0.f);
}

__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v = fmaxf(v, __shfl_down_sync(0xffffffffu, v, off));
    return v;
}

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    return v;
}

// Fence-free float reduction into global memory (the reference's relaxed @red,
// src/gpu/RelaxedAtomics.jl:11-44).
__device__ __forceinline__ void red_add(float *p, float v) {
    asm volatile("red.relaxed.gpu.global.add.f32 [%0], %1;" ::"l"(p), "f"(v) : "memory");
}
__device__ __forceinline__ void red_add_v4(float *p, float a, float b, float c, float d) {
    asm volatile("red.relaxed.gpu.global.add.v4.f32 [%0], {%1,%2,%3,%4};" ::"l"(p), "f"(a), "f"(b), "f"(c), "f"(d)
                 : "memory");
}
// Shared-memory float add without a returned value (no register waits on the result).
__device__ __forceinline__ void red_add_shared(float *p, float v) {
    const unsigned a = (unsigned)__cvta_generic_to_shared(p);
    asm volatile("red.shared.add.f32 [%0], %1;" ::"r"(a), "f"(v) : "memory");
}
__device__ __forceinline__ void red_add_d(double *p, double v) {
    asm volatile("red.relaxed.gpu.global.add.f64 [%0], %1;" ::"l"(p), "d"(v) : "memory");
}

__device__ __forceinline__ float4 ldg_f4(const float4 *p) { return __ldg(p); }

}  // namespace pdb
