// Shared device pieces of the ELL route (ell.cu) and the batched replicas (batch.cu): the device
// state words and their decision, the block-maximum reduction with its last-block ticket, the
// nearest-image shift and the stencil-row ranges.
#pragma once

#include "common.cuh"

namespace pdb {

// Device state words (DN_* of DeviceNeighborCUDA.jl:4-33, plus this library's reduction words).
enum EllWord {
    E_REQUEST = 0,
    E_VALID = 1,
    E_ERROR = 2,        // 0, E_ERR_CAPACITY or E_ERR_COORD (latched)
    E_STEP = 3,
    E_LAST_BUILD = 4,
    E_INTERVAL = 5,
    E_CHECKS = 6,
    E_BUILDS = 7,
    E_REQUIRED = 8,     // largest row of the last build attempt
    E_DMAX = 9,         // displacement maximum of the current decision (float bits)
    E_RMAX = 10,        // largest row of the current build
    E_TICKET_D = 11,    // blocks of the decision kernel that have reported
    E_TICKET_R = 12,    // blocks of the row kernel that have reported
    E_LEN = 16
};
constexpr long long E_ERR_CAPACITY = 1, E_ERR_COORD = 2;
constexpr int ELL_THREADS = 256;
constexpr int ELL_SCAN_CHUNK = 8192;

__device__ __forceinline__ bool ell_requested(const long long *st) { return st[E_REQUEST] != 0 && st[E_ERROR] == 0; }

// mic_fast (src/BondedForces.jl:23-27): one conditional shift each way.
__device__ __forceinline__ float mic_fast(float d, float h, float L) {
    d -= (d > h) ? L : 0.f;
    d += (d < -h) ? L : 0.f;
    return d;
}

// Rebuild decision (_device_decide_kernel!, DeviceNeighborCUDA.jl:198-238) from the displacement
// maximum (squared, since the last build) against threshold = skin^2 / 4, with the adaptive
// interval (x0.9 after a displacement-triggered build, x1.1 when the maximum stays below a tenth
// of the threshold, clamped to 5..100; Julia's round: nearest, ties to even).
template <bool COND>
__device__ void ell_decide(long long *st, float largest, float threshold, cudaGraphConditionalHandle h) {
    st[E_CHECKS] += 1;
    st[E_REQUEST] = 0;
    if (!isfinite(largest)) {
        st[E_ERROR] = E_ERR_COORD;
        st[E_VALID] = 0;
    } else if (st[E_VALID] == 0) {
        st[E_REQUEST] = 1;
    } else if (largest > threshold || st[E_STEP] - st[E_LAST_BUILD] >= st[E_INTERVAL]) {
        st[E_REQUEST] = 1;
        st[E_VALID] = 0;
        const float iv = (float)st[E_INTERVAL];
        if (largest > threshold) {
            const long long v = (long long)rintf(0.9f * iv);
            st[E_INTERVAL] = v > 5 ? v : 5;
        } else if (largest < 0.1f * threshold) {
            const long long v = (long long)rintf(1.1f * iv);
            st[E_INTERVAL] = v < 100 ? v : 100;
        }
    }
    if (COND) cudaGraphSetConditional(h, ell_requested(st) ? 1u : 0u);
}

// Displacement of one particle since the last build (_device_displacement_kernel!,
// DeviceNeighborCUDA.jl:170-196): infinite for a non-finite or uncentred coordinate; the squares
// are accumulated from the last dimension down with nested multiply-adds.
template <int D>
__device__ __forceinline__ float ell_displacement(const float *p, const float4 r, const float *L, bool valid) {
    float value = 0.f;
    const float rr[3] = {r.x, r.y, r.z};
#pragma unroll
    for (int d = D - 1; d >= 0; --d) {
        const float x = p[d];
        const float h = 0.5f * L[d];
        if (!(isfinite(x) && -h <= x && x <= h)) {
            value = __int_as_float(0x7f800000);
        } else if (valid) {
            const float dx = mic_fast(x - rr[d], h, L[d]);
            value = fmaf(dx, dx, value);
        }
    }
    return value;
}

// Block maximum of a 32-bit pattern (a non-negative float's bits or a non-negative int, which
// order like unsigned integers) reported to st[word]; returns true in thread 0 of the last block
// to report (threadfence-reduction pattern), which then owns the complete maximum.
__device__ __forceinline__ bool ell_block_max_last(unsigned v, long long *st, int word, int ticket) {
    __shared__ unsigned sh[ELL_THREADS / 32];
    __shared__ bool last;
    v = __reduce_max_sync(0xffffffffu, v);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) sh[w] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned m = 0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) m = max(m, sh[k]);
        atomicMax(reinterpret_cast<unsigned long long *>(&st[word]), (unsigned long long)m);
        __threadfence();
        last = atomicAdd(reinterpret_cast<unsigned long long *>(&st[ticket]), 1ull) == (unsigned long long)gridDim.x - 1;
        if (last) __threadfence();
    }
    __syncthreads();
    return threadIdx.x == 0 && last;
}

// Cells of the stencil row (oy, oz) within reach of cell cx along x: one or two contiguous
// ranges (two at the periodic seam) (_row_ranges, DeviceNeighborCUDA.jl:498-505).
__device__ __forceinline__ void ell_row_ranges(int cx, float g2, float rl2, float hx, int Sx, int nx, int &a1, int &b1,
                                               int &a2, int &b2) {
    const int ax = min(Sx, 1 + (int)(sqrtf(fmaxf(rl2 - g2, 0.f)) / hx));
    const int lo = cx - ax, hi = cx + ax;
    a2 = 1;
    b2 = 0;
    if (lo < 0) {
        a1 = lo + nx;
        b1 = nx - 1;
        a2 = 0;
        b2 = hi;
    } else if (hi >= nx) {
        a1 = lo;
        b1 = nx - 1;
        a2 = 0;
        b2 = hi - nx;
    } else {
        a1 = lo;
        b1 = hi;
    }
}

__device__ __forceinline__ int ell_reach(float rl, float L, int n) {
    if (n < 3) return 1;
    return min(max(1, (int)ceilf(rl * (float)n / L - 1e-5f)), (n - 1) / 2);
}

}  // namespace pdb
