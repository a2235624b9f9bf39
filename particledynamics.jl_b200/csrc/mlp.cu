// Network of the learned coarse-mesh correction: the 32-128-128-1 SiLU network
// on fifth-generation tensor cores (tcgen05, sm_100a), its fused training pass
// and Adam.
//
// Every GEMM runs as tcgen05.mma (kind::f16: BF16 operands, FP32 accumulators
// in tensor memory) issued by one thread per CTA.  Operands sit in shared
// memory in the K-major no-swizzle core-matrix layout: a core matrix is 8 rows
// x 16 bytes (8 BF16 along K), the K-adjacent core matrices are 128 bytes
// apart (leading byte offset) and the 8-row groups K * 16 bytes apart (stride
// byte offset).  Completion is signalled through an mbarrier by
// tcgen05.commit; accumulators come back with tcgen05.ld (32 lanes x 32
// columns per warp and call) for the fused epilogues.
//
// Rounding points (the parity tests emulate them): x, W1, W2 and the hidden
// activation h1 = silu(x W1^T + b1) are BF16; every product accumulates in
// FP32; b1, b2, w3, b3, the second activation and the output are FP32.
// Training uses the same forward; the backward products take the BF16-rounded
// dz2, h1, dz1 and x.
//
// A CTA of 128 threads owns tiles of 128 rows (particles); thread m of the CTA
// owns tile row m in every epilogue (TMEM lane m).  Waits on the mbarrier are
// bounded (2^31 clock cycles, about one second): a timeout latches the error
// word, skips the remaining work and the tensor memory is still released.
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "internal.hpp"

using namespace pdb;

namespace pdb {

constexpr int MLP_IN = 32, MLP_H = 128, MLP_TILE = 128, MLP_THREADS = 128;

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Byte offset of element (row, k) of a K-major tile with K columns (core-matrix layout).
__device__ __forceinline__ uint32_t cm_off(int row, int k, int K) {
    return (uint32_t)((((row >> 3) * (K >> 3) + (k >> 3)) << 7) + ((row & 7) << 4) + ((k & 7) << 1));
}

// Shared-memory matrix descriptor, no swizzle, K-major: start address, leading byte offset
// (between K-adjacent core matrices), stride byte offset (between 8-row groups), version 1.
__device__ __forceinline__ uint64_t umma_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = (uint64_t)((addr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

// Instruction descriptor of kind::f16: FP32 accumulator (bits 4-5 = 1), BF16 A (bits 7-9 = 1)
// and B (bits 10-12 = 1), both K-major, N >> 3 at bit 17, M >> 4 at bit 24.
__host__ __device__ constexpr uint32_t umma_idesc(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
        :
        : "r"(tmem_d), "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void umma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Bounded wait for the completion of the mbarrier phase with the given parity.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    const long long t0 = clock64();
    while (true) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
        if (clock64() - t0 > (1ll << 31)) return false;
    }
}

__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Whole-CTA hand-over between generic shared-memory writes / tensor-memory reads and the
// next tensor-core instruction.
__device__ __forceinline__ void tc_sync() {
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
}

__device__ __forceinline__ void tmem_alloc(uint32_t dst_smem, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst_smem), "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// 32 consecutive FP32 columns of this thread's TMEM lane (shape 32x32b, 32 repetitions).
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr)
        : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int k = 0; k < 32; ++k) v[k] = __uint_as_float(r[k]);
}

// Logistic function with the fast exponential and division (relative error of a few ulp).
__device__ __forceinline__ float sigm(float z) { return __fdividef(1.f, 1.f + __expf(-z)); }

// Sums v[0..31] over the 32 lanes of the warp (recursive halving); lane l returns the total
// of element l.
__device__ __forceinline__ float warp_reduce_scatter32(float (&v)[32]) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int w = 16; w >= 1; w >>= 1) {
        const bool hi = (lane & w) != 0;
#pragma unroll
        for (int i = 0; i < w; ++i) {
            const float send = hi ? v[i] : v[i + w];
            const float keep = hi ? v[i + w] : v[i];
            v[i] = keep + __shfl_xor_sync(0xffffffffu, send, w);
        }
    }
    return v[0];
}

// M x N x K product of two core-matrix tiles (A: M rows, B: N rows, both K columns) into
// tmem_d; acc0 = false overwrites the accumulator on the first K-slice.  Thread 0 only.
__device__ __forceinline__ void gemm_issue(uint32_t tmem_d, uint32_t a, uint32_t b, int K, int M, int N, bool acc0) {
    const uint32_t idesc = umma_idesc(M, N);
    const uint32_t sbo = (uint32_t)K * 16u;
    for (int s = 0; s < K / 16; ++s)
        umma_bf16(tmem_d, umma_desc(a + 256u * s, 128u, sbo), umma_desc(b + 256u * s, 128u, sbo), idesc,
                  (acc0 || s > 0) ? 1u : 0u);
}

// Eight consecutive values as BF16 (16 bytes) at a core-matrix offset.
__device__ __forceinline__ void st8(unsigned char *base, uint32_t off, const float *v) {
    __align__(16) __nv_bfloat16 h[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) h[k] = __float2bfloat16_rn(v[k]);
    *reinterpret_cast<uint4 *>(base + off) = *reinterpret_cast<const uint4 *>(h);
}
__device__ __forceinline__ void st1(unsigned char *base, uint32_t off, float v) {
    *reinterpret_cast<__nv_bfloat16 *>(base + off) = __float2bfloat16_rn(v);
}

struct MlpWeights {
    const __nv_bfloat16 *w1;   // [128][32]
    const __nv_bfloat16 *w2;   // [128][128]
    const float *b1, *b2, *w3; // [128]
    const float *b3;           // [1]
};

// Rows of W1 (as B: rows o, K = i) and W2 (rows o, K = k) into shared memory; thread t loads row t.
__device__ __forceinline__ void load_weights(unsigned char *sm, uint32_t ow1, uint32_t ow2, const MlpWeights &wt,
                                             int t) {
#pragma unroll
    for (int c = 0; c < MLP_IN / 8; ++c)
        *reinterpret_cast<uint4 *>(sm + ow1 + cm_off(t, 8 * c, MLP_IN)) =
            __ldg(reinterpret_cast<const uint4 *>(wt.w1 + (size_t)t * MLP_IN) + c);
#pragma unroll 4
    for (int c = 0; c < MLP_H / 8; ++c)
        *reinterpret_cast<uint4 *>(sm + ow2 + cm_off(t, 8 * c, MLP_H)) =
            __ldg(reinterpret_cast<const uint4 *>(wt.w2 + (size_t)t * MLP_H) + c);
}

// Inference kernel: persistent, one CTA per SM with four warpgroups; each warpgroup owns one 128-row
// tile at a time (its own X and H1 buffers, 128 TMEM columns and mbarrier), the weights are staged
// once per CTA and shared, so four tiles' load -> MMA -> epilogue chains overlap on every SM.
constexpr int FW_WG = 4, FW_THREADS = 128 * FW_WG;
constexpr int FW_W1 = 0, FW_W2 = FW_W1 + MLP_H * MLP_IN * 2, FW_TILES = FW_W2 + MLP_H * MLP_H * 2;
constexpr int FW_X = 0, FW_H1 = FW_X + MLP_TILE * MLP_IN * 2, FW_TILE_BYTES = FW_H1 + MLP_TILE * MLP_H * 2;
constexpr int FW_BYTES = FW_TILES + FW_WG * FW_TILE_BYTES;

__device__ __forceinline__ void wg_barrier(int g) {   // the 128 threads of warpgroup g
    asm volatile("bar.sync %0, %1;" ::"r"(1 + g), "r"(128) : "memory");
}
// Barrier of warpgroup g that also returns whether every thread's flag is set (a uniform decision).
__device__ __forceinline__ bool wg_and(int g, bool flag) {
    uint32_t res;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.b32 p, %1, 0;\n\t"
        "bar.red.and.pred q, %2, %3, p;\n\t"
        "selp.b32 %0, 1, 0, q;\n\t}\n"
        : "=r"(res)
        : "r"((uint32_t)flag), "r"(1 + g), "r"(128)
        : "memory");
    return res != 0;
}
__device__ __forceinline__ void wg_tc_sync(int g) {
    fence_async_smem();
    tc_fence_before();
    wg_barrier(g);
    tc_fence_after();
}

// s = w3 . silu(W2 h1 + b2) + b3 with h1 = bf16(silu(W1 x + b1)) for every row; out_s[r] = s and,
// with V given, corr[r] = (s V.x, s V.y, s V.z, s): the force residual s_i V_i of the learned
// correction.  Thread t of warpgroup g owns tile row t (TMEM lane t) in both epilogues.
__global__ void __launch_bounds__(FW_THREADS, 1) k_mlp_forward(const __nv_bfloat16 *__restrict__ X, int n,
                                                              MlpWeights wt, float *__restrict__ out_s,
                                                              const float4 *__restrict__ V,
                                                              float4 *__restrict__ corr, int *__restrict__ err) {
    extern __shared__ __align__(1024) unsigned char sm[];
    __shared__ __align__(8) uint64_t bars[FW_WG];
    __shared__ uint32_t tmem_base;
    __shared__ float sb1[MLP_H], sb2[MLP_H], sw3[MLP_H];
    const int t = threadIdx.x, w = t >> 5, lane = t & 31;
    const int g = t >> 7, tl = t & 127;   // warpgroup, thread (= tile row) within it
    if (w == 0) tmem_alloc(smem_u32(&tmem_base), 128 * FW_WG);
    if (t < FW_WG) mbar_init(smem_u32(&bars[t]), 1);
    if (t < MLP_H) {
        sb1[t] = __ldg(wt.b1 + t);
        sb2[t] = __ldg(wt.b2 + t);
        sw3[t] = __ldg(wt.w3 + t);
    }
    // weights once per CTA: row t % 128 of W1 and W2, the chunks split over the four warpgroups
#pragma unroll
    for (int c = g; c < MLP_IN / 8; c += FW_WG)
        *reinterpret_cast<uint4 *>(sm + FW_W1 + cm_off(tl, 8 * c, MLP_IN)) =
            __ldg(reinterpret_cast<const uint4 *>(wt.w1 + (size_t)tl * MLP_IN) + c);
#pragma unroll
    for (int c = g; c < MLP_H / 8; c += FW_WG)
        *reinterpret_cast<uint4 *>(sm + FW_W2 + cm_off(tl, 8 * c, MLP_H)) =
            __ldg(reinterpret_cast<const uint4 *>(wt.w2 + (size_t)tl * MLP_H) + c);
    tc_sync();
    const float b3 = __ldg(wt.b3);
    const uint32_t base = smem_u32(sm), bar = smem_u32(&bars[g]);
    const uint32_t tm = tmem_base + 128u * g;                          // this group's columns
    const uint32_t lane_addr = tm + ((uint32_t)(32 * (w & 3)) << 16);  // this warp's lane quarter
    unsigned char *tile_sm = sm + FW_TILES + g * FW_TILE_BYTES;
    const uint32_t tile_base = base + FW_TILES + g * FW_TILE_BYTES;
    const int ntiles = (n + MLP_TILE - 1) / MLP_TILE;
    uint32_t phase = 0;
    bool ok = true;
    for (int tile = blockIdx.x * FW_WG + g; tile < ntiles; tile += gridDim.x * FW_WG) {
        const int r = tile * MLP_TILE + tl;
        {
            const uint4 zero = make_uint4(0, 0, 0, 0);
#pragma unroll
            for (int c = 0; c < MLP_IN / 8; ++c)
                *reinterpret_cast<uint4 *>(tile_sm + FW_X + cm_off(tl, 8 * c, MLP_IN)) =
                    r < n ? __ldg(reinterpret_cast<const uint4 *>(X + (size_t)r * MLP_IN) + c) : zero;
        }
        wg_tc_sync(g);
        if (tl == 0) {
            gemm_issue(tm, tile_base + FW_X, base + FW_W1, MLP_IN, MLP_TILE, MLP_H, false);
            umma_commit(bar);
        }
        ok = wg_and(g, mbar_wait(bar, phase));
        phase ^= 1;
        if (!ok) break;
        tc_fence_after();
#pragma unroll 1
        for (int c0 = 0; c0 < MLP_H; c0 += 32) {
            float v[32];
            tmem_ld32(lane_addr + c0, v);
#pragma unroll
            for (int k = 0; k < 32; ++k) {
                const float z = v[k] + sb1[c0 + k];
                v[k] = z * sigm(z);
            }
#pragma unroll
            for (int q = 0; q < 4; ++q) st8(tile_sm + FW_H1, cm_off(tl, c0 + 8 * q, MLP_H), v + 8 * q);
        }
        wg_tc_sync(g);
        if (tl == 0) {
            gemm_issue(tm, tile_base + FW_H1, base + FW_W2, MLP_H, MLP_TILE, MLP_H, false);
            umma_commit(bar);
        }
        ok = wg_and(g, mbar_wait(bar, phase));
        phase ^= 1;
        if (!ok) break;
        tc_fence_after();
        float acc = 0.f;
#pragma unroll 1
        for (int c0 = 0; c0 < MLP_H; c0 += 32) {
            float v[32];
            tmem_ld32(lane_addr + c0, v);
#pragma unroll
            for (int k = 0; k < 32; ++k) {
                const float z = v[k] + sb2[c0 + k];
                acc = fmaf(z * sigm(z), sw3[c0 + k], acc);
            }
        }
        const float s = acc + b3;
        if (r < n) {
            if (out_s) out_s[r] = s;
            if (corr) {
                const float4 vv = V[r];
                corr[r] = make_float4(s * vv.x, s * vv.y, s * vv.z, s);
            }
        }
        // the next tile's first product overwrites this group's accumulator and X
        wg_tc_sync(g);
    }
    if (!ok && tl == 0) atomicExch(err, 1);
    tc_fence_before();
    __syncthreads();
    if (w == 0) tmem_dealloc(tmem_base, 128 * FW_WG);
}

struct MlpGrads {
    float *dw1, *db1, *dw2, *db2, *dw3, *db3;
    double *loss;
};

// Shared-memory plan of the training kernel (bytes).
constexpr int TR_W1 = 0, TR_W2 = TR_W1 + 128 * 32 * 2, TR_W2T = TR_W2 + 128 * 128 * 2,
              TR_XA = TR_W2T + 128 * 128 * 2, TR_XT = TR_XA + 128 * 32 * 2, TR_R1 = TR_XT + 32 * 128 * 2,
              TR_R2 = TR_R1 + 128 * 128 * 2, TR_R3 = TR_R2 + 128 * 128 * 2, TR_BYTES = TR_R3 + 128 * 128 * 2;
// Tensor-memory columns of the training kernel.
constexpr uint32_t T_A1 = 0, T_A2 = 128, T_G2 = 256, T_G1 = 384;

// Fused forward + backward over the rows of a persistent CTA's tiles, for the loss
//   L = sum_r (s_r^2 a_r - 2 s_r b_r) * scale / 2   (+ a constant),
// i.e. dL/ds_r = scale (s_r a_r - b_r).  With a_r = |V_r|^2, b_r = V_r . R_r and
// scale = 2 / rows this is the mean squared error of the residual s_r V_r against R_r.
// Weight gradients accumulate in tensor memory over the tiles and are added to the global
// FP32 gradients once per CTA; bias and output-layer gradients are reduced across the
// warp by recursive halving and added once per warp.  Tile sequence:
//   1. x -> XA (rows m) and XT (rows i, K = m)
//   2. A1 = x W1^T                                        (tensor cores)
//   3. h1 = bf16(silu(A1 + b1)) -> R1 (rows m), R2 (rows k, K = m)
//   4. A2 = h1 W2^T                                       (tensor cores)
//   5. s, ds; dz2 = ds w3 silu'(z2) -> R3 (rows m), R1 (rows o, K = m); db2, dw3, db3
//   6. A2 = dz2 W2 (dh1);  G2 += dz2^T h1                 (tensor cores)
//   7. dz1 = dh1 silu'(z1) -> R3 (rows o, K = m); db1
//   8. G1 += dz1^T x                                      (tensor cores)
__global__ void __launch_bounds__(MLP_THREADS, 1) k_mlp_train(const __nv_bfloat16 *__restrict__ X,
                                                             const float2 *__restrict__ ab, int n, float scale,
                                                             MlpWeights wt, MlpGrads g, int *__restrict__ err) {
    extern __shared__ __align__(1024) unsigned char sm[];
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t tmem_base;
    __shared__ float sb1[MLP_H], sb2[MLP_H], sw3[MLP_H];
    const int t = threadIdx.x, w = t >> 5, lane = t & 31;
    const int ntiles = (n + MLP_TILE - 1) / MLP_TILE;
    if ((int)blockIdx.x >= ntiles) return;
    if (w == 0) tmem_alloc(smem_u32(&tmem_base), 512);
    if (t == 0) mbar_init(smem_u32(&bar), 1);
    sb1[t] = __ldg(wt.b1 + t);
    sb2[t] = __ldg(wt.b2 + t);
    sw3[t] = __ldg(wt.w3 + t);
    const float b3 = __ldg(wt.b3);
    load_weights(sm, TR_W1, TR_W2, wt, t);
    // W2^T (rows k, K = o): thread t holds row o = t of W2
#pragma unroll 2
    for (int c = 0; c < MLP_H; c += 8) {
        __align__(16) __nv_bfloat16 ww[8];
        *reinterpret_cast<uint4 *>(ww) = __ldg(reinterpret_cast<const uint4 *>(wt.w2 + (size_t)t * MLP_H + c));
#pragma unroll
        for (int k = 0; k < 8; ++k)
            *reinterpret_cast<__nv_bfloat16 *>(sm + TR_W2T + cm_off(c + k, t, MLP_H)) = ww[k];
    }
    const uint32_t bb = smem_u32(&bar), base = smem_u32(sm);
    // per-lane partial sums of the bias / output-layer gradients: element 32 j + lane of chunk j
    float pdb2[4] = {0.f, 0.f, 0.f, 0.f}, pdw3[4] = {0.f, 0.f, 0.f, 0.f}, pdb1[4] = {0.f, 0.f, 0.f, 0.f};
    float pdb3 = 0.f;
    double ploss = 0.0;
    uint32_t phase = 0;
    bool ok = true;
    bool first = true;
    tc_sync();
    const uint32_t tm = tmem_base;
    const uint32_t la = tm + ((uint32_t)(32 * w) << 16);
    const int m = t;   // tile row of this thread (TMEM lane)
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int r = tile * MLP_TILE + m;
        const bool live = r < n;
        // 1. x
        {
            __align__(16) __nv_bfloat16 xx[MLP_IN];
            const uint4 zero = make_uint4(0, 0, 0, 0);
#pragma unroll
            for (int c = 0; c < MLP_IN / 8; ++c) {
                const uint4 v = live ? __ldg(reinterpret_cast<const uint4 *>(X + (size_t)r * MLP_IN) + c) : zero;
                *reinterpret_cast<uint4 *>(sm + TR_XA + cm_off(m, 8 * c, MLP_IN)) = v;
                *reinterpret_cast<uint4 *>(xx + 8 * c) = v;
            }
#pragma unroll
            for (int i = 0; i < MLP_IN; ++i)
                *reinterpret_cast<__nv_bfloat16 *>(sm + TR_XT + cm_off(i, m, MLP_TILE)) = xx[i];
        }
        const float2 abr = live ? __ldg(ab + r) : make_float2(0.f, 0.f);
        tc_sync();
        // 2. layer 1
        if (t == 0) {
            gemm_issue(tm + T_A1, base + TR_XA, base + TR_W1, MLP_IN, MLP_TILE, MLP_H, false);
            umma_commit(bb);
        }
        ok = mbar_wait(bb, phase);
        phase ^= 1;
        if (!__syncthreads_and(ok)) { ok = false; break; }
        tc_fence_after();
        // 3. h1
#pragma unroll 1
        for (int c0 = 0; c0 < MLP_H; c0 += 32) {
            float v[32];
            tmem_ld32(la + T_A1 + c0, v);
#pragma unroll
            for (int k = 0; k < 32; ++k) {
                const float z = v[k] + sb1[c0 + k];
                v[k] = live ? z * sigm(z) : 0.f;
            }
#pragma unroll
            for (int q = 0; q < 4; ++q) st8(sm + TR_R1, cm_off(m, c0 + 8 * q, MLP_H), v + 8 * q);
#pragma unroll
            for (int k = 0; k < 32; ++k) st1(sm + TR_R2, cm_off(c0 + k, m, MLP_TILE), v[k]);
        }
        tc_sync();
        // 4. layer 2
        if (t == 0) {
            gemm_issue(tm + T_A2, base + TR_R1, base + TR_W2, MLP_H, MLP_TILE, MLP_H, false);
            umma_commit(bb);
        }
        ok = mbar_wait(bb, phase);
        phase ^= 1;
        if (!__syncthreads_and(ok)) { ok = false; break; }
        tc_fence_after();
        // 5. output, loss gradient and dz2
        float s = b3;
#pragma unroll 1
        for (int c0 = 0; c0 < MLP_H; c0 += 32) {
            float v[32];
            tmem_ld32(la + T_A2 + c0, v);
#pragma unroll
            for (int k = 0; k < 32; ++k) {
                const float z = v[k] + sb2[c0 + k];
                s = fmaf(z * sigm(z), sw3[c0 + k], s);
            }
        }
        const float ds = live ? scale * (s * abr.x - abr.y) : 0.f;
        if (live) ploss += (double)s * ((double)s * abr.x - 2.0 * abr.y);
        pdb3 += ds;
#pragma unroll 1
        for (int j = 0; j < 4; ++j) {
            const int c0 = 32 * j;
            float v[32], hd[32];
            tmem_ld32(la + T_A2 + c0, v);
#pragma unroll
            for (int k = 0; k < 32; ++k) {
                const float z = v[k] + sb2[c0 + k];
                const float sg = sigm(z);
                hd[k] = z * sg * ds;                                   // dW3 term h2 ds
                v[k] = ds * sw3[c0 + k] * sg * (1.f + z * (1.f - sg)); // dz2
            }
#pragma unroll
            for (int q = 0; q < 4; ++q) st8(sm + TR_R3, cm_off(m, c0 + 8 * q, MLP_H), v + 8 * q);
#pragma unroll
            for (int k = 0; k < 32; ++k) st1(sm + TR_R1, cm_off(c0 + k, m, MLP_TILE), v[k]);
            pdb2[j] += warp_reduce_scatter32(v);
            pdw3[j] += warp_reduce_scatter32(hd);
        }
        tc_sync();
        // 6. dh1 = dz2 W2 into A2; G2 += dz2^T h1
        if (t == 0) {
            gemm_issue(tm + T_A2, base + TR_R3, base + TR_W2T, MLP_H, MLP_TILE, MLP_H, false);
            gemm_issue(tm + T_G2, base + TR_R1, base + TR_R2, MLP_TILE, MLP_H, MLP_H, !first);
            umma_commit(bb);
        }
        ok = mbar_wait(bb, phase);
        phase ^= 1;
        if (!__syncthreads_and(ok)) { ok = false; break; }
        tc_fence_after();
        // 7. dz1 = dh1 silu'(z1)
#pragma unroll 1
        for (int j = 0; j < 4; ++j) {
            const int c0 = 32 * j;
            float v[32], z1[32];
            tmem_ld32(la + T_A2 + c0, v);
            tmem_ld32(la + T_A1 + c0, z1);
#pragma unroll
            for (int k = 0; k < 32; ++k) {
                const float z = z1[k] + sb1[c0 + k];
                const float sg = sigm(z);
                v[k] = live ? v[k] * sg * (1.f + z * (1.f - sg)) : 0.f;
            }
#pragma unroll
            for (int k = 0; k < 32; ++k) st1(sm + TR_R3, cm_off(c0 + k, m, MLP_TILE), v[k]);
            pdb1[j] += warp_reduce_scatter32(v);
        }
        tc_sync();
        // 8. G1 += dz1^T x
        if (t == 0) {
            gemm_issue(tm + T_G1, base + TR_R3, base + TR_XT, MLP_TILE, MLP_H, MLP_IN, !first);
            umma_commit(bb);
        }
        ok = mbar_wait(bb, phase);
        phase ^= 1;
        first = false;
        if (!__syncthreads_and(ok)) { ok = false; break; }
        tc_fence_after();
    }
    if (ok && !first) {
        // weight gradients: TMEM row o = m of G2 (128 columns) and G1 (32 columns)
#pragma unroll 1
        for (int c0 = 0; c0 < MLP_H; c0 += 32) {
            float v[32];
            tmem_ld32(la + T_G2 + c0, v);
#pragma unroll
            for (int k = 0; k < 32; k += 4)
                red_add_v4(g.dw2 + (size_t)m * MLP_H + c0 + k, v[k], v[k + 1], v[k + 2], v[k + 3]);
        }
        {
            float v[32];
            tmem_ld32(la + T_G1, v);
#pragma unroll
            for (int k = 0; k < 32; k += 4)
                red_add_v4(g.dw1 + (size_t)m * MLP_IN + k, v[k], v[k + 1], v[k + 2], v[k + 3]);
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            red_add(g.db2 + 32 * j + lane, pdb2[j]);
            red_add(g.dw3 + 32 * j + lane, pdw3[j]);
            red_add(g.db1 + 32 * j + lane, pdb1[j]);
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            pdb3 += __shfl_xor_sync(0xffffffffu, pdb3, off);
            ploss += __shfl_xor_sync(0xffffffffu, ploss, off);
        }
        if (lane == 0) {
            red_add(g.db3, pdb3);
            red_add_d(g.loss, ploss * (double)scale * 0.5);
        }
    }
    if (!ok && t == 0) atomicExch(err, 1);
    tc_fence_before();
    __syncthreads();
    if (w == 0) tmem_dealloc(tm, 512);
}

// Adam (Kingma & Ba, 2015) on the FP32 master parameters, gradients cleared afterwards:
//   m = b1 m + (1 - b1) g,  v = b2 v + (1 - b2) g^2,  p -= lr (m / c1) / (sqrt(v / c2) + eps)
// with the bias corrections c1 = 1 - b1^t, c2 = 1 - b2^t.
__global__ void k_adam(float *__restrict__ p, float *__restrict__ gr, float *__restrict__ mo, float *__restrict__ ve,
                       int count, float lr, float b1, float b2, float eps, float c1, float c2, float gscale) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const float gi = gr[i] * gscale;
    const float mi = b1 * mo[i] + (1.f - b1) * gi;
    const float vi = b2 * ve[i] + (1.f - b2) * gi * gi;
    mo[i] = mi;
    ve[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    gr[i] = 0.f;
}

__global__ void k_to_bf16(const float *__restrict__ a, __nv_bfloat16 *__restrict__ b, int count) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) b[i] = __float2bfloat16_rn(a[i]);
}

constexpr int P_W1 = 0, P_B1 = P_W1 + MLP_H * MLP_IN, P_W2 = P_B1 + MLP_H, P_B2 = P_W2 + MLP_H * MLP_H,
              P_W3 = P_B2 + MLP_H, P_B3 = P_W3 + MLP_H, P_COUNT = P_B3 + 1;

}  // namespace pdb

// ------------------------------------------------------------------ host side

struct pd_mlp {
    // parameters: FP32 masters, gradients and Adam moments in one layout each:
    // w1 [128][32] | b1 [128] | w2 [128][128] | b2 [128] | w3 [128] | b3 [1]
    float *p = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;
    __nv_bfloat16 *w1b = nullptr, *w2b = nullptr;   // BF16 copies used by the tensor cores
    double *loss = nullptr;
    int *err = nullptr;
    int step = 0;
};

namespace pdb {

static MlpWeights mlp_weights(const pd_mlp *q) {
    MlpWeights w;
    w.w1 = q->w1b;
    w.w2 = q->w2b;
    w.b1 = q->p + P_B1;
    w.b2 = q->p + P_B2;
    w.w3 = q->p + P_W3;
    w.b3 = q->p + P_B3;
    return w;
}

static void mlp_free(pd_mlp *q) {
    dfree(q->p);
    dfree(q->g);
    dfree(q->m);
    dfree(q->v);
    dfree(q->w1b);
    dfree(q->w2b);
    dfree(q->loss);
    dfree(q->err);
}

static int mlp_refresh_bf16(pd_mlp *q, cudaStream_t st) {
    k_to_bf16<<<(MLP_H * MLP_IN + 255) / 256, 256, 0, st>>>(q->p + P_W1, q->w1b, MLP_H * MLP_IN);
    PD_LAUNCHED();
    k_to_bf16<<<(MLP_H * MLP_H + 255) / 256, 256, 0, st>>>(q->p + P_W2, q->w2b, MLP_H * MLP_H);
    PD_LAUNCHED();
    return PD_OK;
}

static int sm_count() {
    static int nsm = 0;
    if (!nsm) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        if (nsm <= 0) nsm = 148;
    }
    return nsm;
}

// Inference launch (also used by the learned correction of the step engine).
int mlp_forward_launch(const pd_mlp *q, const void *X, int n, float *s, const float4 *V, float4 *corr,
                       cudaStream_t st) {
    if (n <= 0) return PD_OK;
    const int tiles = (n + MLP_TILE - 1) / MLP_TILE;
    const int ctas = std::min(sm_count(), (tiles + FW_WG - 1) / FW_WG);
    k_mlp_forward<<<ctas, FW_THREADS, FW_BYTES, st>>>(static_cast<const __nv_bfloat16 *>(X), n, mlp_weights(q), s, V,
                                                        corr, q->err);
    PD_LAUNCHED();
    return PD_OK;
}

}  // namespace pdb

extern "C" {

int pd_mlp_param_count(void) { return P_COUNT; }

int pd_mlp_create(pd_mlp **out) {
    PD_CHECK(out, PD_EINVAL, "pd_mlp_create: null argument");
    *out = nullptr;
    pd_mlp *q = new pd_mlp();
    int rc;
    if ((rc = dalloc(&q->p, P_COUNT)) || (rc = dalloc(&q->g, P_COUNT)) || (rc = dalloc(&q->m, P_COUNT)) ||
        (rc = dalloc(&q->v, P_COUNT)) || (rc = dalloc(&q->w1b, (size_t)MLP_H * MLP_IN)) ||
        (rc = dalloc(&q->w2b, (size_t)MLP_H * MLP_H)) || (rc = dalloc(&q->loss, 1)) || (rc = dalloc(&q->err, 1))) {
        mlp_free(q);
        delete q;
        return rc;
    }
    cudaError_t e = cudaSuccess;
    for (float *a : {q->p, q->g, q->m, q->v})
        if (e == cudaSuccess) e = cudaMemset(a, 0, sizeof(float) * P_COUNT);
    if (e == cudaSuccess) e = cudaMemset(q->loss, 0, sizeof(double));
    if (e == cudaSuccess) e = cudaMemset(q->err, 0, sizeof(int));
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_mlp_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, FW_BYTES);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_mlp_train, cudaFuncAttributeMaxDynamicSharedMemorySize, TR_BYTES);
    if (e != cudaSuccess) {
        set_error("pd_mlp_create: %s", cudaGetErrorString(e));
        mlp_free(q);
        delete q;
        return PD_ECUDA;
    }
    *out = q;
    return PD_OK;
}

int pd_mlp_destroy(pd_mlp *q) {
    if (!q) return PD_OK;
    mlp_free(q);
    delete q;
    return PD_OK;
}

int pd_mlp_set_params(pd_mlp *q, const float *host) {
    PD_CHECK(q && host, PD_EINVAL, "pd_mlp_set_params: null argument");
    PD_CUDA(cudaMemcpy(q->p, host, sizeof(float) * P_COUNT, cudaMemcpyHostToDevice));
    PD_CUDA(cudaMemset(q->m, 0, sizeof(float) * P_COUNT));
    PD_CUDA(cudaMemset(q->v, 0, sizeof(float) * P_COUNT));
    PD_CUDA(cudaMemset(q->g, 0, sizeof(float) * P_COUNT));
    int rc = mlp_refresh_bf16(q, 0);
    if (rc) return rc;
    PD_CUDA(cudaDeviceSynchronize());
    q->step = 0;
    return PD_OK;
}

int pd_mlp_get_params(pd_mlp *q, float *host) {
    PD_CHECK(q && host, PD_EINVAL, "pd_mlp_get_params: null argument");
    PD_CUDA(cudaMemcpy(host, q->p, sizeof(float) * P_COUNT, cudaMemcpyDeviceToHost));
    return PD_OK;
}

int pd_mlp_get_grads(pd_mlp *q, float *host) {
    PD_CHECK(q && host, PD_EINVAL, "pd_mlp_get_grads: null argument");
    PD_CUDA(cudaMemcpy(host, q->g, sizeof(float) * P_COUNT, cudaMemcpyDeviceToHost));
    return PD_OK;
}

int pd_mlp_forward(pd_mlp *q, const void *X, int n, float *s, const float *V4, float *corr4, pd_stream_t sp) {
    PD_CHECK(q && X && (s || corr4), PD_EINVAL, "pd_mlp_forward: null argument");
    PD_CHECK(n >= 0, PD_EINVAL, "pd_mlp_forward: negative row count");
    PD_CHECK(!corr4 || V4, PD_EINVAL, "pd_mlp_forward: the residual output needs V");
    return mlp_forward_launch(q, X, n, s, reinterpret_cast<const float4 *>(V4), reinterpret_cast<float4 *>(corr4),
                              (cudaStream_t)sp);
}

int pd_mlp_train(pd_mlp *q, const void *X, const float *ab, int n, float scale, pd_stream_t sp) {
    PD_CHECK(q && X && ab, PD_EINVAL, "pd_mlp_train: null argument");
    PD_CHECK(n >= 0, PD_EINVAL, "pd_mlp_train: negative row count");
    if (n == 0) return PD_OK;
    MlpGrads g;
    g.dw1 = q->g + P_W1;
    g.db1 = q->g + P_B1;
    g.dw2 = q->g + P_W2;
    g.db2 = q->g + P_B2;
    g.dw3 = q->g + P_W3;
    g.db3 = q->g + P_B3;
    g.loss = q->loss;
    const int tiles = (n + MLP_TILE - 1) / MLP_TILE;
    const int grid = tiles < sm_count() ? tiles : sm_count();
    k_mlp_train<<<grid, MLP_THREADS, TR_BYTES, (cudaStream_t)sp>>>(static_cast<const __nv_bfloat16 *>(X),
                                                                   reinterpret_cast<const float2 *>(ab), n, scale,
                                                                   mlp_weights(q), g, q->err);
    PD_LAUNCHED();
    return PD_OK;
}

int pd_mlp_adam(pd_mlp *q, float lr, float beta1, float beta2, float eps, float grad_scale, pd_stream_t sp) {
    PD_CHECK(q, PD_EINVAL, "pd_mlp_adam: null handle");
    q->step += 1;
    const float c1 = (float)(1.0 - pow((double)beta1, (double)q->step));
    const float c2 = (float)(1.0 - pow((double)beta2, (double)q->step));
    cudaStream_t st = (cudaStream_t)sp;
    k_adam<<<(P_COUNT + 255) / 256, 256, 0, st>>>(q->p, q->g, q->m, q->v, P_COUNT, lr, beta1, beta2, eps, c1, c2,
                                                  grad_scale);
    PD_LAUNCHED();
    return mlp_refresh_bf16(q, st);
}

int pd_mlp_loss(pd_mlp *q, double *out, int reset) {
    PD_CHECK(q && out, PD_EINVAL, "pd_mlp_loss: null argument");
    PD_CUDA(cudaMemcpy(out, q->loss, sizeof(double), cudaMemcpyDeviceToHost));
    if (reset) PD_CUDA(cudaMemset(q->loss, 0, sizeof(double)));
    return PD_OK;
}

int pd_mlp_zero_grads(pd_mlp *q, pd_stream_t sp) {
    PD_CHECK(q, PD_EINVAL, "pd_mlp_zero_grads: null handle");
    PD_CUDA(cudaMemsetAsync(q->g, 0, sizeof(float) * P_COUNT, (cudaStream_t)sp));
    return PD_OK;
}

int pd_mlp_error(pd_mlp *q, int *out) {
    PD_CHECK(q && out, PD_EINVAL, "pd_mlp_error: null argument");
    PD_CUDA(cudaMemcpy(out, q->err, sizeof(int), cudaMemcpyDeviceToHost));
    return PD_OK;
}

}  // extern "C"
