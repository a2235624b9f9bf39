// Cluster-pair list of libpdb200: clustering, outer-list search, pruning and the
// device build/prune decision.  Semantics follow src/clusterpairs/List.jl and
// src/clusterpairs/Engine.jl of ParticleDynamics.jl; the kernel layout is this
// library's own:
//   * binning keys + histogram in one pass, one-CTA scan that also emits the
//     per-column super-cluster metadata, and a deterministic order inside each
//     z-bin (sorted by z, then particle id) so that a build is bit-reproducible;
//   * one 64-thread CTA per super-cluster does the 2x2x2 rank split, the
//     slot map, the force-coordinate pack and both bounding-box levels;
//   * one warp per super-cluster searches its neighbouring columns with
//     ballot-compacted output (count pass, scan, fill pass);
//   * pruning and compaction run in one kernel per super-cluster that writes
//     the working list in place inside the super-cluster's outer segment.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "internal.hpp"

using namespace pdb;

namespace pdb {

static thread_local std::string g_last_error;
static uint64_t g_launches = 0;

void set_error(const char *fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_last_error = buf;
}
void count_launch(int n) { __atomic_add_fetch(&g_launches, (uint64_t)n, __ATOMIC_RELAXED); }

// ------------------------------------------------------------------ binning
// _column_key_kernel! + _column_histogram_kernel! (List.jl:215-250)
__global__ void k_bin(const float *__restrict__ x, const float *__restrict__ y, const float *__restrict__ z, int n,
                      float Lx, float Ly, float Lz, int ncx, int ncy, int nzb, int *__restrict__ bin,
                      int *__restrict__ bcnt, int *__restrict__ counts, int gated) {
    if (gated && counts[W_BUILD] == 0) return;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float xw = wrap_positive(x[i], Lx), yw = wrap_positive(y[i], Ly), zw = wrap_positive(z[i], Lz);
    if (!(isfinite(xw) && isfinite(yw) && isfinite(zw))) {
        counts[W_ERR] = PD_ENONFINITE;  // the list is invalid; keep the bin in range
        xw = 0.f;
        yw = 0.f;
        zw = 0.f;
    }
    // Far outside the box the wrap can round just below 0 or above L: clamp both ends.
    const int cx = max(0, min((int)__fmul_rn(__fdiv_rn(xw, Lx), (float)ncx), ncx - 1));
    const int cy = max(0, min((int)__fmul_rn(__fdiv_rn(yw, Ly), (float)ncy), ncy - 1));
    const int cz = max(0, min((int)__fmul_rn(__fdiv_rn(zw, Lz), (float)nzb), nzb - 1));
    int key = (cx + ncx * cy) * nzb + cz;
    bin[i] = key;
    atomicAdd(&bcnt[key], 1);
}

// Block-wide exclusive scan of one value per thread (1024 threads); returns the
// exclusive prefix and writes the block total to *total.
__device__ __forceinline__ int block_exclusive_scan(int v, int *warp_tot, int *total) {
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int inc = v;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, inc, off);
        if (lane >= off) inc += y;
    }
    if (lane == 31) warp_tot[w] = inc;
    __syncthreads();
    if (w == 0) {
        int nw = (blockDim.x + 31) >> 5;
        int t = lane < nw ? warp_tot[lane] : 0;
        int ti = t;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, ti, off);
            if (lane >= off) ti += y;
        }
        if (lane < nw) warp_tot[lane] = ti - t;  // exclusive warp offsets
        if (lane == nw - 1) *total = ti;
    }
    __syncthreads();
    int r = warp_tot[w] + inc - v;
    __syncthreads();
    return r;
}

// Exclusive scan of the bin histogram (resetting it to zero for the next build),
// then the per-column super-cluster counts, offsets and metadata
// (_exclusive_kernel!, _super_count/_super_offsets/_super_meta_kernel!, List.jl:253-298).
constexpr int SCAN_CHUNK = 8192;   // bins per pass of k_bin_scan (32 KiB of shared memory)

__global__ void __launch_bounds__(1024) k_bin_scan(int *__restrict__ bcnt, int *__restrict__ bstart,
                                                   int *__restrict__ cursor, int nbin, int nzb, int ncol,
                                                   int *__restrict__ col_sc_off, int *__restrict__ sc_first,
                                                   int *__restrict__ sc_n, int *__restrict__ sc_col,
                                                   int *__restrict__ counts, int gated) {
    if (gated && counts[W_BUILD] == 0) return;
    __shared__ int warp_tot[32];
    __shared__ int total;
    // chunks of SCAN_CHUNK bins: coalesced load into shared memory (skewed by one word per
    // 32 against bank conflicts), a serial scan of 8 consecutive bins per thread, one block
    // scan of the thread totals, coalesced store
    __shared__ int sb[SCAN_CHUNK + SCAN_CHUNK / 32];
    const int t = threadIdx.x;
    int carry = 0;
    for (int c0 = 0; c0 < nbin; c0 += SCAN_CHUNK) {
        const int nc = min(SCAN_CHUNK, nbin - c0);
        for (int k = t; k < SCAN_CHUNK; k += blockDim.x) {
            sb[k + (k >> 5)] = k < nc ? bcnt[c0 + k] : 0;
            if (k < nc) bcnt[c0 + k] = 0;
        }
        __syncthreads();
        constexpr int PER = SCAN_CHUNK / 1024;
        int run = 0;
#pragma unroll
        for (int k = 0; k < PER; ++k) {
            const int i = t * PER + k;
            run += sb[i + (i >> 5)];
        }
        int ex = block_exclusive_scan(run, warp_tot, &total) + carry;
#pragma unroll
        for (int k = 0; k < PER; ++k) {
            const int i = t * PER + k;
            const int v = sb[i + (i >> 5)];
            sb[i + (i >> 5)] = ex;
            ex += v;
        }
        carry += total;
        __syncthreads();
        for (int k = t; k < nc; k += blockDim.x) {
            const int v = sb[k + (k >> 5)];
            bstart[c0 + k] = v;
            cursor[c0 + k] = v;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) bstart[nbin] = carry;
    __syncthreads();
    // columns -> super-clusters
    carry = 0;
    for (int base = 0; base < ncol; base += blockDim.x) {
        int c = base + threadIdx.x;
        int cnt = 0, c0 = 0;
        if (c < ncol) {
            c0 = bstart[c * nzb];
            cnt = bstart[(c + 1) * nzb] - c0;
        }
        int nsc = (cnt + SUPER - 1) / SUPER;
        int ex = block_exclusive_scan(nsc, warp_tot, &total) + carry;
        if (c < ncol) {
            col_sc_off[c] = ex;
            for (int k = 0; k < nsc; ++k) {
                int S = ex + k;
                sc_first[S] = c0 + k * SUPER;
                sc_n[S] = min(SUPER, cnt - k * SUPER);
                sc_col[S] = c;
            }
        }
        carry += total;
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        col_sc_off[ncol] = carry;
        counts[W_NS] = carry;
    }
}

// _bin_scatter_kernel! (List.jl:235-243); the atomic cursor order is made
// deterministic by k_bin_sort.
__global__ void k_bin_scatter(const int *__restrict__ bin, int n, int *__restrict__ cursor, int *__restrict__ sorted,
                              const int *__restrict__ counts, int gated) {
    if (gated && counts[W_BUILD] == 0) return;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int p = atomicAdd(&cursor[bin[i]], 1);
    sorted[p] = i;
}

// Order each bin by (wrapped z, particle id), one warp per bin: every lane takes
// entries of the bin, ranks them against all entries of the bin (the keys are
// distinct, so the ranks form a permutation; non-finite z sorts last, by id) and
// the warp writes the bin back in rank order.
__device__ __forceinline__ bool zid_less(float za, int ia, float zb, int ib) {
    const bool fa = za == za, fb = zb == zb;
    if (fa != fb) return fa;   // finite before non-finite
    if (fa && za != zb) return za < zb;
    return ia < ib;
}

__global__ void k_bin_sort(const int *__restrict__ bstart, int nbin, int *__restrict__ sorted, int *__restrict__ tmp,
                           const float *__restrict__ z, float Lz, const int *__restrict__ counts, int gated) {
    if (gated && counts[W_BUILD] == 0) return;
    const int b = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
    if (b >= nbin) return;   // uniform per warp
    const int a = bstart[b], n = bstart[b + 1] - a;
    if (n <= 1) return;
    if (n <= 32) {
        const int id = lane < n ? sorted[a + lane] : 0x7fffffff;
        const float zk = lane < n ? wrap_positive(z[id], Lz) : 0.f;
        int r = 0;
        for (int j = 0; j < n; ++j) {
            const float zj = __shfl_sync(0xffffffffu, zk, j);
            const int ij = __shfl_sync(0xffffffffu, id, j);
            r += zid_less(zj, ij, zk, id) ? 1 : 0;
        }
        __syncwarp();
        if (lane < n) sorted[a + r] = id;
        return;
    }
    // long bins: every entry is ranked against the whole bin and its id is written to its
    // rank position in `tmp` (the bin-key array, free after the scatter); the bin is then
    // copied back
    for (int k = lane; k < n; k += 32) {
        const int id = sorted[a + k];
        const float zk = wrap_positive(z[id], Lz);
        int r = 0;
        for (int j = 0; j < n; ++j) {
            const int ij = sorted[a + j];
            r += zid_less(wrap_positive(z[ij], Lz), ij, zk, id) ? 1 : 0;
        }
        tmp[a + r] = id;
    }
    __syncwarp();
    for (int k = lane; k < n; k += 32) sorted[a + k] = tmp[a + k];
}

// _cluster_assign_kernel! (List.jl:301-358) fused with the order, the pack of
// the build and force coordinates (_pack_kernel!, List.jl:377-413), the cluster
// and super-cluster bounding boxes (_bbox_kernel!, _super_bbox_kernel!,
// List.jl:415-459) and the build reference coordinates.
__global__ void __launch_bounds__(64) k_assign(const int *__restrict__ sorted, const int *__restrict__ sc_first,
                                               const int *__restrict__ sc_n, const float *__restrict__ x,
                                               const float *__restrict__ y, const float *__restrict__ z,
                                               const float *__restrict__ q, const int *__restrict__ type, float Lx,
                                               float Ly, float Lz, int *__restrict__ perm, int *__restrict__ slot_of,
                                               int *__restrict__ order, float4 *__restrict__ xq, int *__restrict__ ts,
                                               float4 *__restrict__ cbc, float4 *__restrict__ cbh,
                                               float4 *__restrict__ sbc, float4 *__restrict__ sbh,
                                               float4 *__restrict__ ref_build, int *__restrict__ counts, int gated) {
    if (gated && counts[W_BUILD] == 0) return;
    const int S = blockIdx.x, t = threadIdx.x;
    const int NS = counts[W_NS];
    const float nanf_ = __int_as_float(0x7fc00000);
    const int base = S * SUPER;
    __shared__ float sx[SUPER], sy[SUPER], sz[SUPER];
    __shared__ int shx[SUPER], shy[SUPER];
    __shared__ int sloc[SUPER];   // local slot -> local particle index (-1 padding)
    __shared__ float4 cc[8], ch[8];
    if (S >= NS) {  // unused super-cluster: padding everywhere
        perm[base + t] = -1;
        xq[base + t] = pad_point(base + t);
        ts[base + t] = 1;
        if (t < 8) {
            cbc[S * 8 + t] = make_float4(nanf_, nanf_, nanf_, 0.f);
            cbh[S * 8 + t] = make_float4(0.f, 0.f, 0.f, 0.f);
        }
        if (t == 0) {
            sbc[S] = make_float4(nanf_, nanf_, nanf_, 0.f);
            sbh[S] = make_float4(0.f, 0.f, 0.f, 0.f);
        }
        return;
    }
    const int n = sc_n[S], first = sc_first[S];
    int i = -1;
    if (t < n) {
        i = sorted[first + t];
        sx[t] = wrap_positive(x[i], Lx);
        sy[t] = wrap_positive(y[i], Ly);
        sz[t] = wrap_positive(z[i], Lz);
    }
    sloc[t] = -1;
    __syncthreads();
    int hx = 0, hy = 0, slot = -1;
    if (t < n) {
        const float xt = sx[t];
        int r = 0;
#pragma unroll 8
        for (int u = 0; u < n; ++u) {
            const float xu = sx[u];
            r += ((xu < xt) || (xu == xt && u < t)) ? 1 : 0;
        }
        hx = r >= ((n + 1) >> 1) ? 1 : 0;
        shx[t] = hx;
    }
    __syncthreads();
    if (t < n) {
        int m = 0, r = 0;
        const float yt = sy[t];
#pragma unroll 8
        for (int u = 0; u < n; ++u) {
            const bool same = shx[u] == hx;
            const float yu = sy[u];
            m += same ? 1 : 0;
            r += (same && ((yu < yt) || (yu == yt && u < t))) ? 1 : 0;
        }
        hy = r >= ((m + 1) >> 1) ? 1 : 0;
        shy[t] = hy;
    }
    __syncthreads();
    if (t < n) {
        int m = 0, r = 0;
        const float zt = sz[t];
#pragma unroll 8
        for (int u = 0; u < n; ++u) {
            const bool same = shx[u] == hx && shy[u] == hy;
            const float zu = sz[u];
            m += same ? 1 : 0;
            r += (same && ((zu < zt) || (zu == zt && u < t))) ? 1 : 0;
        }
        int m0 = (m + 1) >> 1;
        int hz = r >= m0 ? 1 : 0;
        int pos = r - hz * m0;
        int local = (hx * 4 + hy * 2 + hz) * CLUSTER + pos;
        slot = base + local;
        sloc[local] = t;
        slot_of[i] = slot;
    }
    __syncthreads();
    // thread t now owns local slot t
    const int u = sloc[t];
    const int lane = t & 31, w = t >> 5;
    const bool occ = u >= 0;
    const int pi = occ ? sorted[first + u] : -1;
    perm[base + t] = pi;
    // particles in slot order: rank of this slot among the occupied slots of the super-cluster
    unsigned bal = __ballot_sync(0xffffffffu, occ);
    __shared__ int wcount[2];
    if (lane == 0) wcount[w] = __popc(bal);
    __syncthreads();
    if (occ) order[first + (w ? wcount[0] : 0) + __popc(bal & ((1u << lane) - 1u))] = pi;
    // force coordinates (centred image) and charge
    if (occ) {
        float xi = x[pi], yi = y[pi], zi = z[pi];
        float4 v = make_float4(force_coordinate(xi, Lx), force_coordinate(yi, Ly), force_coordinate(zi, Lz),
                               q ? q[pi] : 0.f);
        xq[base + t] = v;
        ts[base + t] = type ? type[pi] : 1;
        ref_build[pi] = make_float4(v.x, v.y, v.z, 0.f);
    } else {
        xq[base + t] = pad_point(base + t);
        ts[base + t] = 1;
    }
    // cluster boxes from the build coordinates (8 consecutive lanes = one cluster)
    const float inf = __int_as_float(0x7f800000);
    float bx = occ ? sx[u] : nanf_, by = occ ? sy[u] : nanf_, bz = occ ? sz[u] : nanf_;
    float lx = occ ? bx : inf, ly = occ ? by : inf, lz = occ ? bz : inf;
    float ux = occ ? bx : -inf, uy = occ ? by : -inf, uz = occ ? bz : -inf;
#pragma unroll
    for (int off = 1; off < 8; off <<= 1) {
        lx = fminf(lx, __shfl_xor_sync(0xffffffffu, lx, off));
        ly = fminf(ly, __shfl_xor_sync(0xffffffffu, ly, off));
        lz = fminf(lz, __shfl_xor_sync(0xffffffffu, lz, off));
        ux = fmaxf(ux, __shfl_xor_sync(0xffffffffu, ux, off));
        uy = fmaxf(uy, __shfl_xor_sync(0xffffffffu, uy, off));
        uz = fmaxf(uz, __shfl_xor_sync(0xffffffffu, uz, off));
    }
    if ((t & 7) == 0) {
        int c = t >> 3;
        float4 ctr, hw;
        if (lx == inf) {
            ctr = make_float4(nanf_, nanf_, nanf_, 0.f);
            hw = make_float4(0.f, 0.f, 0.f, 0.f);
        } else {
            ctr = make_float4(0.5f * (lx + ux), 0.5f * (ly + uy), 0.5f * (lz + uz), 0.f);
            hw = make_float4(0.5f * (ux - lx), 0.5f * (uy - ly), 0.5f * (uz - lz), 0.f);
        }
        cbc[S * 8 + c] = ctr;
        cbh[S * 8 + c] = hw;
        cc[c] = ctr;
        ch[c] = hw;
    }
    __syncthreads();
    if (t == 0) {
        float a = inf, b = inf, d = inf, e = -inf, f = -inf, g = -inf;
        for (int k = 0; k < 8; ++k) {
            float cx = cc[k].x;
            if (!(cx != cx)) {
                a = fminf(a, cx - ch[k].x);
                e = fmaxf(e, cx + ch[k].x);
                b = fminf(b, cc[k].y - ch[k].y);
                f = fmaxf(f, cc[k].y + ch[k].y);
                d = fminf(d, cc[k].z - ch[k].z);
                g = fmaxf(g, cc[k].z + ch[k].z);
            }
        }
        sbc[S] = make_float4(0.5f * (a + e), 0.5f * (b + f), 0.5f * (d + g), 0.f);
        sbh[S] = make_float4(0.5f * (e - a), 0.5f * (f - b), 0.5f * (g - d), 0.f);
    }
}

// Squared gap between two periodic boxes (_bbgap2, List.jl:203-209).
__device__ __forceinline__ float bbgap2(float4 c1, float4 h1, float4 c2, float4 h2, float Lx, float Ly, float Lz) {
    float gx = fmaxf(fabsf(mic(c1.x - c2.x, Lx)) - h1.x - h2.x, 0.f);
    float gy = fmaxf(fabsf(mic(c1.y - c2.y, Ly)) - h1.y - h2.y, 0.f);
    float gz = fmaxf(fabsf(mic(c1.z - c2.z, Lz)) - h1.z - h2.z, 0.f);
    return __fadd_rn(__fadd_rn(__fmul_rn(gx, gx), __fmul_rn(gy, gy)), __fmul_rn(gz, gz));
}

// Outer-list search (_search_warp_kernel!, List.jl:478-557): one CTA of four
// warps per super-cluster.  The neighbouring columns are walked in (dy, dx)
// order; warp w takes columns w, w + 4, ...; lanes take (candidate
// super-cluster, j-cluster) pairs and emit (cj << 8) | i-mask with
// ballot-ordered positions.  The count pass records every column's entry count,
// so the fill pass writes each column at its own offset and the entry order
// equals a serial loop's.
template <bool FILL>
__global__ void __launch_bounds__(128) k_search(const int *__restrict__ sc_col, const int *__restrict__ col_sc_off,
                                                int ncx, int ncy, int mx, int my, const float4 *__restrict__ cbc,
                                                const float4 *__restrict__ cbh, const float4 *__restrict__ sbc,
                                                const float4 *__restrict__ sbh, float Lx, float Ly, float Lz,
                                                float rl2, int *__restrict__ cnt_sc, int *__restrict__ colcnt, int ncs,
                                                const int *__restrict__ scio, uint32_t *__restrict__ cjo,
                                                int *__restrict__ counts, int gated) {
    if (gated && counts[W_BUILD] == 0) return;
    if (FILL && counts[W_ERR] != 0) return;
    const int S = blockIdx.x;
    if (S >= counts[W_NS]) return;
    const int t = threadIdx.x, w = t >> 5, lane = t & 31;
    __shared__ float4 ic[8], ih[8];
    __shared__ int s_off[SEARCH_MAX_COLS];
    __shared__ int s_tot[4];
    if (t < 8) {
        ic[t] = cbc[S * 8 + t];
        ih[t] = cbh[S * 8 + t];
    }
    const int c = sc_col[S];
    const int cx = c % ncx, cy = c / ncx;
    const int nxr = min(2 * mx + 1, ncx), nyr = min(2 * my + 1, ncy);
    const int ncand = nxr * nyr;   // == ncs
    const int x0 = nxr == ncx ? 0 : cx - mx;
    const int y0 = nyr == ncy ? 0 : cy - my;
    if (FILL && w == 0) {
        // exclusive prefix of the column counts of the count pass
        int carry = 0;
        for (int k0 = 0; k0 < ncand; k0 += 32) {
            const int v = k0 + lane < ncand ? colcnt[(size_t)S * ncs + k0 + lane] : 0;
            int inc = v;
#pragma unroll
            for (int off = 1; off < 32; off <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, inc, off);
                if (lane >= off) inc += y;
            }
            if (k0 + lane < ncand) s_off[k0 + lane] = carry + inc - v;
            carry += __shfl_sync(0xffffffffu, inc, 31);
        }
    }
    __syncthreads();
    const float4 s1c = sbc[S], s1h = sbh[S];
    const int e0 = FILL ? scio[S] : 0;
    int total = 0;
    for (int k = w; k < ncand; k += 4) {
        const int dy = k / nxr, dx = k % nxr;
        const int ccx = ((x0 + dx) % ncx + ncx) % ncx, ccy = ((y0 + dy) % ncy + ncy) % ncy;
        const int cc = ccx + ncx * ccy;
        int lo = col_sc_off[cc], hi = col_sc_off[cc + 1];
        lo = max(lo, S);
        const int out = FILL ? e0 + s_off[k] : 0;
        int n = 0;
        for (int base = lo * 8; base < hi * 8; base += 32) {
            const int idx = base + lane;
            uint32_t m = 0;
            int cj = 0;
            if (idx < hi * 8) {
                const int S2 = idx >> 3;
                cj = idx;
                if (bbgap2(s1c, s1h, sbc[S2], sbh[S2], Lx, Ly, Lz) < rl2) {
                    const float4 jc = cbc[cj];
                    if (!(jc.x != jc.x)) {
                        const float4 jh = cbh[cj];
#pragma unroll
                        for (int a = 0; a < 8; ++a) {
                            const int ci = S * 8 + a;
                            if (cj < ci) continue;
                            const float4 ac = ic[a];
                            if (ac.x != ac.x) continue;
                            if (bbgap2(ac, ih[a], jc, jh, Lx, Ly, Lz) < rl2) m |= 1u << a;
                        }
                    }
                }
            }
            const unsigned bal = __ballot_sync(0xffffffffu, m != 0);
            if (FILL && m) cjo[out + n + __popc(bal & ((1u << lane) - 1u))] = ((uint32_t)cj << 8) | m;
            n += __popc(bal);
        }
        if (!FILL && lane == 0) colcnt[(size_t)S * ncs + k] = n;
        total += n;
    }
    if (!FILL) {
        if (lane == 0) s_tot[w] = total;
        __syncthreads();
        if (t == 0) cnt_sc[S] = s_tot[0] + s_tot[1] + s_tot[2] + s_tot[3];
    }
}

// scio = exclusive scan of the per-super-cluster entry counts; NE and the
// capacity latch (_entry_offsets_kernel!, List.jl:561-576).
__global__ void __launch_bounds__(1024) k_entry_scan(const int *__restrict__ cnt_sc, int nsmax, int *__restrict__ scio,
                                                     int necap, int *__restrict__ counts, int gated) {
    if (gated && counts[W_BUILD] == 0) return;
    __shared__ int warp_tot[32];
    __shared__ int total;
    const int NS = counts[W_NS];
    int carry = 0;
    for (int base = 0; base < nsmax; base += blockDim.x) {
        int S = base + threadIdx.x;
        int v = S < NS ? cnt_sc[S] : 0;
        int ex = block_exclusive_scan(v, warp_tot, &total) + carry;
        if (S < nsmax) scio[S] = ex;
        carry += total;
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        scio[nsmax] = carry;
        counts[W_NE] = carry;
        if (carry > necap && counts[W_ERR] == 0) {
            counts[W_ERR] = PD_ECAPACITY;
            counts[W_REQ] = carry;
        }
    }
}

// Distance-only prune of the outer list (_prune_only_kernel!, Kernels.jl:349-394)
// fused with the compaction (_compact_warp_kernel!, List.jl:719-759): one CTA of
// eight warps per super-cluster.  A tile is kept when any pair lies inside the
// prune radius, widened by the rounding bound of a branch-free nearest image.
// The kept entries are written in order at the start of the super-cluster's own
// outer segment, so no global scan is needed.  The prune reference coordinates
// of the super-cluster's particles are refreshed here.
//
// Layout: the segment's entries are staged in shared memory; a warp takes four
// consecutive entries at a time, lane l loading atom l & 7 of entry l >> 3 (one
// coalesced 512-byte load), and prefetches its next group while it evaluates the
// current one.  For each entry, lane (ti, q) pairs i-atom ti of every i-cluster
// in the mask with j-atoms q and q + 4 (the two j halves), taken from the loading
// lanes by shuffles.
//
// Face codes: an atom's side bits mark coordinates within m = 1.01 r_p + prune
// buffer of a face (bit 2d for +, 2d+1 for - in dimension d) and bit 6 marks
// coordinates within half the prune buffer of a face (it may wrap before the
// displacement trigger forces a new prune).  A pair can be nearer as a periodic
// image than as a plain difference only if its atoms sit within r_p of opposite
// faces, so an entry whose i- and j-side bits do not face each other takes the
// plain difference, which then equals the nearest image bit for bit; the other
// entries take the nearest image.  Bit 16 of a kept entry's mask word marks the
// tiles with facing sides or a bit-6 atom: the pair kernel takes the compensated
// periodic difference for those and the plain one for the rest.  Padding slots
// (coordinates above PAD_LIMIT) carry no code and never pass the distance test.
constexpr int PRUNE_CHUNK = 512;

__device__ __forceinline__ int face_code(float x, float y, float z, float slx, float sly, float slz, float wlx,
                                         float wly, float wlz) {
    int c = (x > slx ? 1 : 0) | (x < -slx ? 2 : 0) | (y > sly ? 4 : 0) | (y < -sly ? 8 : 0) | (z > slz ? 16 : 0) |
            (z < -slz ? 32 : 0);
    if (fabsf(x) > wlx || fabsf(y) > wly || fabsf(z) > wlz) c |= 64;
    return c;
}

// With exceptions (xid != null) a tile that holds an excluded pair is kept whatever its distances
// (the pair kernel removes that pair's mesh part), the working entry is marked (bit 17) and its mask
// slot copied to wxid (Kernels.jl:370-373).
__global__ void __launch_bounds__(256) k_prune(const float4 *__restrict__ xq, const int *__restrict__ perm,
                                               const int *__restrict__ scio, const uint32_t *__restrict__ cjo,
                                               uint2 *__restrict__ cjw, int *__restrict__ nw,
                                               float4 *__restrict__ ref_prune, float Lx, float Ly, float Lz,
                                               float rp2, float pbuf, int *__restrict__ counts, int gated,
                                               const int *__restrict__ xid,
                                               const unsigned long long *__restrict__ xmask,
                                               int *__restrict__ wxid) {
    if (gated && counts[W_PRUNE] == 0) return;
    if (counts[W_ERR] != 0) return;
    const int S = blockIdx.x;
    if (S >= counts[W_NS]) return;
    __shared__ float4 si[SUPER];   // i-atom coordinates; .w = 1 for padding
    __shared__ int s_or[256];      // OR of the i-cluster face codes for every i-mask
    __shared__ int s_cc[8];
    __shared__ float4 s_blo[8], s_bhi[8];   // current i-cluster boxes
    __shared__ uint32_t s_ent[PRUNE_CHUNK];
    __shared__ uint32_t s_res[PRUNE_CHUNK];
    __shared__ int s_xid[PRUNE_CHUNK];
    __shared__ int s_wtot[8];
    const int t = threadIdx.x;
    const float wlx = __fsub_rn(__fmul_rn(0.5f, Lx), __fmul_rn(0.5f, pbuf));
    const float wly = __fsub_rn(__fmul_rn(0.5f, Ly), __fmul_rn(0.5f, pbuf));
    const float wlz = __fsub_rn(__fmul_rn(0.5f, Lz), __fmul_rn(0.5f, pbuf));
    const float mg = __fadd_rn(__fmul_rn(1.01f, sqrtf(rp2)), pbuf);
    const float slx = __fsub_rn(__fmul_rn(0.5f, Lx), mg);
    const float sly = __fsub_rn(__fmul_rn(0.5f, Ly), mg);
    const float slz = __fsub_rn(__fmul_rn(0.5f, Lz), mg);
    if (t < SUPER) {
        const float4 v = xq[S * SUPER + t];
        const bool pad = v.x > PAD_LIMIT;
        int c = pad ? 0 : face_code(v.x, v.y, v.z, slx, sly, slz, wlx, wly, wlz);
        c |= __shfl_xor_sync(0xffffffffu, c, 1);
        c |= __shfl_xor_sync(0xffffffffu, c, 2);
        c |= __shfl_xor_sync(0xffffffffu, c, 4);
        if ((t & 7) == 0) s_cc[t >> 3] = c;
        // current box of each i-cluster over its real atoms (padding contributes nothing)
        const float inf = __int_as_float(0x7f800000);
        float lx = pad ? inf : v.x, ly = pad ? inf : v.y, lz = pad ? inf : v.z;
        float ux = pad ? -inf : v.x, uy = pad ? -inf : v.y, uz = pad ? -inf : v.z;
#pragma unroll
        for (int off = 1; off < 8; off <<= 1) {
            lx = fminf(lx, __shfl_xor_sync(0xffffffffu, lx, off));
            ly = fminf(ly, __shfl_xor_sync(0xffffffffu, ly, off));
            lz = fminf(lz, __shfl_xor_sync(0xffffffffu, lz, off));
            ux = fmaxf(ux, __shfl_xor_sync(0xffffffffu, ux, off));
            uy = fmaxf(uy, __shfl_xor_sync(0xffffffffu, uy, off));
            uz = fmaxf(uz, __shfl_xor_sync(0xffffffffu, uz, off));
        }
        if ((t & 7) == 0) {
            s_blo[t >> 3] = make_float4(lx, ly, lz, 0.f);
            s_bhi[t >> 3] = make_float4(ux, uy, uz, 0.f);
        }
        si[t] = make_float4(v.x, v.y, v.z, pad ? 1.f : 0.f);
        const int p = perm[S * SUPER + t];
        if (p >= 0) ref_prune[p] = make_float4(v.x, v.y, v.z, 0.f);
    }
    __syncthreads();
    {
        int c = 0;
#pragma unroll
        for (int a = 0; a < 8; ++a) c |= ((t >> a) & 1) ? s_cc[a] : 0;
        s_or[t] = c;
    }
    const float iLx = 1.f / Lx, iLy = 1.f / Ly, iLz = 1.f / Lz;
    const float Lmax = fmaxf(Lx, fmaxf(Ly, Lz));
    const float epsf = 1.1920929e-7f;
    const float rp2w = __fadd_rn(rp2, __fmul_rn(epsf, __fadd_rn(__fmul_rn(__fmul_rn(16.f, sqrtf(rp2)), Lmax),
                                                                __fmul_rn(16.f, rp2))));
    const int w = t >> 5, lane = t & 31;
    const int ti = lane & 7, q = lane >> 3;
    const int e0 = scio[S], e1 = scio[S + 1];
    int nkeep = 0;
    for (int cb = e0; cb < e1; cb += PRUNE_CHUNK) {
        const int nch = min(e1 - cb, PRUNE_CHUNK);
        for (int k = t; k < nch; k += blockDim.x) {
            s_ent[k] = cjo[cb + k];
            s_xid[k] = xid ? xid[cb + k] : 0;
        }
        __syncthreads();
        const int ngroups = (nch + 3) >> 2;
        // loader role: atom (lane & 7) of entry 4 g + (lane >> 3)
        auto load = [&](int g) {
            const int k = 4 * g + (lane >> 3);
            return (g < ngroups && k < nch) ? xq[(int)(s_ent[k] >> 8) * 8 + (lane & 7)]
                                            : make_float4(2.f * PAD_LIMIT, 2.f * PAD_LIMIT, 2.f * PAD_LIMIT, 0.f);
        };
        float4 nxt = load(w);
        for (int g = w; g < ngroups; g += 8) {
            const float4 cur = nxt;
            nxt = load(g + 8);
            const bool lpad = cur.x > PAD_LIMIT;
            int jc = lpad ? 0 : face_code(cur.x, cur.y, cur.z, slx, sly, slz, wlx, wly, wlz);
            jc |= __shfl_xor_sync(0xffffffffu, jc, 1);
            jc |= __shfl_xor_sync(0xffffffffu, jc, 2);
            jc |= __shfl_xor_sync(0xffffffffu, jc, 4);
            // current box of each loaded j-cluster (8 lanes each, real atoms only)
            const float inf = __int_as_float(0x7f800000);
            float jlx = lpad ? inf : cur.x, jly = lpad ? inf : cur.y, jlz = lpad ? inf : cur.z;
            float jux = lpad ? -inf : cur.x, juy = lpad ? -inf : cur.y, juz = lpad ? -inf : cur.z;
#pragma unroll
            for (int off = 1; off < 8; off <<= 1) {
                jlx = fminf(jlx, __shfl_xor_sync(0xffffffffu, jlx, off));
                jly = fminf(jly, __shfl_xor_sync(0xffffffffu, jly, off));
                jlz = fminf(jlz, __shfl_xor_sync(0xffffffffu, jlz, off));
                jux = fmaxf(jux, __shfl_xor_sync(0xffffffffu, jux, off));
                juy = fmaxf(juy, __shfl_xor_sync(0xffffffffu, juy, off));
                juz = fmaxf(juz, __shfl_xor_sync(0xffffffffu, juz, off));
            }
#pragma unroll 1
            for (int kk = 0; kk < 4; ++kk) {
                const int k = 4 * g + kk;
                if (k >= nch) break;   // uniform per warp
                // the entry word is the same for every lane; the reduction makes that visible
                const uint32_t ent = __reduce_or_sync(0xffffffffu, s_ent[k]);
                const int cj = (int)(ent >> 8);
                uint32_t imask = ent & 0xffu;
                const int sa = kk * 8 + q, sb = sa + 4;
                const float ax = __shfl_sync(0xffffffffu, cur.x, sa), ay = __shfl_sync(0xffffffffu, cur.y, sa),
                            az = __shfl_sync(0xffffffffu, cur.z, sa);
                const float bx = __shfl_sync(0xffffffffu, cur.x, sb), by = __shfl_sync(0xffffffffu, cur.y, sb),
                            bz = __shfl_sync(0xffffffffu, cur.z, sb);
                const int jcode = __shfl_sync(0xffffffffu, jc, kk * 8);
                const int icode = s_or[imask];
                const int jswap = ((jcode & 0x15) << 1) | ((jcode >> 1) & 0x15);
                const bool cross = __any_sync(0xffffffffu, (icode & jswap & 0x3f) != 0);
                const bool mark = cross || ((icode | jcode) & 64);
                uint32_t bits = 0;   // this lane's hits: bit a (j half 0), bit 8 + a (j half 1)
                if (!cross) {
                    // i-clusters whose box lies beyond the prune radius from the j-cluster's box hold no
                    // pair inside it (the factor covers the rounding of the pair distances)
                    {
                        const int src = kk * 8;
                        const float4 bl = s_blo[lane & 7], bh = s_bhi[lane & 7];
                        const float gx = fmaxf(0.f, fmaxf(bl.x - __shfl_sync(0xffffffffu, jux, src),
                                                          __shfl_sync(0xffffffffu, jlx, src) - bh.x));
                        const float gy = fmaxf(0.f, fmaxf(bl.y - __shfl_sync(0xffffffffu, juy, src),
                                                          __shfl_sync(0xffffffffu, jly, src) - bh.y));
                        const float gz = fmaxf(0.f, fmaxf(bl.z - __shfl_sync(0xffffffffu, juz, src),
                                                          __shfl_sync(0xffffffffu, jlz, src) - bh.z));
                        const bool near = fmaf(gx, gx, fmaf(gy, gy, gz * gz)) <= 1.0001f * rp2w;
                        imask &= __ballot_sync(0xffffffffu, near) & 0xffu;
                    }
#pragma unroll
                    for (int a = 0; a < 8; ++a) {
                        if ((imask >> a) & 1u) {
                            const float4 p = si[a * 8 + ti];
                            const float rax = p.x - ax, ray = p.y - ay, raz = p.z - az;
                            const float rbx = p.x - bx, rby = p.y - by, rbz = p.z - bz;
                            const float r2a = fmaf(rax, rax, fmaf(ray, ray, raz * raz));
                            const float r2b = fmaf(rbx, rbx, fmaf(rby, rby, rbz * rbz));
                            const bool self = cj == S * 8 + a;
                            const bool okA = r2a < rp2w && (!self || q > ti);
                            const bool okB = r2b < rp2w && (!self || q + 4 > ti);
                            bits |= (okA ? (1u << a) : 0u) | (okB ? (0x100u << a) : 0u);
                        }
                    }
                } else {
                    const bool apad = __shfl_sync(0xffffffffu, lpad, sa), bpad = __shfl_sync(0xffffffffu, lpad, sb);
#pragma unroll
                    for (int a = 0; a < 8; ++a) {
                        if ((imask >> a) & 1u) {
                            const float4 p = si[a * 8 + ti];
                            const bool ipad = p.w != 0.f;
                            const float rax = p.x - ax, ray = p.y - ay, raz = p.z - az;
                            const float rbx = p.x - bx, rby = p.y - by, rbz = p.z - bz;
                            const float dax = fmaf(-Lx, rintf(rax * iLx), rax);
                            const float day = fmaf(-Ly, rintf(ray * iLy), ray);
                            const float daz = fmaf(-Lz, rintf(raz * iLz), raz);
                            const float dbx = fmaf(-Lx, rintf(rbx * iLx), rbx);
                            const float dby = fmaf(-Ly, rintf(rby * iLy), rby);
                            const float dbz = fmaf(-Lz, rintf(rbz * iLz), rbz);
                            const float r2a = fmaf(dax, dax, fmaf(day, day, daz * daz));
                            const float r2b = fmaf(dbx, dbx, fmaf(dby, dby, dbz * dbz));
                            const bool self = cj == S * 8 + a;
                            const bool okA = !ipad && !apad && r2a < rp2w && (!self || q > ti);
                            const bool okB = !ipad && !bpad && r2b < rp2w && (!self || q + 4 > ti);
                            bits |= (okA ? (1u << a) : 0u) | (okB ? (0x100u << a) : 0u);
                        }
                    }
                }
                bits = __reduce_or_sync(0xffffffffu, bits);
                const int x = s_xid[k];
                if (x > 0 && lane < 8) {   // half tiles of excluded pairs: tj < 4 (low nibbles), tj >= 4
                    const unsigned long long mk = xmask[(size_t)(x - 1) * 8 + lane];
                    const uint32_t xb = ((mk & 0x0F0F0F0F0F0F0F0Full) ? (1u << lane) : 0u) |
                                        ((mk & 0xF0F0F0F0F0F0F0F0ull) ? (0x100u << lane) : 0u);
                    bits |= __reduce_or_sync(0xffu, xb);
                }
                if (lane == 0) s_res[k] = bits | (mark ? 0x10000u : 0u) | (x > 0 ? 0x20000u : 0u);
            }
        }
        __syncthreads();
        // in-order compaction of the chunk by the whole block
        for (int base = 0; base < nch; base += blockDim.x) {
            const int k = base + t;
            const uint32_t m = k < nch ? s_res[k] : 0u;
            const bool live = (m & 0xffffu) != 0;
            const unsigned bal = __ballot_sync(0xffffffffu, live);
            if (lane == 0) s_wtot[w] = __popc(bal);
            __syncthreads();
            int off = 0, tot = 0;
#pragma unroll
            for (int v = 0; v < 8; ++v) {
                const int c = s_wtot[v];
                off += v < w ? c : 0;
                tot += c;
            }
            if (live) {
                const int ew = e0 + nkeep + off + __popc(bal & ((1u << lane) - 1u));
                cjw[ew] = make_uint2(s_ent[k] >> 8, m);
                if (wxid) wxid[ew] = (m & 0x20000u) ? s_xid[k] : 0;
            }
            nkeep += tot;
            __syncthreads();
        }
    }
    if (t == 0) nw[S] = nkeep;
}

// Displacement ratios since the build and the last prune (_displacement_kernel!,
// List.jl:787-819), reduced per block and combined with an integer max on the
// float bits (non-negative floats order like their bit patterns).
__global__ void __launch_bounds__(256) k_displacement(const float *__restrict__ x, const float *__restrict__ y,
                                                      const float *__restrict__ z, int n,
                                                      const float4 *__restrict__ rb, const float4 *__restrict__ rp,
                                                      float Lx, float Ly, float Lz, float tb2, float tp2,
                                                      int *__restrict__ counts) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    float ra = 0.f, rbv = 0.f;
    if (i < n) {
        float xi = x[i], yi = y[i], zi = z[i];
        float4 b = rb[i];
        float dx = mic(xi - b.x, Lx), dy = mic(yi - b.y, Ly), dz = mic(zi - b.z, Lz);
        float d2 = dx * dx + dy * dy + dz * dz;
        rbv = tb2 > 0.f ? d2 / tb2 : (d2 > 0.f ? __int_as_float(0x7f800000) : 0.f);
        if (!isfinite(rbv)) rbv = __int_as_float(0x7f800000);
        float4 p = rp[i];
        dx = mic(xi - p.x, Lx);
        dy = mic(yi - p.y, Ly);
        dz = mic(zi - p.z, Lz);
        d2 = dx * dx + dy * dy + dz * dz;
        float rpv = tp2 > 0.f ? d2 / tp2 : (d2 > 0.f ? __int_as_float(0x7f800000) : 0.f);
        ra = fmaxf(rbv, rpv);
    }
    ra = warp_max(ra);
    rbv = warp_max(rbv);
    __shared__ float sh[2][8];
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) {
        sh[0][w] = ra;
        sh[1][w] = rbv;
    }
    __syncthreads();
    if (w == 0) {
        int nwp = (blockDim.x + 31) >> 5;
        float a = lane < nwp ? sh[0][lane] : 0.f;
        float c = lane < nwp ? sh[1][lane] : 0.f;
        a = warp_max(a);
        c = warp_max(c);
        if (lane == 0) {
            atomicMax(&counts[W_FLAG_ANY], __float_as_int(a));
            atomicMax(&counts[W_FLAG_BUILD], __float_as_int(c));
        }
    }
}

// Device build/prune decision (_decide_kernel!, Engine.jl:301-324).
__global__ void k_decide(int *__restrict__ counts, int nstlist, int nstprune) {
    float anyr = __int_as_float(counts[W_FLAG_ANY]);
    float br = __int_as_float(counts[W_FLAG_BUILD]);
    bool build, prune;
    if (nstlist > 0) {
        int k = counts[W_DSTEP];
        counts[W_DSTEP] = k + 1;
        build = (k % nstlist == 0) || (counts[W_REQUEST] != 0) || !isfinite(br);
        prune = build || (nstprune > 0 && k % nstprune == 0);
    } else {
        build = (br > 1.0f) || (counts[W_REQUEST] != 0);
        prune = build || (anyr > 1.0f);
    }
    counts[W_BUILD] = build ? 1 : 0;
    counts[W_PRUNE] = prune ? 1 : 0;
    counts[W_REQUEST] = 0;
    counts[W_NBUILD] += build ? 1 : 0;
    counts[W_NPRUNE] += prune ? 1 : 0;
    counts[W_FLAG_ANY] = 0;
    counts[W_FLAG_BUILD] = 0;
}

// Build entry: reset the error latch when this step builds (List.jl:985).
__global__ void k_build_begin(int *__restrict__ counts, int gated) {
    if (gated && counts[W_BUILD] == 0) return;
    counts[W_ERR] = 0;
    counts[W_REQ] = 0;
}

// _pack_kernel! (List.jl:377-413) in the force coordinates of the current positions.
__global__ void k_pack(const int *__restrict__ perm, int nslot, const float *__restrict__ x,
                       const float *__restrict__ y, const float *__restrict__ z, const float *__restrict__ q,
                       const int *__restrict__ type, float Lx, float Ly, float Lz, float4 *__restrict__ xq,
                       int *__restrict__ ts) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nslot) return;
    int i = perm[s];
    if (i < 0) return;  // padding keeps its far-away coordinates and zero charge
    xq[s] = make_float4(force_coordinate(x[i], Lx), force_coordinate(y[i], Ly), force_coordinate(z[i], Lz),
                        q ? q[i] : 0.f);
    if (type) ts[s] = type[i];
}

__global__ void k_set_word(int *counts, int word, int value) { counts[word] = value; }

// ------------------------------------------------------------------ host side

int cluster_read_counts(pd_cluster *c, int *host, cudaStream_t s) {
    PD_CUDA(cudaMemcpyAsync(host, c->counts, W_LEN * sizeof(int), cudaMemcpyDeviceToHost, s));
    PD_CUDA(cudaStreamSynchronize(s));
    return PD_OK;
}

int cluster_set_word(pd_cluster *c, int word, int value, cudaStream_t s) {
    k_set_word<<<1, 1, 0, s>>>(c->counts, word, value);
    PD_LAUNCHED();
    return PD_OK;
}

static void free_entries(pd_cluster *c) {
    dfree(c->cjo);
    dfree(c->cjw);
    dfree(c->xid);
    dfree(c->wxid);
}

static int alloc_entries(pd_cluster *c, int necap) {
    free_entries(c);
    c->necap = necap;
    int rc;
    if ((rc = dalloc(&c->cjo, (size_t)necap))) return rc;
    if ((rc = dalloc(&c->cjw, (size_t)necap))) return rc;
    if (c->nexc > 0) {   // exclusion slots follow the entry storage
        if ((rc = dalloc(&c->xid, (size_t)necap)) || (rc = dalloc(&c->wxid, (size_t)necap))) return rc;
        PD_CUDA(cudaMemset(c->xid, 0, sizeof(int) * (size_t)necap));
        PD_CUDA(cudaMemset(c->wxid, 0, sizeof(int) * (size_t)necap));
    }
    return PD_OK;
}

// ---------------------------------------------------------------- exceptions
// _exclusion_kernel! (List.jl:629-688) after a build.  An exception pair belongs to the tile of its
// lower cluster (the lower slot inside one cluster): super-cluster S = ci / 8, i-cluster k = ci % 8.
// Pass 1 finds the outer entry of S holding cj with bit k set and gives it a mask slot (xid, from 1);
// pass 2 sets the pair's bit (ti * 8 + tj) in that slot's mask of i-cluster k and records the pairs
// computed outside the tiles: in-list pairs with a nonzero scale (coef = scale, added to the
// excluded tile pair's zero) and pairs beyond the list (coef = scale - 1, the mesh holds their 1/r).

__global__ void k_excl_begin(int *__restrict__ xid, const int *__restrict__ scio, int *__restrict__ counts, int gated) {
    if (gated && counts[W_BUILD] == 0) return;
    if (counts[W_ERR] != 0) return;   // an overflowed list is rebuilt after growth
    const int ne = scio[counts[W_NS]];
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < ne; e += gridDim.x * blockDim.x) xid[e] = 0;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        counts[W_NX] = 0;
        counts[W_NP] = 0;
    }
}

// One warp per particle i takes its exception pairs in turn (the orientation with the lower slot);
// the warp finds the pair's outer entry (super-cluster S = ci / 8 with j-cluster cj and i-cluster
// bit k = ci % 8) by scanning S's segment 32 entries at a time.
template <int PASS>
__global__ void k_excl_pass(int n, const int *__restrict__ exo, const int *__restrict__ exj,
                            const float *__restrict__ exs, const int *__restrict__ slot_of,
                            const int *__restrict__ scio, const uint32_t *__restrict__ cjo, int *__restrict__ xid,
                            unsigned long long *__restrict__ xmask, int *__restrict__ xpi, int *__restrict__ xpj,
                            float *__restrict__ xpc, int *__restrict__ counts, int gated) {
    if (gated && counts[W_BUILD] == 0) return;
    if (counts[W_ERR] != 0) return;
    const int lane = threadIdx.x & 31;
    const int i = (int)(((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (i >= n) return;   // uniform over the warp
    const int si = slot_of[i];
    for (int p = exo[i]; p < exo[i + 1]; ++p) {
        const int j = exj[p];
        const int sj = slot_of[j];
        const int ci = si >> 3, cj = sj >> 3;
        if (!(ci < cj || (ci == cj && (si & 7) < (sj & 7)))) continue;   // the other orientation
        const int S = ci >> 3, k = ci & 7;
        const int b1 = scio[S + 1];
        int e = -1;
        for (int b = scio[S]; b < b1 && e < 0; b += 32) {
            bool hit = false;
            if (b + lane < b1) {
                const uint32_t ent = cjo[b + lane];
                hit = (int)(ent >> 8) == cj && ((ent >> k) & 1u);
            }
            const unsigned m = __ballot_sync(0xffffffffu, hit);
            if (m) e = b + __ffs(m) - 1;
        }
        if (lane == 0) {
            const float sc = exs[p];
            if (PASS == 1) {
                if (e >= 0 && atomicCAS(&xid[e], 0, -1) == 0) xid[e] = atomicAdd(&counts[W_NX], 1) + 1;
            } else if (e >= 0) {
                const unsigned long long bit = 1ull << ((si & 7) * 8 + (sj & 7));
                atomicOr(&xmask[(size_t)(xid[e] - 1) * 8 + k], bit);
                if (sc != 0.f) {
                    const int m = atomicAdd(&counts[W_NP], 1);
                    xpi[m] = i;
                    xpj[m] = j;
                    xpc[m] = sc;
                }
            } else {
                const int m = atomicAdd(&counts[W_NP], 1);
                xpi[m] = i;
                xpj[m] = j;
                xpc[m] = sc - 1.f;
            }
        }
    }
}

__global__ void k_excl_masks_clear(unsigned long long *__restrict__ xmask, int *__restrict__ counts, int gated) {
    if (gated && counts[W_BUILD] == 0) return;
    const int m = 8 * counts[W_NX];
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < m; k += gridDim.x * blockDim.x) xmask[k] = 0ull;
}

static void free_geometry(pd_cluster *c) {
    dfree(c->bin);
    dfree(c->bcnt);
    dfree(c->bstart);
    dfree(c->cursor);
    dfree(c->sorted);
    dfree(c->col_sc_off);
    dfree(c->sc_first);
    dfree(c->sc_n);
    dfree(c->sc_col);
    dfree(c->perm);
    dfree(c->xq);
    dfree(c->ts);
    dfree(c->cbc);
    dfree(c->cbh);
    dfree(c->sbc);
    dfree(c->sbh);
    dfree(c->cnt_sc);
    dfree(c->colcnt);
    dfree(c->scio);
    dfree(c->nw);
    dfree(c->fc);
    dfree(c->vc);
}

int cluster_build_launch(pd_cluster *c, const float *x, const float *y, const float *z, const float *q,
                         const int *type, int conditional, cudaStream_t s) {
    const int N = c->n, g = conditional ? 1 : 0;
    const float Lx = c->L[0], Ly = c->L[1], Lz = c->L[2];
    k_build_begin<<<1, 1, 0, s>>>(c->counts, g);
    PD_LAUNCHED();
    k_bin<<<(N + 255) / 256, 256, 0, s>>>(x, y, z, N, Lx, Ly, Lz, c->ncx, c->ncy, c->nzb, c->bin, c->bcnt, c->counts, g);
    PD_LAUNCHED();
    k_bin_scan<<<1, 1024, 0, s>>>(c->bcnt, c->bstart, c->cursor, c->nbin, c->nzb, c->ncol, c->col_sc_off, c->sc_first,
                                  c->sc_n, c->sc_col, c->counts, g);
    PD_LAUNCHED();
    k_bin_scatter<<<(N + 255) / 256, 256, 0, s>>>(c->bin, N, c->cursor, c->sorted, c->counts, g);
    PD_LAUNCHED();
    k_bin_sort<<<(int)(((long long)c->nbin * 32 + 255) / 256), 256, 0, s>>>(c->bstart, c->nbin, c->sorted, c->bin, z, Lz,
                                                                          c->counts, g);
    PD_LAUNCHED();
    k_assign<<<c->nsmax, SUPER, 0, s>>>(c->sorted, c->sc_first, c->sc_n, x, y, z, q, type, Lx, Ly, Lz, c->perm,
                                        c->slot_of, c->order, c->xq, c->ts, c->cbc, c->cbh, c->sbc, c->sbh,
                                        c->ref_build, c->counts, g);
    PD_LAUNCHED();
    const float rl2 = (float)c->rlist * (float)c->rlist;
    k_search<false><<<c->nsmax, 128, 0, s>>>(c->sc_col, c->col_sc_off, c->ncx, c->ncy, c->mx, c->my, c->cbc, c->cbh,
                                             c->sbc, c->sbh, Lx, Ly, Lz, rl2, c->cnt_sc, c->colcnt, c->ncs, c->scio,
                                             c->cjo, c->counts, g);
    PD_LAUNCHED();
    k_entry_scan<<<1, 1024, 0, s>>>(c->cnt_sc, c->nsmax, c->scio, c->necap, c->counts, g);
    PD_LAUNCHED();
    k_search<true><<<c->nsmax, 128, 0, s>>>(c->sc_col, c->col_sc_off, c->ncx, c->ncy, c->mx, c->my, c->cbc, c->cbh,
                                            c->sbc, c->sbh, Lx, Ly, Lz, rl2, c->cnt_sc, c->colcnt, c->ncs, c->scio,
                                            c->cjo, c->counts, g);
    PD_LAUNCHED();
    if (c->nexc > 0) {
        const int nb = (int)(((long long)N * 32 + 255) / 256);
        k_excl_begin<<<2 * c->num_sms, 256, 0, s>>>(c->xid, c->scio, c->counts, g);
        PD_LAUNCHED();
        k_excl_pass<1><<<nb, 256, 0, s>>>(N, c->exo, c->exj, c->exs, c->slot_of, c->scio, c->cjo, c->xid, c->xmask,
                                          c->xpi, c->xpj, c->xpc, c->counts, g);
        PD_LAUNCHED();
        k_excl_masks_clear<<<2 * c->num_sms, 256, 0, s>>>(c->xmask, c->counts, g);
        PD_LAUNCHED();
        k_excl_pass<2><<<nb, 256, 0, s>>>(N, c->exo, c->exj, c->exs, c->slot_of, c->scio, c->cjo, c->xid, c->xmask,
                                          c->xpi, c->xpj, c->xpc, c->counts, g);
        PD_LAUNCHED();
    }
    return PD_OK;
}

int cluster_prune_launch(pd_cluster *c, int conditional, cudaStream_t s) {
    const double rp = c->p.rmax + c->p.prune_buffer;
    const float rp2 = (float)rp * (float)rp;
    k_prune<<<c->nsmax, 256, 0, s>>>(c->xq, c->perm, c->scio, c->cjo, c->cjw, c->nw, c->ref_prune, c->L[0], c->L[1],
                                     c->L[2], rp2, (float)c->p.prune_buffer, c->counts, conditional ? 1 : 0,
                                     c->nexc > 0 ? c->xid : nullptr, c->xmask, c->nexc > 0 ? c->wxid : nullptr);
    PD_LAUNCHED();
    return PD_OK;
}

int cluster_decide_launch(pd_cluster *c, const float *x, const float *y, const float *z, int fixed, cudaStream_t s) {
    const float hb = (float)(0.5 * c->p.skin), hp = (float)(0.5 * c->p.prune_buffer);
    k_displacement<<<(c->n + 255) / 256, 256, 0, s>>>(x, y, z, c->n, c->ref_build, c->ref_prune, c->L[0], c->L[1],
                                                      c->L[2], hb * hb, hp * hp, c->counts);
    PD_LAUNCHED();
    k_decide<<<1, 1, 0, s>>>(c->counts, fixed ? c->p.nstlist : 0, c->p.nstprune);
    PD_LAUNCHED();
    return PD_OK;
}

int cluster_check_params(const pd_cluster_params *p) {
    PD_CHECK(p->n >= 1, PD_EINVAL, "cluster-pair engine needs at least one particle");
    PD_CHECK(p->skin >= 0 && p->prune_buffer >= 0 && p->prune_buffer <= p->skin, PD_EINVAL,
             "cluster pairs need 0 <= prune_buffer <= skin.");
    PD_CHECK(p->rmax > 0, PD_EINVAL, "The cluster-pair backend needs a vdW term or an electrostatics solver.");
    PD_CHECK(p->lj_kind >= PD_LJ_NONE && p->lj_kind <= PD_LJ_TABLE, PD_EINVAL, "unknown LJ kind %d", p->lj_kind);
    PD_CHECK(p->lj_kind != PD_LJ_TABLE || (p->ntypes >= 1 && p->ntypes <= PD_MAX_TYPES), PD_EINVAL,
             "LJ type table needs 1 <= ntypes <= %d", PD_MAX_TYPES);
    PD_CHECK(!p->coulomb || (p->coul_ne >= 1 && p->coul_ne <= PD_MAX_POLY && p->coul_nf >= 1 &&
                             p->coul_nf <= PD_MAX_POLY),
             PD_EINVAL, "Coulomb polynomial needs 1..%d coefficients", PD_MAX_POLY);
    return PD_OK;
}

// setup! (List.jl:874-937): super-cluster edge b = cbrt(64 / rho), z-bins of about 4 particles,
// NSmax = ceil(N / 64) + ncol, search span with a 2 % shrink allowance.
int cluster_geometry(int N, double rlist, const double box[3], ClusterGeom *g) {
    const double Lx = (float)box[0], Ly = (float)box[1], Lz = (float)box[2];
    PD_CHECK(std::isfinite(Lx) && std::isfinite(Ly) && std::isfinite(Lz) && Lx > 0 && Ly > 0 && Lz > 0, PD_EINVAL,
             "box lengths must be finite and positive");
    PD_CHECK(std::min(Lx, std::min(Ly, Lz)) > 2 * rlist, PD_EINVAL,
             "cluster-pair list radius %g needs every box length above %g.", rlist, 2 * rlist);
    g->rlist = rlist;
    g->rho = N / (Lx * Ly * Lz);
    const double b = std::cbrt(SUPER / g->rho);
    g->ncx = std::max(1, (int)std::floor(Lx / b));
    g->ncy = std::max(1, (int)std::floor(Ly / b));
    g->ncol = g->ncx * g->ncy;
    g->nzb = std::max(1, (int)std::nearbyint(Lz * g->rho * (Lx / g->ncx) * (Ly / g->ncy) / 4));
    g->nbin = (long long)g->ncol * g->nzb;
    PD_CHECK(g->nbin < (1LL << 30), PD_EINVAL, "cluster-pair binning exceeds int range.");
    g->nsmax = (N + SUPER - 1) / SUPER + g->ncol;
    g->nslot = SUPER * g->nsmax;
    const double shrink = 0.98;
    g->mx = (int)std::floor(rlist / (shrink * Lx / g->ncx)) + 1;
    g->my = (int)std::floor(rlist / (shrink * Ly / g->ncy)) + 1;
    g->ncs = std::min(2 * g->mx + 1, g->ncx) * std::min(2 * g->my + 1, g->ncy);
    PD_CHECK(g->ncs <= SEARCH_MAX_COLS, PD_EINVAL,
             "cluster-pair search needs %d columns per super-cluster (limit %d).", g->ncs, SEARCH_MAX_COLS);
    return PD_OK;
}

void cluster_pair_params(const pd_cluster_params *p, const double box[3], PairParams *pp) {
    memset(pp, 0, sizeof *pp);
    pp->Lx = (float)box[0];
    pp->Ly = (float)box[1];
    pp->Lz = (float)box[2];
    pp->lj_kind = p->lj_kind;
    pp->c6 = p->lj_c6;
    pp->c12 = p->lj_c12;
    pp->lrc2 = p->lj_rc2;
    pp->esh = p->lj_esh;
    pp->ntypes = p->lj_kind == PD_LJ_TABLE ? p->ntypes : 1;
    pp->coulomb = p->coulomb;
    pp->C = p->coul_C;
    pp->rc2 = p->coul_rc2;
    pp->sx = p->coul_sx;
    pp->eshift = p->coul_eshift;
    pp->ne = p->coulomb ? p->coul_ne : 1;
    pp->nf = p->coulomb ? p->coul_nf : 1;
    pp->has_mesh = p->coulomb ? p->coul_has_mesh : 0;
    for (int k = 0; k < PD_MAX_POLY; ++k) {   // coefficients past the fitted length are zero (exact padding)
        pp->pe[k] = k < pp->ne ? p->coul_pe[k] : 0.f;
        pp->pf[k] = k < pp->nf ? p->coul_pf[k] : 0.f;
    }
}

}  // namespace pdb

// ------------------------------------------------------------------ C ABI

extern "C" {

int pd_version(void) { return 100; }

const char *pd_strerror(int code) {
    switch (code) {
        case PD_OK: return "ok";
        case PD_EINVAL: return "invalid argument";
        case PD_ENOMEM: return "device allocation failed";
        case PD_ECAPACITY: return "outer cluster list capacity exceeded";
        case PD_ENONFINITE: return "non-finite coordinates";
        case PD_ECUFFT: return "cuFFT failure";
        case PD_ECUDA: return "CUDA runtime failure";
        case PD_ESTATE: return "call out of order";
        case PD_ENOTSUP: return "not supported";
        default: return "unknown status";
    }
}

const char *pd_last_error(void) { return pdb::g_last_error.c_str(); }

uint64_t pd_launch_count(void) { return __atomic_load_n(&pdb::g_launches, __ATOMIC_RELAXED); }

int pd_cluster_create(pd_cluster **out, const pd_cluster_params *p, const double box[3]) {
    PD_CHECK(out && p && box, PD_EINVAL, "pd_cluster_create: null argument");
    *out = nullptr;
    int rc = cluster_check_params(p);
    if (rc) return rc;
    pd_cluster *c = new pd_cluster();
    c->p = *p;
    c->n = p->n;
    if ((rc = dalloc(&c->counts, W_LEN)) || (rc = dalloc(&c->slot_of, (size_t)c->n)) ||
        (rc = dalloc(&c->order, (size_t)c->n)) || (rc = dalloc(&c->ref_build, (size_t)c->n)) ||
        (rc = dalloc(&c->ref_prune, (size_t)c->n)) || (rc = dalloc(&c->lj_table, PD_MAX_TYPES * PD_MAX_TYPES * 4))) {
        pd_cluster_destroy(c);
        return rc;
    }
    cudaMemset(c->counts, 0, W_LEN * sizeof(int));
    cudaMemcpy(c->lj_table, p->lj_table, sizeof(p->lj_table), cudaMemcpyHostToDevice);
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, dev);
    cluster_pair_params(p, box, &c->pp);   // kernel parameters of the pair pass
    if ((rc = pd_cluster_setup(c, box))) {
        pd_cluster_destroy(c);
        return rc;
    }
    *out = c;
    return PD_OK;
}

int pd_cluster_destroy(pd_cluster *c) {
    if (!c) return PD_OK;
    free_geometry(c);
    free_entries(c);
    cluster_free_exceptions(c);
    dfree(c->counts);
    dfree(c->slot_of);
    dfree(c->order);
    dfree(c->ref_build);
    dfree(c->ref_prune);
    dfree(c->lj_table);
    delete c;
    return PD_OK;
}

int pd_cluster_setup(pd_cluster *c, const double box[3]) {
    PD_CHECK(c && box, PD_EINVAL, "pd_cluster_setup: null argument");
    const int N = c->n;
    ClusterGeom g;
    int grc = cluster_geometry(N, c->p.rmax + c->p.skin, box, &g);
    if (grc) return grc;
    const double rlist = g.rlist, rho = g.rho;
    const int ncx = g.ncx, ncy = g.ncy, ncol = g.ncol, nzb = g.nzb, nsmax = g.nsmax, nslot = g.nslot;
    const int mx = g.mx, my = g.my, ncs = g.ncs;
    const long long nbin = g.nbin;
    bool same_geom = c->nslot > 0 && ncx == c->ncx && ncy == c->ncy && nzb == c->nzb && nsmax == c->nsmax &&
                     ncs == c->ncs;
    for (int d = 0; d < 3; ++d) {
        c->box[d] = box[d];
        c->L[d] = (float)box[d];
    }
    c->rlist = rlist;
    c->ncx = ncx;
    c->ncy = ncy;
    c->nzb = nzb;
    c->ncol = ncol;
    c->nbin = (int)nbin;
    c->mx = mx;
    c->my = my;
    c->pp.Lx = c->L[0];
    c->pp.Ly = c->L[1];
    c->pp.Lz = c->L[2];
    c->nsplit = std::max(1, std::min(32, (32 * c->num_sms + nsmax - 1) / std::max(nsmax, 1)));
    if (!same_geom) {
        free_geometry(c);
        c->ncs = ncs;
        c->nsmax = nsmax;
        c->nslot = nslot;
        int rc;
        if ((rc = dalloc(&c->bin, (size_t)N)) || (rc = dalloc(&c->bcnt, (size_t)nbin)) ||
            (rc = dalloc(&c->bstart, (size_t)nbin + 1)) || (rc = dalloc(&c->cursor, (size_t)nbin)) ||
            (rc = dalloc(&c->sorted, (size_t)N)) || (rc = dalloc(&c->col_sc_off, (size_t)ncol + 1)) ||
            (rc = dalloc(&c->sc_first, (size_t)nsmax)) || (rc = dalloc(&c->sc_n, (size_t)nsmax)) ||
            (rc = dalloc(&c->sc_col, (size_t)nsmax)) || (rc = dalloc(&c->perm, (size_t)nslot)) ||
            (rc = dalloc(&c->xq, (size_t)nslot)) || (rc = dalloc(&c->ts, (size_t)nslot)) ||
            (rc = dalloc(&c->cbc, (size_t)8 * nsmax)) || (rc = dalloc(&c->cbh, (size_t)8 * nsmax)) ||
            (rc = dalloc(&c->sbc, (size_t)nsmax)) || (rc = dalloc(&c->sbh, (size_t)nsmax)) ||
            (rc = dalloc(&c->cnt_sc, (size_t)nsmax)) || (rc = dalloc(&c->colcnt, (size_t)nsmax * ncs)) ||
            (rc = dalloc(&c->scio, (size_t)nsmax + 1)) ||
            (rc = dalloc(&c->nw, (size_t)nsmax)) || (rc = dalloc(&c->fc, (size_t)nslot)) ||
            (rc = dalloc(&c->vc, (size_t)6 * nslot)))
            return rc;
        PD_CUDA(cudaMemset(c->bcnt, 0, sizeof(int) * (size_t)nbin));
        PD_CUDA(cudaMemset(c->fc, 0, sizeof(float4) * (size_t)nslot));
        PD_CUDA(cudaMemset(c->vc, 0, sizeof(float) * 6 * (size_t)nslot));
        PD_CUDA(cudaMemset(c->nw, 0, sizeof(int) * (size_t)nsmax));
        PD_CUDA(cudaMemset(c->scio, 0, sizeof(int) * ((size_t)nsmax + 1)));
        PD_CUDA(cudaMemset(c->perm, 0xff, sizeof(int) * (size_t)nslot));
        if (c->necap == 0) {
            // First sizing: an estimate of the outer entries per super-cluster from the
            // number of clusters within r_list of a cluster, with headroom; an overflow
            // latches PD_ECAPACITY and pd_cluster_grow resizes (List.jl:959-969).
            const double cl = std::cbrt(CLUSTER / rho);
            const double reach = rlist + 2.0 * cl;
            const double per_cluster = (4.0 / 3.0) * M_PI * reach * reach * reach * rho / CLUSTER;
            long long est = (long long)(nsmax * (0.5 * 8.0 * per_cluster + 16.0) * 1.5) + 4096;
            est = std::min<long long>(est, (long long)nsmax * 64LL * 8LL + 4096);
            int rc2 = alloc_entries(c, (int)std::min<long long>(est, (1LL << 30)));
            if (rc2) return rc2;
        }
    }
    int one = 1;
    PD_CUDA(cudaMemcpy(c->counts + W_REQUEST, &one, sizeof(int), cudaMemcpyHostToDevice));
    c->have_build = false;
    return PD_OK;
}

int pd_cluster_set_pair_shape(pd_cluster *c, int nsplit, int warps) {
    PD_CHECK(c, PD_EINVAL, "pd_cluster_set_pair_shape: null handle");
    PD_CHECK(nsplit >= 1 && nsplit <= 64, PD_EINVAL, "pd_cluster_set_pair_shape: parts per super-cluster 1..64");
    PD_CHECK(warps == 1 || warps == 2 || warps == 4, PD_EINVAL, "pd_cluster_set_pair_shape: warps 1, 2 or 4");
    if (c->nsplit != nsplit || c->pair_warps != warps) {
        c->nsplit = nsplit;
        c->pair_warps = warps;
        c->shape_epoch += 1;
    }
    return PD_OK;
}

int pd_cluster_pair_shape(pd_cluster *c, int *nsplit, int *warps) {
    PD_CHECK(c && nsplit && warps, PD_EINVAL, "pd_cluster_pair_shape: null argument");
    *nsplit = c->nsplit;
    *warps = c->pair_warps;
    return PD_OK;
}

int pd_cluster_grow(pd_cluster *c) {
    PD_CHECK(c, PD_EINVAL, "pd_cluster_grow: null handle");
    int h[W_LEN];
    int rc = cluster_read_counts(c, h, 0);
    if (rc) return rc;
    if (h[W_ERR] == 0) return PD_OK;
    PD_CHECK(h[W_ERR] != PD_ENONFINITE, PD_ENONFINITE, "Cluster-pair list: non-finite coordinates");
    const double growth = c->grown ? 1.25 : 1.5;
    long long need = (long long)std::ceil(growth * h[W_REQ]) + 1024;
    PD_CHECK(need < (1LL << 31), PD_ENOMEM, "outer list would need %lld entries", need);
    if ((rc = alloc_entries(c, (int)need))) return rc;
    c->grown = true;
    int zero2[2] = {0, 0}, one = 1;
    PD_CUDA(cudaMemcpy(c->counts + W_ERR, zero2, 2 * sizeof(int), cudaMemcpyHostToDevice));
    PD_CUDA(cudaMemcpy(c->counts + W_REQUEST, &one, sizeof(int), cudaMemcpyHostToDevice));
    c->have_build = false;
    return PD_OK;
}

int pd_cluster_request_build(pd_cluster *c, pd_stream_t s) {
    PD_CHECK(c, PD_EINVAL, "pd_cluster_request_build: null handle");
    k_set_word<<<1, 1, 0, (cudaStream_t)s>>>(c->counts, W_REQUEST, 1);
    PD_LAUNCHED();
    return PD_OK;
}

int pd_cluster_decide(pd_cluster *c, const float *x, const float *y, const float *z, int fixed, pd_stream_t s) {
    PD_CHECK(c && x && y && z, PD_EINVAL, "pd_cluster_decide: null argument");
    return cluster_decide_launch(c, x, y, z, fixed, (cudaStream_t)s);
}

int pd_cluster_build(pd_cluster *c, const float *x, const float *y, const float *z, const float *q,
                     const int *type, int conditional, pd_stream_t s) {
    PD_CHECK(c && x && y && z, PD_EINVAL, "pd_cluster_build: null argument");
    cudaStream_t st = (cudaStream_t)s;
    int rc = cluster_build_launch(c, x, y, z, q, type, conditional, st);
    if (rc) return rc;
    if (!conditional) {
        // an unconditional build is followed by a pruning pass (prune decision forced)
        k_set_word<<<1, 1, 0, st>>>(c->counts, W_PRUNE, 1);
        PD_LAUNCHED();
    }
    rc = cluster_prune_launch(c, 1, st);
    if (rc) return rc;
    c->have_build = true;
    return PD_OK;
}

int pd_cluster_pack(pd_cluster *c, const float *x, const float *y, const float *z, const float *q, const int *type,
                    pd_stream_t s) {
    PD_CHECK(c && x && y && z, PD_EINVAL, "pd_cluster_pack: null argument");
    k_pack<<<(c->nslot + 255) / 256, 256, 0, (cudaStream_t)s>>>(c->perm, c->nslot, x, y, z, q, type, c->L[0], c->L[1],
                                                                  c->L[2], c->xq, c->ts);
    PD_LAUNCHED();
    return PD_OK;
}

int pd_cluster_prune(pd_cluster *c, const float *x, const float *y, const float *z, int conditional, pd_stream_t s) {
    PD_CHECK(c, PD_EINVAL, "pd_cluster_prune: null handle");
    (void)x;
    (void)y;
    (void)z;
    cudaStream_t st = (cudaStream_t)s;
    if (!conditional) {
        k_set_word<<<1, 1, 0, st>>>(c->counts, W_PRUNE, 1);
        PD_LAUNCHED();
    }
    return cluster_prune_launch(c, 1, st);
}

int pd_cluster_status(pd_cluster *c, pd_cluster_stats *out, pd_stream_t s) {
    PD_CHECK(c && out, PD_EINVAL, "pd_cluster_status: null argument");
    int h[W_LEN];
    int rc = cluster_read_counts(c, h, (cudaStream_t)s);
    if (rc) return rc;
    memset(out, 0, sizeof *out);
    out->superclusters = h[W_NS];
    out->outer_entries = h[W_NE];
    out->error = h[W_ERR];
    out->required = h[W_REQ];
    out->capacity = c->necap;
    out->builds = h[W_NBUILD];
    out->prunes = h[W_NPRUNE];
    out->nsmax = c->nsmax;
    out->nslot = c->nslot;
    out->last_build = h[W_BUILD];
    out->last_prune = h[W_PRUNE];
    if (h[W_NS] > 0 && h[W_ERR] == 0) {
        std::vector<int> nw(h[W_NS]), scio(h[W_NS] + 1);
        PD_CUDA(cudaMemcpy(nw.data(), c->nw, sizeof(int) * h[W_NS], cudaMemcpyDeviceToHost));
        PD_CUDA(cudaMemcpy(scio.data(), c->scio, sizeof(int) * (h[W_NS] + 1), cudaMemcpyDeviceToHost));
        long long tot = 0, bits = 0;
        std::vector<uint2> ent;
        for (int S = 0; S < h[W_NS]; ++S) {
            tot += nw[S];
            if (nw[S] > 0) {
                ent.resize(nw[S]);
                PD_CUDA(cudaMemcpy(ent.data(), c->cjw + scio[S], sizeof(uint2) * nw[S], cudaMemcpyDeviceToHost));
                for (auto &e : ent) bits += __builtin_popcount(e.y & 0xffffu);
            }
        }
        out->working_entries = (int)tot;
        out->tile_bits = bits;
        out->mask_entries = h[W_NX];
        out->outside_pairs = h[W_NP];
    }
    return PD_OK;
}

const int *pd_cluster_order(pd_cluster *c) { return c ? c->order : nullptr; }

int pd_cluster_buffers(pd_cluster *c, const int **perm, const float **xq, const int **scio, const uint32_t **cjo,
                       const uint32_t **cjw, const int **nw) {
    PD_CHECK(c, PD_EINVAL, "pd_cluster_buffers: null handle");
    if (perm) *perm = c->perm;
    if (xq) *xq = (const float *)c->xq;
    if (scio) *scio = c->scio;
    if (cjo) *cjo = c->cjo;
    if (cjw) *cjw = (const uint32_t *)c->cjw;
    if (nw) *nw = c->nw;
    return PD_OK;
}

}  // extern "C"
