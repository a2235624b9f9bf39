// Learned coarse-mesh correction of libpdb200: per-particle local charge
// descriptors over neighbour rows, and the force residual of the network.
//
// Model (rotation-equivariant by construction):
//   features  x_i[16 s + k] = sum_{j in species s, r_ij < r_c} q_j g_k(r_ij) f_c(r_ij)
//             g_k(r) = exp(-(r - mu_k)^2 / (2 sigma^2)), mu_k = mu0 + k dmu (k < 16),
//             f_c(r) = (1 - r^2 / r_c^2)^2, two species: type id 1 and every other id
//             (1-based type ids; no type array: one species);
//   scalar    s_i = MLP(x_i)  (32-128-128-1 SiLU, BF16 tensor cores, mlp.cu);
//   residual  F_i = sum_j w_ij (r_i - r_j),  w_ij = s_i q_i q_j b(r_ij),
//             b(r) = f_c(r) sum_m c_m exp(-(r - nu_m)^2 / (2 tau^2)),  nu_m = nu0 + m dnu,
//   so F_i = s_i V_i with V_i = sum_j q_i q_j b(r_ij) (r_i - r_j): the network supplies a
//   per-neighbour scalar weight that multiplies the displacement vector.  The radial
//   coefficients c_m are fitted by linear least squares to the training residuals
//   (basis mode below: V_i^(m) per radial term), the network then learns the
//   environment-dependent scale s_i.
//
// Neighbour rows come from a device ELL list (ell.cu) of radius r_c + skin, rebuilt by its
// own displacement decision; eight lanes per particle walk its row, keep partial features and
// V_i in registers, reduce them by shuffles and write them once (no atomics).
#include <cuda_bf16.h>

#include <cmath>
#include <cstring>

#include "common.cuh"
#include "internal.hpp"

using namespace pdb;

namespace pdb {

constexpr int DESC_THREADS = 256;
constexpr int DESC_F = 16;   // Gaussians per species
constexpr int DESC_LANES = 8; // lanes per particle

struct DescParams {
    float Lx, Ly, Lz;
    float rc2, inv_rc2;
    float mu0, dmu, inv2s2, cmu;   // cmu = exp(-2 dmu^2 / (2 sigma^2)): ratio step of the feature run
    int nb;
    float nu0, dnu, inv2t2, cnu;   // cnu: ratio step of the radial-term run
    float coef[PD_LEARNED_MAX_RADIAL];
};

// A run of equally spaced Gaussians g_k = exp(-a (r - c0 - k dc)^2) by products: g_{k+1} = g_k rho_k
// with rho_k = exp(a dc (2 (r - c_k) - dc)) and rho_{k+1} = rho_k exp(-2 a dc^2) (two exponentials per
// run).  Terms that underflow at the start of a run are below exp(-87) of their peak.
struct GaussRun {
    float g, rho, c;
    __device__ __forceinline__ GaussRun(float r, float c0, float dc, float a, float step) {
        const float d = r - c0;
        g = __expf(-a * d * d);
        rho = __expf(a * dc * (2.f * d - dc));
        c = step;
    }
    __device__ __forceinline__ float next() {
        const float v = g;
        g *= rho;
        rho *= c;
        return v;
    }
};

__device__ __forceinline__ float mic_d(float d, float L) {
    const float h = 0.5f * L;
    d -= (d > h) ? L : 0.f;
    d += (d < -h) ? L : 0.f;
    return d;
}

// Packed neighbour record (x, y, z, q) with the species in the lowest mantissa bit of q (a change
// of at most one ulp of the charge), so that a row entry costs one 16-byte gather.
__global__ void k_desc_pack(const float *__restrict__ x, const float *__restrict__ y, const float *__restrict__ z,
                            const float *__restrict__ q, const int *__restrict__ type, int n,
                            float4 *__restrict__ xq) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int s1 = (type != nullptr && type[i] > 1) ? 1 : 0;
    xq[i] = make_float4(x[i], y[i], z[i], __int_as_float((__float_as_int(q[i]) & ~1) | s1));
}

// Sum over the G consecutive lanes of a particle's group (butterfly: every lane gets the total).
template <int G>
__device__ __forceinline__ float group_sum(float v) {
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Features, V_i (or with BASIS the radial-term vectors V_i^(m), m < nb, at Vb[m n + i]).  G lanes per
// particle stride its row (entries g, g + G, ...) and reduce their partial sums by shuffles; lane g < 4
// of the group stores the g-th 16-byte chunk of the particle's BF16 features.
template <bool BASIS, int G>
__global__ void __launch_bounds__(DESC_THREADS, 4) k_descriptors(const float4 *__restrict__ xq, int n,
                                                              const int *__restrict__ rows,
                                                              const int *__restrict__ counts, int cap, DescParams p,
                                                              __nv_bfloat16 *__restrict__ X, float4 *__restrict__ V,
                                                              float4 *__restrict__ Vb) {
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = tid / G, g = tid % G;
    const bool live = i < n;   // whole groups are live or not (G divides the warp)
    if (__all_sync(0xffffffffu, !live)) return;
    const int ii = live ? i : 0;
    const float4 pi = xq[ii];
    const float xi = pi.x, yi = pi.y, zi = pi.z, qi = pi.w;
    float a0[DESC_F], a1[DESC_F];
#pragma unroll
    for (int k = 0; k < DESC_F; ++k) a0[k] = a1[k] = 0.f;
    float vx = 0.f, vy = 0.f, vz = 0.f;
    float bx[PD_LEARNED_MAX_RADIAL], by[PD_LEARNED_MAX_RADIAL], bz[PD_LEARNED_MAX_RADIAL];
#pragma unroll
    for (int m = 0; m < PD_LEARNED_MAX_RADIAL; ++m) bx[m] = by[m] = bz[m] = 0.f;
    const int cnt = live ? min(counts[ii], cap) : 0;
    // one entry ahead: the row index and the neighbour record of the next entry are in flight
    // while this one is evaluated
    int jn = g < cnt ? __ldg(rows + (size_t)g * n + ii) : ii;
    float4 pn = __ldg(xq + jn);
    for (int t = g; t < cnt; t += G) {
        const float4 pj = pn;
        if (t + G < cnt) {
            jn = __ldg(rows + (size_t)(t + G) * n + ii);
            pn = __ldg(xq + jn);
        }
        const float dx = mic_d(xi - pj.x, p.Lx);
        const float dy = mic_d(yi - pj.y, p.Ly);
        const float dz = mic_d(zi - pj.z, p.Lz);
        const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
        if (!(r2 < p.rc2) || r2 == 0.f) continue;
        const float r = r2 * rsqrtf(r2);
        const float u2 = 1.f - r2 * p.inv_rc2;
        const float fc = u2 * u2;
        const float qj = pj.w;
        const bool s1 = (__float_as_int(pj.w) & 1) != 0;
        const float wq = qj * fc;
        const float w0 = s1 ? 0.f : wq, w1 = s1 ? wq : 0.f;
        {   // two runs of eight feature Gaussians, from centres 0 and 8
            GaussRun lo(r, p.mu0, p.dmu, p.inv2s2, p.cmu);
            GaussRun hi(r, fmaf(8.f, p.dmu, p.mu0), p.dmu, p.inv2s2, p.cmu);
#pragma unroll
            for (int k = 0; k < DESC_F / 2; ++k) {
                const float el = lo.next(), eh = hi.next();
                a0[k] = fmaf(el, w0, a0[k]);
                a1[k] = fmaf(el, w1, a1[k]);
                a0[k + DESC_F / 2] = fmaf(eh, w0, a0[k + DESC_F / 2]);
                a1[k + DESC_F / 2] = fmaf(eh, w1, a1[k + DESC_F / 2]);
            }
        }
        const float qq = qi * qj * fc;
        GaussRun rad(r, p.nu0, p.dnu, p.inv2t2, p.cnu);
        if (BASIS) {
#pragma unroll
            for (int m = 0; m < PD_LEARNED_MAX_RADIAL; ++m) {
                if (m >= p.nb) break;
                const float e = qq * rad.next();
                bx[m] = fmaf(e, dx, bx[m]);
                by[m] = fmaf(e, dy, by[m]);
                bz[m] = fmaf(e, dz, bz[m]);
            }
        } else {
            float b = 0.f;
#pragma unroll
            for (int m = 0; m < PD_LEARNED_MAX_RADIAL; ++m) {
                if (m >= p.nb) break;
                b = fmaf(p.coef[m], rad.next(), b);
            }
            const float e = qq * b;
            vx = fmaf(e, dx, vx);
            vy = fmaf(e, dy, vy);
            vz = fmaf(e, dz, vz);
        }
    }
#pragma unroll
    for (int k = 0; k < DESC_F; ++k) {
        a0[k] = group_sum<G>(a0[k]);
        a1[k] = group_sum<G>(a1[k]);
    }
    if (BASIS) {
#pragma unroll
        for (int m = 0; m < PD_LEARNED_MAX_RADIAL; ++m) {
            if (m >= p.nb) break;   // p.nb is uniform: every lane takes the same shuffles
            bx[m] = group_sum<G>(bx[m]);
            by[m] = group_sum<G>(by[m]);
            bz[m] = group_sum<G>(bz[m]);
        }
    } else {
        vx = group_sum<G>(vx);
        vy = group_sum<G>(vy);
        vz = group_sum<G>(vz);
    }
    if (!live) return;
    if (X && g < 4) {
        __align__(16) __nv_bfloat16 h[8];
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            if (c != g) continue;
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const int f = 8 * c + k;
                h[k] = __float2bfloat16_rn(f < DESC_F ? a0[f] : a1[f - DESC_F]);
            }
        }
        reinterpret_cast<uint4 *>(X + (size_t)i * 32)[g] = *reinterpret_cast<const uint4 *>(h);
    }
    if (g != 0) return;
    if (BASIS) {
#pragma unroll
        for (int m = 0; m < PD_LEARNED_MAX_RADIAL; ++m)
            if (m < p.nb) Vb[(size_t)m * n + i] = make_float4(bx[m], by[m], bz[m], 0.f);
    } else if (V) {
        V[i] = make_float4(vx, vy, vz, 0.f);
    }
}

}  // namespace pdb

struct pd_learned {
    pd_learned_params p;
    int n = 0;
    double box[3] = {0, 0, 0};
    pd_ell *ell = nullptr;
    __nv_bfloat16 *X = nullptr;   // n x 32
    float4 *V = nullptr;          // n
    float4 *corr = nullptr;       // n: (s V, s)
    float4 *xq = nullptr;         // n: packed (x, y, z, q | species bit)
};

namespace pdb {

static DescParams desc_params(const pd_learned *h) {
    DescParams d;
    memset(&d, 0, sizeof d);
    d.Lx = (float)h->box[0];
    d.Ly = (float)h->box[1];
    d.Lz = (float)h->box[2];
    d.rc2 = h->p.rcut * h->p.rcut;
    d.inv_rc2 = 1.f / d.rc2;
    d.mu0 = h->p.mu0;
    d.dmu = h->p.dmu;
    d.inv2s2 = 0.5f / (h->p.sigma * h->p.sigma);
    d.cmu = (float)exp(-2.0 * (double)d.inv2s2 * (double)d.dmu * (double)d.dmu);
    d.nb = h->p.nb;
    d.nu0 = h->p.nu0;
    d.dnu = h->p.dnu;
    d.inv2t2 = 0.5f / (h->p.tau * h->p.tau);
    d.cnu = (float)exp(-2.0 * (double)d.inv2t2 * (double)d.dnu * (double)d.dnu);
    for (int m = 0; m < PD_LEARNED_MAX_RADIAL; ++m) d.coef[m] = h->p.coef[m];
    return d;
}

static int descriptors_launch(pd_learned *h, const float *x, const float *y, const float *z, const float *q,
                              const int *type, __nv_bfloat16 *X, float4 *V, float4 *Vb, cudaStream_t s) {
    int rc;
    if ((rc = pd_ell_update(h->ell, x, y, z, (pd_stream_t)s))) return rc;
    int *rows = nullptr, *counts = nullptr;
    if ((rc = pd_ell_rows(h->ell, &rows, &counts))) return rc;
    const int cap = ell_capacity(h->ell);
    const DescParams d = desc_params(h);
    k_desc_pack<<<(h->n + 255) / 256, 256, 0, s>>>(x, y, z, q, type, h->n, h->xq);
    PD_LAUNCHED();
    constexpr int G = DESC_LANES;
    const int blocks = (int)(((long long)h->n * G + DESC_THREADS - 1) / DESC_THREADS);
    if (Vb)
        k_descriptors<true, G><<<blocks, DESC_THREADS, 0, s>>>(h->xq, h->n, rows, counts, cap, d, X, V, Vb);
    else
        k_descriptors<false, G><<<blocks, DESC_THREADS, 0, s>>>(h->xq, h->n, rows, counts, cap, d, X, V, Vb);
    PD_LAUNCHED();
    return PD_OK;
}

// Descriptors and network residual into h->corr (step engine and C entry point).
int learned_correction_launch(pd_learned *h, const pd_mlp *net, const float *x, const float *y, const float *z,
                              const float *q, const int *type, float4 *corr, cudaStream_t s) {
    int rc;
    if ((rc = descriptors_launch(h, x, y, z, q, type, h->X, h->V, nullptr, s))) return rc;
    if (!net) return PD_OK;   // radial term only: the correction is V itself (s = 1)
    return mlp_forward_launch(net, h->X, h->n, nullptr, h->V, corr ? corr : h->corr, s);
}

const float4 *learned_corr(const pd_learned *h) { return h->corr; }
const float4 *learned_radial(const pd_learned *h) { return h->V; }

static void learned_free(pd_learned *h) {
    if (h->ell) pd_ell_destroy(h->ell);
    h->ell = nullptr;
    dfree(h->X);
    dfree(h->V);
    dfree(h->corr);
    dfree(h->xq);
}

}  // namespace pdb

extern "C" {

int pd_learned_create(pd_learned **out, const pd_learned_params *p, int n, const double box[3]) {
    PD_CHECK(out && p && box, PD_EINVAL, "pd_learned_create: null argument");
    *out = nullptr;
    PD_CHECK(n > 0, PD_EINVAL, "pd_learned_create: particle count must be positive");
    PD_CHECK(std::isfinite(p->rcut) && p->rcut > 0, PD_EINVAL, "pd_learned_create: cutoff must be positive");
    PD_CHECK(p->nb >= 1 && p->nb <= PD_LEARNED_MAX_RADIAL, PD_EINVAL, "pd_learned_create: 1..%d radial terms",
             PD_LEARNED_MAX_RADIAL);
    PD_CHECK(p->sigma > 0 && p->tau > 0, PD_EINVAL, "pd_learned_create: Gaussian widths must be positive");
    PD_CHECK(p->cap > 0, PD_EINVAL, "pd_learned_create: row capacity must be positive");
    pd_learned *h = new pd_learned();
    h->p = *p;
    h->n = n;
    for (int d = 0; d < 3; ++d) h->box[d] = box[d];
    pd_ell_params ep;
    memset(&ep, 0, sizeof ep);
    ep.dim = 3;
    ep.n = n;
    ep.cutoff = p->rcut;
    ep.skin = p->skin;
    ep.cap = p->cap;
    ep.interval = 100;
    ep.model = PD_PAIR_LJ;   // rows only: the pair model is never evaluated
    ep.eps = 1.f;
    ep.sigma = 1.f;
    ep.rc2 = p->rcut * p->rcut;
    ep.lanes = 1;
    int rc;
    if ((rc = pd_ell_create(&h->ell, &ep, box)) || (rc = dalloc(&h->X, (size_t)n * 32)) ||
        (rc = dalloc(&h->V, (size_t)n)) || (rc = dalloc(&h->corr, (size_t)n)) || (rc = dalloc(&h->xq, (size_t)n))) {
        learned_free(h);
        delete h;
        return rc;
    }
    if (cudaMemset(h->corr, 0, sizeof(float4) * (size_t)n) != cudaSuccess ||
        cudaMemset(h->V, 0, sizeof(float4) * (size_t)n) != cudaSuccess) {
        learned_free(h);
        delete h;
        set_error("pd_learned_create: device initialisation failed");
        return PD_ECUDA;
    }
    *out = h;
    return PD_OK;
}

int pd_learned_destroy(pd_learned *h) {
    if (!h) return PD_OK;
    learned_free(h);
    delete h;
    return PD_OK;
}

int pd_learned_set_radial(pd_learned *h, const float *coef, int nb) {
    PD_CHECK(h && coef, PD_EINVAL, "pd_learned_set_radial: null argument");
    PD_CHECK(nb == h->p.nb, PD_EINVAL, "pd_learned_set_radial: %d coefficients, the model has %d", nb, h->p.nb);
    for (int m = 0; m < nb; ++m) h->p.coef[m] = coef[m];
    return PD_OK;
}

int pd_learned_descriptors(pd_learned *h, const float *x, const float *y, const float *z, const float *q,
                           const int *type, void *X, float *V4, float *Vb4, pd_stream_t s) {
    PD_CHECK(h && x && y && z && q, PD_EINVAL, "pd_learned_descriptors: null argument");
    return descriptors_launch(h, x, y, z, q, type, X ? static_cast<__nv_bfloat16 *>(X) : h->X,
                              V4 ? reinterpret_cast<float4 *>(V4) : h->V, reinterpret_cast<float4 *>(Vb4),
                              (cudaStream_t)s);
}

int pd_learned_correction(pd_learned *h, pd_mlp *net, const float *x, const float *y, const float *z, const float *q,
                          const int *type, float *corr4, pd_stream_t s) {
    PD_CHECK(h && net && x && y && z && q, PD_EINVAL, "pd_learned_correction: null argument");
    return learned_correction_launch(h, net, x, y, z, q, type, reinterpret_cast<float4 *>(corr4), (cudaStream_t)s);
}

int pd_learned_buffers(pd_learned *h, void **X, float **V4, float **corr4) {
    PD_CHECK(h, PD_EINVAL, "pd_learned_buffers: null handle");
    if (X) *X = h->X;
    if (V4) *V4 = reinterpret_cast<float *>(h->V);
    if (corr4) *corr4 = reinterpret_cast<float *>(h->corr);
    return PD_OK;
}

int pd_learned_status(pd_learned *h, pd_ell_stats *out) {
    PD_CHECK(h && out, PD_EINVAL, "pd_learned_status: null argument");
    return pd_ell_status(h->ell, out);
}

int pd_learned_resize(pd_learned *h, int cap) {
    PD_CHECK(h, PD_EINVAL, "pd_learned_resize: null handle");
    const int rc = pd_ell_resize(h->ell, cap);
    if (rc == PD_OK) h->p.cap = cap;
    return rc;
}

}  // extern "C"
