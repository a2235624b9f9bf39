// Learned coarse-mesh correction of libpdb200: per-particle local charge
// descriptors over neighbour rows, and the force residual of the network.
//
// Model (rotation-equivariant by construction):
//   features  x_i[16 s + k] = sum_{j in species s, r_ij < r_c} q_j g_k(r_ij) f_c(r_ij)
//             g_k(r) = exp(-(r - mu_k)^2 / (2 sigma^2)), mu_k = mu0 + k dmu (k < 16),
//             f_c(r) = (cos(pi r / r_c) + 1) / 2, two species: type id 1 and every other id
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
// own displacement decision; one thread per particle walks its row, keeps the 32 features
// and V_i in registers and writes them once (no atomics).
#include <cuda_bf16.h>

#include <cmath>
#include <cstring>

#include "common.cuh"
#include "internal.hpp"

using namespace pdb;

namespace pdb {

constexpr int DESC_THREADS = 256;
constexpr int DESC_F = 16;   // Gaussians per species

struct DescParams {
    float Lx, Ly, Lz;
    float rc2, inv_rc;
    float mu0, dmu, inv2s2;
    int nb;
    float nu0, dnu, inv2t2;
    float coef[PD_LEARNED_MAX_RADIAL];
};

__device__ __forceinline__ float mic_d(float d, float L) {
    const float h = 0.5f * L;
    d -= (d > h) ? L : 0.f;
    d += (d < -h) ? L : 0.f;
    return d;
}

// Features, V_i (or with BASIS the radial-term vectors V_i^(m), m < nb, at Vb[m n + i]).
template <bool BASIS>
__global__ void __launch_bounds__(DESC_THREADS) k_descriptors(const float *__restrict__ x, const float *__restrict__ y,
                                                              const float *__restrict__ z, const float *__restrict__ q,
                                                              const int *__restrict__ type, int n,
                                                              const int *__restrict__ rows,
                                                              const int *__restrict__ counts, int cap, DescParams p,
                                                              __nv_bfloat16 *__restrict__ X, float4 *__restrict__ V,
                                                              float4 *__restrict__ Vb) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float xi = x[i], yi = y[i], zi = z[i], qi = q[i];
    float a0[DESC_F], a1[DESC_F];
#pragma unroll
    for (int k = 0; k < DESC_F; ++k) a0[k] = a1[k] = 0.f;
    float vx = 0.f, vy = 0.f, vz = 0.f;
    float bx[PD_LEARNED_MAX_RADIAL], by[PD_LEARNED_MAX_RADIAL], bz[PD_LEARNED_MAX_RADIAL];
#pragma unroll
    for (int m = 0; m < PD_LEARNED_MAX_RADIAL; ++m) bx[m] = by[m] = bz[m] = 0.f;
    const int cnt = min(counts[i], cap);
    for (int t = 0; t < cnt; ++t) {
        const int j = __ldg(rows + (size_t)t * n + i);
        const float dx = mic_d(xi - __ldg(x + j), p.Lx);
        const float dy = mic_d(yi - __ldg(y + j), p.Ly);
        const float dz = mic_d(zi - __ldg(z + j), p.Lz);
        const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
        if (!(r2 < p.rc2) || r2 == 0.f) continue;
        const float r = sqrtf(r2);
        const float fc = 0.5f * (cospif(r * p.inv_rc) + 1.f);
        const float qj = __ldg(q + j);
        const bool s1 = type != nullptr && __ldg(type + j) > 1;
        const float wq = qj * fc;
        const float w0 = s1 ? 0.f : wq, w1 = s1 ? wq : 0.f;
#pragma unroll
        for (int k = 0; k < DESC_F; ++k) {
            const float u = r - fmaf((float)k, p.dmu, p.mu0);
            const float g = __expf(-u * u * p.inv2s2);
            a0[k] = fmaf(g, w0, a0[k]);
            a1[k] = fmaf(g, w1, a1[k]);
        }
        const float qq = qi * qj * fc;
        if (BASIS) {
#pragma unroll
            for (int m = 0; m < PD_LEARNED_MAX_RADIAL; ++m) {
                if (m >= p.nb) break;
                const float u = r - fmaf((float)m, p.dnu, p.nu0);
                const float e = qq * __expf(-u * u * p.inv2t2);
                bx[m] = fmaf(e, dx, bx[m]);
                by[m] = fmaf(e, dy, by[m]);
                bz[m] = fmaf(e, dz, bz[m]);
            }
        } else {
            float b = 0.f;
#pragma unroll
            for (int m = 0; m < PD_LEARNED_MAX_RADIAL; ++m) {
                if (m >= p.nb) break;
                const float u = r - fmaf((float)m, p.dnu, p.nu0);
                b = fmaf(p.coef[m], __expf(-u * u * p.inv2t2), b);
            }
            const float e = qq * b;
            vx = fmaf(e, dx, vx);
            vy = fmaf(e, dy, vy);
            vz = fmaf(e, dz, vz);
        }
    }
    if (X) {
        uint4 *dst = reinterpret_cast<uint4 *>(X + (size_t)i * 32);
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            __align__(16) __nv_bfloat16 h[8];
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const int f = 8 * c + k;
                h[k] = __float2bfloat16_rn(f < DESC_F ? a0[f] : a1[f - DESC_F]);
            }
            dst[c] = *reinterpret_cast<const uint4 *>(h);
        }
    }
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
};

namespace pdb {

static DescParams desc_params(const pd_learned *h) {
    DescParams d;
    memset(&d, 0, sizeof d);
    d.Lx = (float)h->box[0];
    d.Ly = (float)h->box[1];
    d.Lz = (float)h->box[2];
    d.rc2 = h->p.rcut * h->p.rcut;
    d.inv_rc = 1.f / h->p.rcut;
    d.mu0 = h->p.mu0;
    d.dmu = h->p.dmu;
    d.inv2s2 = 0.5f / (h->p.sigma * h->p.sigma);
    d.nb = h->p.nb;
    d.nu0 = h->p.nu0;
    d.dnu = h->p.dnu;
    d.inv2t2 = 0.5f / (h->p.tau * h->p.tau);
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
    const int blocks = (h->n + DESC_THREADS - 1) / DESC_THREADS;
    if (Vb)
        k_descriptors<true><<<blocks, DESC_THREADS, 0, s>>>(x, y, z, q, type, h->n, rows, counts, cap, d, X, V, Vb);
    else
        k_descriptors<false><<<blocks, DESC_THREADS, 0, s>>>(x, y, z, q, type, h->n, rows, counts, cap, d, X, V, Vb);
    PD_LAUNCHED();
    return PD_OK;
}

// Descriptors and network residual into h->corr (step engine and C entry point).
int learned_correction_launch(pd_learned *h, const pd_mlp *net, const float *x, const float *y, const float *z,
                              const float *q, const int *type, float4 *corr, cudaStream_t s) {
    int rc;
    if ((rc = descriptors_launch(h, x, y, z, q, type, h->X, h->V, nullptr, s))) return rc;
    return mlp_forward_launch(net, h->X, h->n, nullptr, h->V, corr ? corr : h->corr, s);
}

const float4 *learned_corr(const pd_learned *h) { return h->corr; }

static void learned_free(pd_learned *h) {
    if (h->ell) pd_ell_destroy(h->ell);
    h->ell = nullptr;
    dfree(h->X);
    dfree(h->V);
    dfree(h->corr);
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
        (rc = dalloc(&h->V, (size_t)n)) || (rc = dalloc(&h->corr, (size_t)n))) {
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
