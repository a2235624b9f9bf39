// PME / P3M / ESP mesh engine of libpdb200: host setup, influence functions,
// solve and transforms.
//
// Semantics follow src/electrostatics of ParticleDynamics.jl: B-spline and
// prolate windows (Windows.jl:18-308), Gaussian and prolate splits
// (Splits.jl:21-240), influence functions and virial coefficients in FP64
// (Influence.jl:24-227), the solve with the FP64 energy/virial reduction
// (MeshKernels.jl:34-81), the ik field (MeshKernels.jl:84-102) and the AD / ik
// gathers (MeshKernels.jl:105-147, 281-333); cuFFT does the transforms
// (Solver.jl:34-65, 305-347).  The spread and gather kernels are in
// mesh_kernels.cuh.  The charge grid is kept zero between transforms: the solve
// clears it after the forward transform has consumed it, and the inverse
// transform writes the potential into a second grid.
#include <cufft.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "internal.hpp"
#include "mesh_kernels.cuh"

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

// Long-range transform of the split: Gaussian (alpha) or prolate (quadrature of c_hat on device).
struct Spectral {
    double alpha;
    double rc;
    int nq;
    const double *xq, *wchi;   // prolate: nodes on [0, 1] and weights times chi; null for Gaussian
};

// spectral_g(::GaussianSpectral, k) and spectral_g(::ProlateSpectral, k) (Splits.jl:202-225): g(k)
// and g'(k)/k, with g = 4 pi exp(-k^2 / 4 alpha^2) / k^2 or g = 4 pi c_hat(k r_c) / k^2,
// c_hat(u) = sum_q wchi_q cos(u x_q).
__device__ __forceinline__ void spectral_g(const Spectral &sp, double k, double &g, double &gpk) {
    const double k2 = k * k;
    if (!sp.xq) {
        g = 4.0 * M_PI * exp(-k2 / (4.0 * sp.alpha * sp.alpha)) / k2;
        gpk = g * (-2.0 / k2 - 1.0 / (2.0 * sp.alpha * sp.alpha));
        return;
    }
    const double u = k * sp.rc;
    double c = 0.0, dc = 0.0;
    for (int q = 0; q < sp.nq; ++q) {
        const double x = sp.xq[q], w = sp.wchi[q];
        double sn, cs;
        sincos(u * x, &sn, &cs);
        c += w * cs;
        dc -= w * x * sn;
    }
    g = 4.0 * M_PI * c / k2;
    const double gp = 4.0 * M_PI * (sp.rc * dc / k2 - 2.0 * c / (k2 * k));
    gpk = gp / k;
}

// _influence_ewald_kernel! (Influence.jl:35-67): SPME and ESP with the plain deconvolution
__global__ void k_influence_spme(float *__restrict__ G, float *__restrict__ Vc, const double *__restrict__ D1,
                                 const double *__restrict__ D2, const double *__restrict__ D3, int K1, int K2, int K3,
                                 double L1, double L2, double L3, double C, Spectral sp) {
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
    spectral_g(sp, k, g, gpk);
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

// _influence_alias_kernel! (Influence.jl:77-181): optimal influence for AD or ik (P3M, ESP).
__global__ void k_influence_alias(float *__restrict__ G, float *__restrict__ Vc, const double *__restrict__ U1,
                                  const double *__restrict__ U2, const double *__restrict__ U3, int K1, int K2, int K3,
                                  double L1, double L2, double L3, double C, Spectral sp, int nmax, int ik) {
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
                spectral_g(sp, sqrt(qq), g, gpk);
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

static bool plain_deconvolution(const pd_mesh *m) {
    return m->p.kind == PD_MESH_SPME || m->p.kind == PD_MESH_ESP_DECONV;
}

static int compute_influence(pd_mesh *m) {
    const int K1 = m->K1, K2 = m->K2, K3 = m->K3, P = m->p.order;
    const int threads = 128, blocks = (m->nmodes + threads - 1) / threads;
    if (m->prolate) {   // the caller's window tables, the split's quadrature
        const Spectral sp{0.0, m->split_rc, m->nquad, m->xq, m->wchi};
        if (plain_deconvolution(m))
            k_influence_spme<<<blocks, threads>>>(m->G, m->Vc, m->wtab[0], m->wtab[1], m->wtab[2], K1, K2, K3,
                                                  m->box[0], m->box[1], m->box[2], m->p.C, sp);
        else
            k_influence_alias<<<blocks, threads>>>(m->G, m->Vc, m->wtab[0], m->wtab[1], m->wtab[2], K1, K2, K3,
                                                   m->box[0], m->box[1], m->box[2], m->p.C, sp, m->p.alias_order, 0);
        count_launch();
        cudaError_t e = cudaGetLastError();
        cudaError_t e2 = cudaDeviceSynchronize();
        PD_CHECK(e == cudaSuccess && e2 == cudaSuccess, PD_ECUDA, "influence kernel failed: %s",
                 cudaGetErrorString(e != cudaSuccess ? e : e2));
        return PD_OK;
    }
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
    const Spectral sp{m->p.alpha, 0.0, 0, nullptr, nullptr};
    if (m->p.kind == PD_MESH_SPME) {
        k_influence_spme<<<blocks, threads>>>(m->G, m->Vc, d1, d2, d3, K1, K2, K3, m->box[0], m->box[1], m->box[2],
                                              m->p.C, sp);
    } else {
        k_influence_alias<<<blocks, threads>>>(m->G, m->Vc, d1, d2, d3, K1, K2, K3, m->box[0], m->box[1], m->box[2],
                                               m->p.C, sp, m->p.alias_order, m->p.kind == PD_MESH_P3M_IK);
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
    // background_coefficient (Splits.jl:85-86): pi / (2 alpha^2) or pi r_c^2 m_2
    const double bgcoef = m->prolate ? m->bg_coef : M_PI / (2.0 * m->p.alpha * m->p.alpha);
    m->bg = m->p.background ? (float)(-m->p.C * bgcoef * m->p.qtotal / V) : 0.f;
    m->ubg = m->p.background ? -m->p.C * bgcoef * m->p.qtotal * m->p.qtotal / V : 0.0;
}

static WindowPoly window_poly(const pd_mesh *m) { return WindowPoly{m->wpoly, m->wdeg}; }

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

int mesh_transform_packed(pd_mesh *m, const float4 *xq, int nchunks, const int *ns_dev, int energy, cudaStream_t s,
                          cudaEvent_t ev_spread, cudaEvent_t ev_r2c) {
    const float Lx = (float)m->box[0], Ly = (float)m->box[1], Lz = (float)m->box[2];
    PD_CHECK(m->p.order >= MESH_ORDER_MIN && m->p.order <= MESH_ORDER_MAX, PD_EINVAL, "unsupported order %d",
             m->p.order);
    if (m->prolate)
        launch_spread_t<WIN_PROLATE>(m->p.order, xq, nchunks, ns_dev, m->gridA, m->K1, m->K2, m->K3, Lx, Ly, Lz,
                                     window_poly(m), s);
    else
        launch_spread_t<WIN_BSPLINE>(m->p.order, xq, nchunks, ns_dev, m->gridA, m->K1, m->K2, m->K3, Lx, Ly, Lz,
                                     window_poly(m), s);
    PD_LAUNCHED();
    if (ev_spread) PD_CUDA(cudaEventRecord(ev_spread, s));
    PD_CUFFT(cufftSetStream(m->fwd, s));
    PD_CUFFT(cufftExecR2C(m->fwd, m->gridA, m->spec));
    if (ev_r2c) PD_CUDA(cudaEventRecord(ev_r2c, s));
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

int mesh_store_virial(pd_mesh *m, float *vglobal6, cudaStream_t s) {
    if (!vglobal6) return PD_OK;
    k_store_virial<<<1, 32, 0, s>>>(vglobal6, m->acc, m->ubg);
    PD_LAUNCHED();
    return PD_OK;
}

// MODE 0 (add) or 1 (set) through the SoA entry point, 2 the join of the step.
template <int MODE, bool ENERGY>
static void launch_gather(pd_mesh *m, const float4 *xq, int nchunks, const int *ns_dev, const GatherOut &o,
                          cudaStream_t s) {
    const float Lx = (float)m->box[0], Ly = (float)m->box[1], Lz = (float)m->box[2];
    const int K1 = m->K1, K2 = m->K2, K3 = m->K3, P = m->p.order;
    GatherOut oo = o;
    oo.wp = window_poly(m);
    if (m->prolate) {
        const GatherGrids g = {{m->gridB, nullptr, nullptr, nullptr}};
        launch_gather_t<WIN_PROLATE, false, MODE>(P, ENERGY, xq, nchunks, ns_dev, g, K1, K2, K3, Lx, Ly, Lz, oo, s);
    } else if (m->p.kind == PD_MESH_P3M_IK) {
        const GatherGrids g = {{m->field[0], m->field[1], m->field[2], m->gridB}};
        launch_gather_t<WIN_BSPLINE, true, MODE>(P, ENERGY, xq, nchunks, ns_dev, g, K1, K2, K3, Lx, Ly, Lz, oo, s);
    } else {
        const GatherGrids g = {{m->gridB, nullptr, nullptr, nullptr}};
        launch_gather_t<WIN_BSPLINE, false, MODE>(P, ENERGY, xq, nchunks, ns_dev, g, K1, K2, K3, Lx, Ly, Lz, oo, s);
    }
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
    dfree(m->xq);
    dfree(m->wchi);
    dfree(m->wpoly);
    for (int d = 0; d < 3; ++d) dfree(m->wtab[d]);
    if (m->plans) {
        cufftDestroy(m->fwd);
        cufftDestroy(m->bwd);
        m->plans = false;
    }
    if (m->work) cudaFree(m->work);
    m->work = nullptr;
}

}  // namespace pdb

namespace {

// Device copy of the prolate split and window (pd_prolate) into m.
int copy_prolate(pd_mesh *m, const pd_prolate *w) {
    const int P = m->p.order, H = (P + 1) / 2;
    m->prolate = true;
    m->split_rc = w->cutoff;
    m->bg_coef = w->background_coefficient;
    m->nquad = w->nquad;
    m->wdeg = w->deg;
    std::vector<float> poly((size_t)(w->deg + 1) * H);
    for (int k = 0; k <= w->deg; ++k)
        for (int h = 0; h < H; ++h) poly[(size_t)k * H + h] = (float)w->poly[k][h];
    int rc;
    if ((rc = dalloc(&m->xq, (size_t)w->nquad)) || (rc = dalloc(&m->wchi, (size_t)w->nquad)) ||
        (rc = dalloc(&m->wpoly, poly.size())))
        return rc;
    PD_CUDA(cudaMemcpy(m->xq, w->xq, sizeof(double) * w->nquad, cudaMemcpyHostToDevice));
    PD_CUDA(cudaMemcpy(m->wchi, w->wchi, sizeof(double) * w->nquad, cudaMemcpyHostToDevice));
    PD_CUDA(cudaMemcpy(m->wpoly, poly.data(), sizeof(float) * poly.size(), cudaMemcpyHostToDevice));
    const int K[3] = {m->K1, m->K2, m->K3};
    const int per = m->p.kind == PD_MESH_ESP ? 2 * m->p.alias_order + 1 : 1;
    for (int d = 0; d < 3; ++d) {
        const size_t len = (size_t)K[d] * per;
        for (size_t i = 0; i < len; ++i)
            PD_CHECK(std::isfinite(w->table[d][i]), PD_EINVAL, "prolate window table %d has a non-finite entry", d);
        if ((rc = dalloc(&m->wtab[d], len))) return rc;
        PD_CUDA(cudaMemcpy(m->wtab[d], w->table[d], sizeof(double) * len, cudaMemcpyHostToDevice));
    }
    return PD_OK;
}

int mesh_create(pd_mesh **out, const pd_mesh_params *p, const pd_prolate *w, const double box[3]) {
    const bool esp = w != nullptr;
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
    if ((esp && (rc = copy_prolate(m, w))) || (rc = pd_mesh_set_box(m, box))) {
        free_mesh(m);
        delete m;
        return rc;
    }
    *out = m;
    return PD_OK;
}

}  // namespace

extern "C" {


int pd_mesh_create(pd_mesh **out, const pd_mesh_params *p, const double box[3]) {
    PD_CHECK(out && p && box, PD_EINVAL, "pd_mesh_create: null argument");
    *out = nullptr;
    PD_CHECK(p->kind >= PD_MESH_SPME && p->kind <= PD_MESH_P3M_IK, PD_EINVAL,
             "Unknown influence kind %d (ESP meshes come from pd_mesh_create_prolate).", p->kind);
    PD_CHECK(p->order >= 3 && p->order <= 12, PD_EINVAL,
             "B-spline assignment order must be between 3 and 12; got %d.", p->order);
    PD_CHECK(p->alias_order >= 0 && p->alias_order <= 6, PD_EINVAL, "alias_order must be between 0 and 6.");
    PD_CHECK(p->C > 0 && std::isfinite(p->C), PD_EINVAL, "coulomb constant must be finite and positive");
    PD_CHECK(p->alpha > 0 && std::isfinite(p->alpha), PD_EINVAL, "Ewald alpha must be finite and positive.");
    return mesh_create(out, p, nullptr, box);
}

int pd_mesh_create_prolate(pd_mesh **out, const pd_mesh_params *p, const pd_prolate *w, const double box[3]) {
    PD_CHECK(out && p && w && box, PD_EINVAL, "pd_mesh_create_prolate: null argument");
    *out = nullptr;
    PD_CHECK(p->kind == PD_MESH_ESP || p->kind == PD_MESH_ESP_DECONV, PD_EINVAL,
             "pd_mesh_create_prolate needs an ESP influence kind; got %d.", p->kind);
    PD_CHECK(p->order >= 3 && p->order <= 12, PD_EINVAL,
             "Prolate window width must be between 3 and 12 grid points in this build; got %d.", p->order);
    PD_CHECK(p->alias_order >= 0 && p->alias_order <= 6, PD_EINVAL, "alias_order must be between 0 and 6.");
    PD_CHECK(p->C > 0 && std::isfinite(p->C), PD_EINVAL, "coulomb constant must be finite and positive");
    PD_CHECK(std::isfinite(w->cutoff) && w->cutoff > 0, PD_EINVAL, "ESP cutoff must be finite and positive.");
    PD_CHECK(w->nquad >= 1 && w->nquad <= PD_PROLATE_MAX_QUAD, PD_EINVAL, "ESP quadrature needs 1..%d nodes",
             PD_PROLATE_MAX_QUAD);
    PD_CHECK(w->deg >= 1 && w->deg <= PD_PROLATE_MAX_DEG, PD_EINVAL, "node polynomial degree must be 1..%d",
             PD_PROLATE_MAX_DEG);
    PD_CHECK((p->order + 1) / 2 <= PD_PROLATE_MAX_NODES, PD_EINVAL, "too many window nodes");
    PD_CHECK(w->table[0] && w->table[1] && w->table[2], PD_EINVAL, "pd_mesh_create_prolate: window tables missing");
    PD_CHECK(std::isfinite(w->background_coefficient), PD_EINVAL, "background coefficient must be finite");
    return mesh_create(out, p, w, box);
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
    PD_CHECK(table_size == 0 || (m->p.kind != PD_MESH_P3M_IK && !m->prolate), PD_ENOTSUP,
             "self-force removal needs a B-spline window with analytic differentiation (SPME or P3M-AD)");
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
