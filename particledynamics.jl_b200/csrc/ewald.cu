// FP64 Ewald oracle on the GPU: a restatement of ewald_reference
// (test/ewald_reference.jl:50-127) that states the error of the mesh forms on
// full-size systems, where the CPU sum is out of reach.
//
//   real space   sum over minimum images within r_cut = x / alpha (pairs of one tile of
//                256 particles against every particle, FP64 erfc and exp);
//   reciprocal   S(k) = sum_j q_j exp(i k.r_j) over the half space of k vectors with
//                |k| < 2 alpha x (x = sqrt(digits ln 10)); F_i = sum_k 2 (C / V) g(k) q_i
//                (sin(k.r_i) Re S - cos(k.r_i) Im S) k with g(k) = 4 pi exp(-k^2 / 4 alpha^2) / k^2;
//   self         -C alpha / sqrt(pi) sum q^2 (energy only).
// Everything is FP64; the k list is built on the host.  This is test and measurement
// infrastructure: synchronous, allocating, not capture-safe.
#include <cmath>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "internal.hpp"

using namespace pdb;

namespace pdb {

constexpr int EW_T = 256;
constexpr int EW_KSPLIT = 16;

__global__ void __launch_bounds__(EW_T) k_ewald_real(const double4 *__restrict__ rq, int n, double Lx, double Ly,
                                                     double Lz, double alpha, double rcut2, double C,
                                                     double *__restrict__ F, double *__restrict__ E) {
    __shared__ double4 sp[EW_T];
    const int i = blockIdx.x * EW_T + threadIdx.x;
    const double4 pi = i < n ? rq[i] : make_double4(0, 0, 0, 0);
    const double tap = 2.0 * alpha / sqrt(M_PI);
    double fx = 0, fy = 0, fz = 0, e = 0;
    const int per = (n + gridDim.y - 1) / gridDim.y;
    const int j0 = blockIdx.y * per, j1 = min(n, j0 + per);
    for (int base = j0; base < j1; base += EW_T) {
        const int j = base + threadIdx.x;
        sp[threadIdx.x] = j < j1 ? rq[j] : make_double4(0, 0, 0, 0);
        __syncthreads();
        const int m = min(EW_T, j1 - base);
        if (i < n) {
            for (int t = 0; t < m; ++t) {
                if (base + t == i) continue;
                const double4 p = sp[t];
                double dx = pi.x - p.x, dy = pi.y - p.y, dz = pi.z - p.z;
                dx -= Lx * rint(dx / Lx);
                dy -= Ly * rint(dy / Ly);
                dz -= Lz * rint(dz / Lz);
                const double r2 = dx * dx + dy * dy + dz * dz;
                if (!(r2 < rcut2)) continue;
                const double r = sqrt(r2);
                const double qq = C * pi.w * p.w;
                const double ec = erfc(alpha * r);
                const double fm = qq * (ec / r + tap * exp(-alpha * alpha * r2)) / r2;
                fx += fm * dx;
                fy += fm * dy;
                fz += fm * dz;
                e += 0.5 * qq * ec / r;
            }
        }
        __syncthreads();
    }
    if (i < n) {
        atomicAdd(F + 3 * (size_t)i, fx);
        atomicAdd(F + 3 * (size_t)i + 1, fy);
        atomicAdd(F + 3 * (size_t)i + 2, fz);
        atomicAdd(E, e);
    }
}

// Structure factor of each k vector (kv = kx, ky, kz, A with A = 2 (C / V) g(k)); the
// reciprocal energy sum_k A / 2 |S|^2 (half space, so the full-space (C / 2V) g |S|^2).
__global__ void __launch_bounds__(EW_T) k_ewald_structure(const double4 *__restrict__ rq, int n,
                                                          const double4 *__restrict__ kv, int nk,
                                                          double2 *__restrict__ S, double *__restrict__ E) {
    __shared__ double4 sp[EW_T];
    const int k = blockIdx.x * EW_T + threadIdx.x;
    const double4 kk = k < nk ? kv[k] : make_double4(0, 0, 0, 0);
    double sr = 0, si = 0;
    for (int base = 0; base < n; base += EW_T) {
        const int j = base + threadIdx.x;
        sp[threadIdx.x] = j < n ? rq[j] : make_double4(0, 0, 0, 0);
        __syncthreads();
        const int m = min(EW_T, n - base);
        for (int t = 0; t < m; ++t) {
            const double4 p = sp[t];
            double s, c;
            sincos(kk.x * p.x + kk.y * p.y + kk.z * p.z, &s, &c);
            sr = fma(p.w, c, sr);
            si = fma(p.w, s, si);
        }
        __syncthreads();
    }
    if (k < nk) {
        S[k] = make_double2(sr, si);
        atomicAdd(E, 0.5 * kk.w * (sr * sr + si * si));
    }
}

__global__ void __launch_bounds__(EW_T) k_ewald_recip_force(const double4 *__restrict__ rq, int n,
                                                            const double4 *__restrict__ kv,
                                                            const double2 *__restrict__ S, int nk,
                                                            double *__restrict__ F) {
    __shared__ double4 sk[EW_T];
    __shared__ double2 ss[EW_T];
    const int i = blockIdx.x * EW_T + threadIdx.x;
    const double4 pi = i < n ? rq[i] : make_double4(0, 0, 0, 0);
    double fx = 0, fy = 0, fz = 0;
    const int per = (nk + gridDim.y - 1) / gridDim.y;
    const int k0 = blockIdx.y * per, k1 = min(nk, k0 + per);
    for (int base = k0; base < k1; base += EW_T) {
        const int k = base + threadIdx.x;
        sk[threadIdx.x] = k < k1 ? kv[k] : make_double4(0, 0, 0, 0);
        ss[threadIdx.x] = k < k1 ? S[k] : make_double2(0, 0);
        __syncthreads();
        const int m = min(EW_T, k1 - base);
        for (int t = 0; t < m; ++t) {
            const double4 kk = sk[t];
            const double2 s2 = ss[t];
            double s, c;
            sincos(kk.x * pi.x + kk.y * pi.y + kk.z * pi.z, &s, &c);
            const double f = kk.w * (s * s2.x - c * s2.y);
            fx = fma(f, kk.x, fx);
            fy = fma(f, kk.y, fy);
            fz = fma(f, kk.z, fz);
        }
        __syncthreads();
    }
    if (i < n) {
        atomicAdd(F + 3 * (size_t)i, pi.w * fx);
        atomicAdd(F + 3 * (size_t)i + 1, pi.w * fy);
        atomicAdd(F + 3 * (size_t)i + 2, pi.w * fz);
    }
}

__global__ void k_ewald_self(const double4 *__restrict__ rq, int n, double coef, double *__restrict__ E) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) atomicAdd(E, coef * rq[i].w * rq[i].w);
}

}  // namespace pdb

extern "C" {

int pd_ewald_oracle(int n, const double *rq4, const double box[3], double C, double alpha, double digits, int parts,
                    double *F, double *E) {
    PD_CHECK(n > 0 && rq4 && box && F, PD_EINVAL, "pd_ewald_oracle: bad argument");
    PD_CHECK(alpha > 0 && digits > 0, PD_EINVAL, "pd_ewald_oracle: alpha and digits must be positive");
    const double xx = sqrt(digits * log(10.0));
    const double rcut = xx / alpha, kmax = 2.0 * alpha * xx;
    const double wmin = fmin(box[0], fmin(box[1], box[2]));
    PD_CHECK(!(parts & 1) || 2.0 * rcut < wmin, PD_EINVAL,
             "pd_ewald_oracle: real-space cutoff %g needs every box length above %g", rcut, 2.0 * rcut);
    const double V = box[0] * box[1] * box[2];
    const double4 *r = reinterpret_cast<const double4 *>(rq4);
    double *Ed = nullptr;
    double4 *kv = nullptr;
    double2 *S = nullptr;
    int rc = dalloc(&Ed, 1);
    if (rc) return rc;
    PD_CUDA(cudaMemset(Ed, 0, sizeof(double)));
    PD_CUDA(cudaMemset(F, 0, sizeof(double) * 3 * (size_t)n));
    const int nb = (n + EW_T - 1) / EW_T;
    if (parts & 1) {
        k_ewald_real<<<dim3(nb, EW_KSPLIT), EW_T>>>(r, n, box[0], box[1], box[2], alpha, rcut * rcut, C, F, Ed);
        PD_LAUNCHED();
    }
    if (parts & 2) {
        // half space: m3 > 0, or m3 = 0 and m2 > 0, or m3 = m2 = 0 and m1 > 0
        int mm[3];
        for (int d = 0; d < 3; ++d) mm[d] = (int)ceil(kmax / (2.0 * M_PI / box[d])) + 1;
        std::vector<double4> hk;
        for (int m3 = 0; m3 <= mm[2]; ++m3)
            for (int m2 = (m3 == 0 ? 0 : -mm[1]); m2 <= mm[1]; ++m2)
                for (int m1 = ((m3 == 0 && m2 == 0) ? 1 : -mm[0]); m1 <= mm[0]; ++m1) {
                    const double k[3] = {2.0 * M_PI * m1 / box[0], 2.0 * M_PI * m2 / box[1], 2.0 * M_PI * m3 / box[2]};
                    const double k2 = k[0] * k[0] + k[1] * k[1] + k[2] * k[2];
                    if (!(k2 < kmax * kmax)) continue;
                    const double g = 4.0 * M_PI * exp(-k2 / (4.0 * alpha * alpha)) / k2;
                    hk.push_back(make_double4(k[0], k[1], k[2], 2.0 * (C / V) * g));
                }
        const int nk = (int)hk.size();
        if (nk > 0) {
            if ((rc = dalloc(&kv, (size_t)nk)) || (rc = dalloc(&S, (size_t)nk))) {
                dfree(Ed);
                dfree(kv);
                return rc;
            }
            PD_CUDA(cudaMemcpy(kv, hk.data(), sizeof(double4) * nk, cudaMemcpyHostToDevice));
            k_ewald_structure<<<(nk + EW_T - 1) / EW_T, EW_T>>>(r, n, kv, nk, S, Ed);
            PD_LAUNCHED();
            k_ewald_recip_force<<<dim3(nb, EW_KSPLIT), EW_T>>>(r, n, kv, S, nk, F);
            PD_LAUNCHED();
        }
    }
    if (parts & 4) {
        k_ewald_self<<<nb, EW_T>>>(r, n, -C * alpha / sqrt(M_PI), Ed);
        PD_LAUNCHED();
    }
    const cudaError_t e = cudaDeviceSynchronize();
    double eh = 0.0;
    if (e == cudaSuccess) cudaMemcpy(&eh, Ed, sizeof(double), cudaMemcpyDeviceToHost);
    dfree(Ed);
    dfree(kv);
    dfree(S);
    PD_CHECK(e == cudaSuccess, PD_ECUDA, "pd_ewald_oracle: %s", cudaGetErrorString(e));
    if (E) *E = eh;
    return PD_OK;
}

}  // extern "C"
