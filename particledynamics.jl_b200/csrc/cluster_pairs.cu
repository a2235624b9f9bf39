// Cluster-pair pass (tiles without exclusion masks) and slot scatter of libpdb200.
//
// Semantics: _cluster_pair_kernel! and _scatter_kernel! of src/clusterpairs/Kernels.jl
// (ParticleDynamics.jl); the kernel itself is in cluster_pairs.cuh.
#include "cluster_pairs.cuh"

using namespace pdb;

namespace pdb {

// Slot buffers to storage order, self energy, zeroing (_scatter_kernel!, Kernels.jl:207-240).
template <bool ENERGY, bool ADD>
__global__ void k_scatter(const int *__restrict__ perm, int nslot, const int *__restrict__ counts,
                          float4 *__restrict__ fc, float *__restrict__ vc, const float *__restrict__ q,
                          float half_c_self, float *__restrict__ fx, float *__restrict__ fy, float *__restrict__ fz,
                          float *__restrict__ epot, float *__restrict__ vir6) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nslot) return;
    const int used = counts[W_NS] * SUPER;
    if (s >= used) return;   // slots past the super-cluster count hold nothing
    const int i = perm[s];
    const float4 f = fc[s];
    if (i >= 0) {
        if (ADD) {
            fx[i] += f.x;
            fy[i] += f.y;
            fz[i] += f.z;
        } else {
            fx[i] = f.x;
            fy[i] = f.y;
            fz[i] = f.z;
        }
        if (ENERGY) {
            float e = f.w;
            if (q) {
                const float qi = q[i];
                e -= half_c_self * qi * qi;
            }
            epot[i] = ADD ? epot[i] + e : e;
            if (vir6) {
#pragma unroll
                for (int k = 0; k < 6; ++k) vir6[(size_t)i * 6 + k] = vc[(size_t)k * nslot + s];
            }
        }
    }
    fc[s] = make_float4(0.f, 0.f, 0.f, 0.f);
    if (ENERGY) {
#pragma unroll
        for (int k = 0; k < 6; ++k) vc[(size_t)k * nslot + s] = 0.f;
    }
}

int cluster_pairs_launch(pd_cluster *c, int energy, cudaStream_t s) {
    if (c->nexc > 0) return cluster_pairs_launch_excl(c, energy, s);
    pairs_dispatch<false>(c, energy, s);
    PD_LAUNCHED();
    return PD_OK;
}

}  // namespace pdb

extern "C" {

int pd_cluster_pairs(pd_cluster *c, int energy, pd_stream_t s) {
    PD_CHECK(c, PD_EINVAL, "pd_cluster_pairs: null handle");
    PD_CHECK(c->have_build, PD_ESTATE, "pd_cluster_pairs: the list has not been built");
    return cluster_pairs_launch(c, energy, (cudaStream_t)s);
}

int pd_cluster_scatter(pd_cluster *c, float *fx, float *fy, float *fz, float *epot, float *vir6, const float *q,
                       int energy, int add, pd_stream_t s) {
    PD_CHECK(c && fx && fy && fz, PD_EINVAL, "pd_cluster_scatter: null argument");
    PD_CHECK(!energy || epot, PD_EINVAL, "pd_cluster_scatter: energy needs epot");
    const float hcs = 0.5f * c->p.coul_C * c->p.selfc;
    const float *qq = c->p.coulomb ? q : nullptr;
    cudaStream_t st = (cudaStream_t)s;
    const int blocks = (c->nslot + 255) / 256;
    if (energy) {
        if (add)
            k_scatter<true, true><<<blocks, 256, 0, st>>>(c->perm, c->nslot, c->counts, c->fc, c->vc, qq, hcs, fx, fy, fz,
                                                          epot, vir6);
        else
            k_scatter<true, false><<<blocks, 256, 0, st>>>(c->perm, c->nslot, c->counts, c->fc, c->vc, qq, hcs, fx, fy,
                                                           fz, epot, vir6);
    } else {
        if (add)
            k_scatter<false, true><<<blocks, 256, 0, st>>>(c->perm, c->nslot, c->counts, c->fc, c->vc, qq, hcs, fx, fy,
                                                           fz, epot, vir6);
        else
            k_scatter<false, false><<<blocks, 256, 0, st>>>(c->perm, c->nslot, c->counts, c->fc, c->vc, qq, hcs, fx,
                                                            fy, fz, epot, vir6);
    }
    PD_LAUNCHED();
    return PD_OK;
}

int pd_cluster_compute(pd_cluster *c, const float *x, const float *y, const float *z, const float *q, const int *type,
                       float *fx, float *fy, float *fz, float *epot, float *vir6, int energy, pd_stream_t s) {
    PD_CHECK(c && x && y && z && fx && fy && fz, PD_EINVAL, "pd_cluster_compute: null argument");
    cudaStream_t st = (cudaStream_t)s;
    int rc;
    int h[W_LEN];
    // update_list! (Engine.jl:160-176): decision at the current coordinates
    if ((rc = cluster_decide_launch(c, x, y, z, 0, st))) return rc;
    if ((rc = cluster_read_counts(c, h, st))) return rc;
    if (h[W_BUILD] || !c->have_build) {
        for (int attempt = 0; attempt < 8; ++attempt) {
            if ((rc = cluster_build_launch(c, x, y, z, q, type, 0, st))) return rc;
            if ((rc = cluster_read_counts(c, h, st))) return rc;
            if (h[W_ERR] == 0) break;
            if (h[W_ERR] == PD_ENONFINITE) {
                set_error("Cluster-pair list: non-finite coordinates");
                return PD_ENONFINITE;
            }
            if ((rc = pd_cluster_grow(c))) return rc;
        }
        PD_CHECK(h[W_ERR] == 0, PD_ECAPACITY, "outer list still overflows after growth");
        c->have_build = true;
        if ((rc = cluster_set_word(c, W_PRUNE, 1, st))) return rc;
    } else {
        if ((rc = pd_cluster_pack(c, x, y, z, q, type, s))) return rc;
    }
    if ((rc = cluster_prune_launch(c, 1, st))) return rc;
    if ((rc = cluster_pairs_launch(c, energy, st))) return rc;
    return pd_cluster_scatter(c, fx, fy, fz, epot, vir6, q, energy, 0, s);
}

}  // extern "C"
