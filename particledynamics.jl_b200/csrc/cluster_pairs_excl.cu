// Exceptions on the cluster route of libpdb200: the pair pass with exclusion masks, the pairs computed
// outside the tiles and the host set-up of the exception rows.
//
// Semantics (ParticleDynamics.jl): the excluded branch of pair_force (src/clusterpairs/PairFunctor.jl:
// 127-156), _scaled_pairs_kernel!, _lj_restore_kernel! and _coulomb_shift_kernel!
// (src/clusterpairs/Kernels.jl:244-339), normalize_exceptions (src/electrostatics/Spec.jl:200-227) and
// bond_exclusion_rows (src/clusterpairs/Engine.jl:274-290).  Layout of this library: the corrections
// run in slot space, on the packed coordinates and into the slot accumulators, before the scatter (or
// the mesh's fused gather and kick) takes the slots to storage order; one thread per pair.
#include <algorithm>
#include <cmath>
#include <map>
#include <set>
#include <utility>
#include <vector>

#include "cluster_pairs.cuh"

using namespace pdb;

namespace pdb {

// Threads [0, npmax): the scaled and out-of-list pairs the build recorded (counts[W_NP] of them),
// coef C qi qj / r; [npmax, npmax + nlr): the LJ term of masked pairs that are not bonded;
// the rest: the Coulomb potential shift of bonded pairs restored to scale 1 (energy only).
__global__ void k_exceptions(int npmax, int nlr, int nsh, const int *__restrict__ counts,
                             const int *__restrict__ xpi, const int *__restrict__ xpj, const float *__restrict__ xpc,
                             const int *__restrict__ lri, const int *__restrict__ lrj, const int *__restrict__ shi,
                             const int *__restrict__ shj, const int *__restrict__ slot_of,
                             const float4 *__restrict__ xq, const int *__restrict__ ts,
                             const float *__restrict__ lj_table, const PairParams pp, float4 *__restrict__ fc,
                             float *__restrict__ vc, int nslot, int energy) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (counts[W_ERR] != 0) return;
    int i, j, kind;
    if (t < npmax) {
        if (t >= counts[W_NP]) return;
        i = xpi[t];
        j = xpj[t];
        kind = 0;
    } else if (t < npmax + nlr) {
        i = lri[t - npmax];
        j = lrj[t - npmax];
        kind = 1;
    } else if (t < npmax + nlr + nsh) {
        if (!energy) return;
        i = shi[t - npmax - nlr];
        j = shj[t - npmax - nlr];
        kind = 2;
    } else {
        return;
    }
    const int si = slot_of[i], sj = slot_of[j];
    const float4 a = xq[si], b = xq[sj];
    const float dx = periodic_delta(a.x, b.x, 0.5f * pp.Lx, pp.Lx);
    const float dy = periodic_delta(a.y, b.y, 0.5f * pp.Ly, pp.Ly);
    const float dz = periodic_delta(a.z, b.z, 0.5f * pp.Lz, pp.Lz);
    const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
    float f = 0.f, e = 0.f;
    if (kind == 0) {
        const float rinv = 1.f / sqrtf(r2);
        const float sc = xpc[t] * pp.C * a.w * b.w;
        f = sc * rinv * rinv * rinv;
        e = sc * rinv;
    } else if (kind == 1) {
        float c6, c12, lrc2, esh;
        if (pp.lj_kind == PD_LJ_TABLE) {
            const float4 tb = reinterpret_cast<const float4 *>(lj_table)[(ts[si] - 1) * pp.ntypes + ts[sj] - 1];
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
        if (!(r2 < lrc2)) return;
        const float rinv2 = 1.f / r2;
        const float ir6 = rinv2 * rinv2 * rinv2;
        f = (12.f * c12 * ir6 - 6.f * c6) * ir6 * rinv2;
        e = (c12 * ir6 - c6) * ir6 - esh;
    } else {
        if (!(r2 < pp.rc2)) return;
        e = -pp.C * a.w * b.w * pp.eshift;
    }
    float *fi = reinterpret_cast<float *>(&fc[si]), *fj = reinterpret_cast<float *>(&fc[sj]);
    if (kind != 2) {
        red_add(fi + 0, f * dx);
        red_add(fi + 1, f * dy);
        red_add(fi + 2, f * dz);
        red_add(fj + 0, -f * dx);
        red_add(fj + 1, -f * dy);
        red_add(fj + 2, -f * dz);
    }
    if (energy) {
        const float h = 0.5f * e;
        red_add(fi + 3, h);
        red_add(fj + 3, h);
        if (kind != 2) {
            const float hf = 0.5f * f;
            const float w[6] = {hf * dx * dx, hf * dy * dy, hf * dz * dz, hf * dx * dy, hf * dx * dz, hf * dy * dz};
#pragma unroll
            for (int k = 0; k < 6; ++k) {
                red_add(&vc[(size_t)k * nslot + si], w[k]);
                red_add(&vc[(size_t)k * nslot + sj], w[k]);
            }
        }
    }
}

int cluster_exceptions_launch(pd_cluster *c, int energy, cudaStream_t s) {
    const int npmax = c->p.coulomb ? c->nexc : 0;   // the scaled pairs act on charges only
    const int nsh = c->p.coulomb ? c->nsh : 0;
    const int total = npmax + c->nlr + nsh;
    if (total == 0) return PD_OK;
    k_exceptions<<<(total + 255) / 256, 256, 0, s>>>(npmax, c->nlr, nsh, c->counts, c->xpi, c->xpj, c->xpc, c->lri,
                                                     c->lrj, c->shi, c->shj, c->slot_of, c->xq, c->ts, c->lj_table,
                                                     c->pp, c->fc, c->vc, c->nslot, energy);
    PD_LAUNCHED();
    return PD_OK;
}

int cluster_pairs_launch_excl(pd_cluster *c, int energy, cudaStream_t s) {
    pairs_dispatch<true>(c, energy, s);
    PD_LAUNCHED();
    return cluster_exceptions_launch(c, energy, s);
}

void cluster_free_exceptions(pd_cluster *c) {
    dfree(c->exo);
    dfree(c->exj);
    dfree(c->exs);
    dfree(c->xid);
    dfree(c->wxid);
    dfree(c->xmask);
    dfree(c->xpi);
    dfree(c->xpj);
    dfree(c->xpc);
    dfree(c->lri);
    dfree(c->lrj);
    dfree(c->shi);
    dfree(c->shj);
    c->nexc = c->nlr = c->nsh = 0;
    c->lj_excl = 0;
    c->pp.lj_excl = 0;
}

template <typename T>
static int upload(T **d, const std::vector<T> &h) {
    int rc;
    if ((rc = dalloc(d, h.size()))) return rc;
    if (!h.empty()) PD_CUDA(cudaMemcpy(*d, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice));
    return PD_OK;
}

}  // namespace pdb

extern "C" {

int pd_cluster_set_exceptions(pd_cluster *c, int n, const int *pi, const int *pj, const double *scale, int nbond,
                              const int *bi, const int *bj) {
    PD_CHECK(c, PD_EINVAL, "pd_cluster_set_exceptions: null handle");
    PD_CHECK(n >= 0 && nbond >= 0, PD_EINVAL, "pd_cluster_set_exceptions: negative count");
    PD_CHECK(n == 0 || (pi && pj && scale), PD_EINVAL, "pd_cluster_set_exceptions: null exception arrays");
    PD_CHECK(nbond == 0 || (bi && bj), PD_EINVAL, "pd_cluster_set_exceptions: null bond arrays");
    const int N = c->n;
    typedef std::pair<int, int> Key;
    auto key = [](int i, int j) { return i < j ? Key(i, j) : Key(j, i); };
    // normalize_exceptions (Spec.jl:200-227)
    std::map<Key, double> cx;
    for (int k = 0; k < n; ++k) {
        const int i = pi[k], j = pj[k];
        const double sc = scale[k];
        PD_CHECK(i >= 0 && i < N && j >= 0 && j < N, PD_EINVAL,
                 "Exception pair (%d, %d) is out of range for N=%d", i, j, N);
        PD_CHECK(i != j, PD_EINVAL, "Exception pair (%d, %d) refers to a single particle", i, j);
        PD_CHECK(std::isfinite(sc) && sc >= 0.0, PD_EINVAL, "Exception scale must be finite and nonnegative; got %g",
                 sc);
        const Key kk = key(i, j);
        auto it = cx.find(kk);
        if (it != cx.end())
            PD_CHECK(it->second == sc, PD_EINVAL, "Exception pair (%d, %d) is listed with conflicting scales %g and %g",
                     kk.first, kk.second, it->second, sc);
        else
            cx[kk] = sc;
    }
    for (auto it = cx.begin(); it != cx.end();) it = it->second == 1.0 ? cx.erase(it) : std::next(it);
    PD_CHECK(cx.empty() || c->p.coulomb, PD_EINVAL, "Coulomb exceptions need the engine's Coulomb term");
    std::set<Key> bonded;
    for (int k = 0; k < nbond; ++k) {
        const int i = bi[k], j = bj[k];
        PD_CHECK(i >= 0 && i < N && j >= 0 && j < N && i != j, PD_EINVAL, "Bonded pair (%d, %d) is invalid for N=%d",
                 i, j, N);
        bonded.insert(key(i, j));
    }
    PD_CHECK(bonded.empty() || c->p.lj_kind != PD_LJ_NONE, PD_EINVAL,
             "bond exclusions drop the LJ term: the engine has none");
    // bond_exclusion_rows (Engine.jl:274-290): the masks cover the union
    std::vector<std::pair<Key, double>> pairs(cx.begin(), cx.end());
    std::vector<int> lri, lrj, shi, shj;
    for (const Key &kk : bonded) {
        if (cx.count(kk)) continue;
        pairs.push_back({kk, c->p.coulomb ? 1.0 : 0.0});
        if (c->p.coulomb) {
            shi.push_back(kk.first);
            shj.push_back(kk.second);
        }
    }
    if (!bonded.empty())
        for (const auto &kv : cx)
            if (!bonded.count(kv.first)) {
                lri.push_back(kv.first.first);
                lrj.push_back(kv.first.second);
            }
    std::sort(pairs.begin(), pairs.end());
    cluster_free_exceptions(c);
    c->shape_epoch += 1;   // captured steps re-capture with (or without) the exclusion kernels
    int one = 1;
    PD_CUDA(cudaMemcpy(c->counts + W_REQUEST, &one, sizeof(int), cudaMemcpyHostToDevice));
    c->have_build = false;
    if (pairs.empty()) return PD_OK;
    // CSR rows by particle, both orientations (_exception_rows, Solver.jl:100-119)
    const int np = (int)pairs.size();
    std::vector<int> exo(N + 1, 0), exj(2 * (size_t)np);
    std::vector<float> exs(2 * (size_t)np);
    for (const auto &kv : pairs) {
        exo[kv.first.first + 1] += 1;
        exo[kv.first.second + 1] += 1;
    }
    for (int i = 0; i < N; ++i) exo[i + 1] += exo[i];
    std::vector<int> fill(exo.begin(), exo.end() - 1);
    for (const auto &kv : pairs) {
        const int i = kv.first.first, j = kv.first.second;
        exj[fill[i]] = j;
        exs[fill[i]++] = (float)kv.second;
        exj[fill[j]] = i;
        exs[fill[j]++] = (float)kv.second;
    }
    int rc;
    if ((rc = upload(&c->exo, exo)) || (rc = upload(&c->exj, exj)) || (rc = upload(&c->exs, exs)) ||
        (rc = dalloc(&c->xmask, 8 * (size_t)np)) || (rc = dalloc(&c->xpi, (size_t)np)) ||
        (rc = dalloc(&c->xpj, (size_t)np)) || (rc = dalloc(&c->xpc, (size_t)np)) ||
        (rc = dalloc(&c->xid, (size_t)c->necap)) || (rc = dalloc(&c->wxid, (size_t)c->necap)) ||
        (rc = upload(&c->lri, lri)) || (rc = upload(&c->lrj, lrj)) || (rc = upload(&c->shi, shi)) ||
        (rc = upload(&c->shj, shj))) {
        cluster_free_exceptions(c);
        return rc;
    }
    PD_CUDA(cudaMemset(c->xmask, 0, sizeof(unsigned long long) * 8 * (size_t)np));
    PD_CUDA(cudaMemset(c->xid, 0, sizeof(int) * (size_t)c->necap));
    PD_CUDA(cudaMemset(c->wxid, 0, sizeof(int) * (size_t)c->necap));
    c->nexc = np;
    c->nlr = (int)lri.size();
    c->nsh = (int)shi.size();
    c->lj_excl = bonded.empty() ? 0 : 1;
    c->pp.lj_excl = c->lj_excl;
    return PD_OK;
}

}  // extern "C"
