// Device step engine of libpdb200: one velocity-Verlet NVE step as a fixed
// sequence of kernels that is captured once into a CUDA graph and replayed.
//
// The reference's device engine (src/engine/ClusterBackend.jl:90-220,
// src/engine/Run.jl:247-294, src/simulation/NVEFusion.jl:3-27) runs
// kick+drift, the list decision, conditional build / prune bodies, the pair
// pass beside the mesh transform, a scatter and the closing kick.  Here:
//   1. k_kick_drift: half kick, drift, wrap, pack of the cluster-ordered force
//      coordinates and the displacement maxima for the list decision, fused;
//   2. the one-thread decision;
//   3. build and prune kernels that run only when the device flags ask for them;
//   4. the pair pass on the main stream and the mesh transform (spread, R2C,
//      solve, C2R) on a second stream;
//   5. the join: mesh gather + slot pair forces + store in storage order +
//      closing half kick, one kernel per super-cluster (k_gather, mesh.cu), or
//      k_scatter_kick without a mesh.
#include <cmath>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "internal.hpp"

using namespace pdb;

struct pd_md {
    pd_cluster *c = nullptr;
    pd_mesh *m = nullptr;
    pd_md_state st;
    float L[3] = {0, 0, 0};
    cudaStream_t side = nullptr;
    cudaStream_t body = nullptr;   // captures the bodies of the conditional nodes
    bool cond_nodes = true;        // false after a failed conditional capture: gated kernels instead
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    // schedule: the pair pass starts after the prune (0), or also waits until the mesh chain has
    // finished its spread (1) or its forward transform (2), so that the critical mesh chain meets
    // less contention from the pair pass's CTAs (pd_md_set_schedule; the bench times the three)
    int pair_wait = 0;
    cudaEvent_t ev_spread = nullptr, ev_r2c = nullptr;
    cudaGraphExec_t exec[2] = {nullptr, nullptr};   // [energy]
    float exec_dt[2] = {0.f, 0.f};
    cudaStream_t exec_stream[2] = {nullptr, nullptr};
    int exec_epoch[2] = {-1, -1};   // pair-kernel shape the graphs were captured with
    int exec_mepoch[2] = {-1, -1};  // mesh epoch the graphs were captured with
    double *esum = nullptr;   // device FP64 energy sum
    float half_c_self = 0.f;
    // learned coarse-mesh correction: descriptors + network on a third stream
    pd_learned *learned = nullptr;
    const pd_mlp *net = nullptr;
    cudaStream_t side2 = nullptr;
    cudaEvent_t ev_fork2 = nullptr, ev_join2 = nullptr;
    // host-buffer steps: the positions are final after the drift, so their copy back runs on its
    // own stream beside the force pass (ev_pos is recorded in every captured step)
    cudaStream_t copy = nullptr;
    cudaEvent_t ev_pos = nullptr, ev_copied = nullptr;
};

namespace pdb {

// Device build/prune decision (_decide_kernel!, Engine.jl:301-324), taken by the
// last block of k_kick_drift once every block's displacement maxima are in.  In a
// captured step it also sets the graph's IF condition for the build body, so the
// build kernels are not launched at all on steps that keep the list (the
// reference's conditional graph nodes, DeviceConditionalGraph.jl:88-132); the
// prune kernel reads the prune flag and returns at once when it is clear.
template <bool COND>
__device__ void decide_step(int *counts, int nstlist, int nstprune, cudaGraphConditionalHandle hb) {
    const float anyr = __int_as_float(atomicAdd(&counts[W_FLAG_ANY], 0));
    const float br = __int_as_float(atomicAdd(&counts[W_FLAG_BUILD], 0));
    bool build, prune;
    if (nstlist > 0) {
        const int k = counts[W_DSTEP];
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
    if (COND) cudaGraphSetConditional(hb, build ? 1u : 0u);
}

// _nve_kick_drift3_kernel! (NVEFusion.jl:3-27) fused with the pack of the force
// coordinates (_pack_kernel!, List.jl:377-413), the displacement maxima of
// _displacement_kernel! (List.jl:787-819) and, in the last block to finish, the
// list decision.
template <bool COND>
__global__ void __launch_bounds__(256) k_kick_drift(int n, float *__restrict__ x, float *__restrict__ y,
                                                    float *__restrict__ z, float *__restrict__ vx,
                                                    float *__restrict__ vy, float *__restrict__ vz,
                                                    const float *__restrict__ fx, const float *__restrict__ fy,
                                                    const float *__restrict__ fz, const float *__restrict__ inv_mass,
                                                    float inv_mass_uniform, float dt, float Lx, float Ly, float Lz,
                                                    const float *__restrict__ q, const int *__restrict__ slot_of,
                                                    float4 *__restrict__ xq, const float4 *__restrict__ rb,
                                                    const float4 *__restrict__ rp, float tb2, float tp2,
                                                    int *__restrict__ counts, int nstlist, int nstprune,
                                                    cudaGraphConditionalHandle hb) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    float ra = 0.f, rbv = 0.f;
    if (i < n) {
        const float c = 0.5f * dt * (inv_mass ? inv_mass[i] : inv_mass_uniform);
        const float ux = fmaf(c, fx[i], vx[i]), uy = fmaf(c, fy[i], vy[i]), uz = fmaf(c, fz[i], vz[i]);
        vx[i] = ux;
        vy[i] = uy;
        vz[i] = uz;
        float xi = fmaf(dt, ux, x[i]), yi = fmaf(dt, uy, y[i]), zi = fmaf(dt, uz, z[i]);
        xi -= (xi >= 0.5f * Lx) ? Lx : 0.f;
        xi += (xi < -0.5f * Lx) ? Lx : 0.f;
        yi -= (yi >= 0.5f * Ly) ? Ly : 0.f;
        yi += (yi < -0.5f * Ly) ? Ly : 0.f;
        zi -= (zi >= 0.5f * Lz) ? Lz : 0.f;
        zi += (zi < -0.5f * Lz) ? Lz : 0.f;
        x[i] = xi;
        y[i] = yi;
        z[i] = zi;
        xq[slot_of[i]] = make_float4(force_coordinate(xi, Lx), force_coordinate(yi, Ly), force_coordinate(zi, Lz),
                                     q ? q[i] : 0.f);
        const float4 b = rb[i];
        float dx = mic(xi - b.x, Lx), dy = mic(yi - b.y, Ly), dz = mic(zi - b.z, Lz);
        float d2 = dx * dx + dy * dy + dz * dz;
        rbv = tb2 > 0.f ? d2 / tb2 : (d2 > 0.f ? __int_as_float(0x7f800000) : 0.f);
        if (!isfinite(rbv)) rbv = __int_as_float(0x7f800000);
        const float4 p = rp[i];
        dx = mic(xi - p.x, Lx);
        dy = mic(yi - p.y, Ly);
        dz = mic(zi - p.z, Lz);
        d2 = dx * dx + dy * dy + dz * dz;
        const float rpv = tp2 > 0.f ? d2 / tp2 : (d2 > 0.f ? __int_as_float(0x7f800000) : 0.f);
        ra = fmaxf(rbv, rpv);
    }
    ra = warp_max(ra);
    rbv = warp_max(rbv);
    __shared__ float sh[2][8];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) {
        sh[0][w] = ra;
        sh[1][w] = rbv;
    }
    __syncthreads();
    if (w == 0) {
        float a = lane < 8 ? sh[0][lane] : 0.f;
        float c = lane < 8 ? sh[1][lane] : 0.f;
        a = warp_max(a);
        c = warp_max(c);
        if (lane == 0) {
            atomicMax(&counts[W_FLAG_ANY], __float_as_int(a));
            atomicMax(&counts[W_FLAG_BUILD], __float_as_int(c));
            __threadfence();
            // the last block to arrive takes the decision (threadfence-reduction pattern)
            if (atomicAdd(&counts[W_TICKET], 1) == (int)gridDim.x - 1) {
                __threadfence();
                counts[W_TICKET] = 0;
                decide_step<COND>(counts, nstlist, nstprune, hb);
            }
        }
    }
}

// Slot forces to storage order with the closing half kick (no mesh):
// _scatter_kernel! (Kernels.jl:207-240) + _nve_kick3_kernel! (SimulationCore.jl:581-592).
template <bool ENERGY>
__global__ void k_scatter_kick(const int *__restrict__ perm, int nslot, const int *__restrict__ counts,
                               float4 *__restrict__ fc, float *__restrict__ vc, const float4 *__restrict__ xq,
                               float half_c_self, float *__restrict__ fx, float *__restrict__ fy,
                               float *__restrict__ fz, float *__restrict__ vx, float *__restrict__ vy,
                               float *__restrict__ vz, const float *__restrict__ inv_mass, float inv_mass_uniform,
                               float half_dt, float *__restrict__ epot, float *__restrict__ vir6) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nslot || s >= counts[W_NS] * SUPER) return;
    const int i = perm[s];
    const float4 f = fc[s];
    fc[s] = make_float4(0.f, 0.f, 0.f, 0.f);
    if (i >= 0) {
        fx[i] = f.x;
        fy[i] = f.y;
        fz[i] = f.z;
        const float cm = half_dt * (inv_mass ? inv_mass[i] : inv_mass_uniform);
        vx[i] = fmaf(cm, f.x, vx[i]);
        vy[i] = fmaf(cm, f.y, vy[i]);
        vz[i] = fmaf(cm, f.z, vz[i]);
        if (ENERGY) {
            const float qi = xq[s].w;
            epot[i] = f.w - half_c_self * qi * qi;
#pragma unroll
            for (int k = 0; k < 6; ++k) vir6[(size_t)i * 6 + k] = vc[(size_t)k * nslot + s];
        }
    }
    if (ENERGY) {
#pragma unroll
        for (int k = 0; k < 6; ++k) vc[(size_t)k * nslot + s] = 0.f;
    }
}

__global__ void k_sum(const float *__restrict__ v, int n, double *__restrict__ out) {
    double s = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) s += (double)v[i];
    s = warp_sum_d(s);
    __shared__ double sh[8];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) sh[w] = s;
    __syncthreads();
    if (w == 0) {
        s = lane < 8 ? sh[lane] : 0.0;
        s = warp_sum_d(s);
        if (lane == 0) red_add_d(out, s);
    }
}

}  // namespace pdb

// The mesh transform forks onto the side stream as soon as the packed coordinates
// of the step exist (after the pack or build), so that it runs beside the prune and
// the pair pass; it reads only the packed coordinates and the super-cluster count.
static int fork_mesh(pd_md *md, int energy, cudaStream_t s) {
    if (!md->m) return PD_OK;
    pd_cluster *c = md->c;
    int rc;
    PD_CUDA(cudaEventRecord(md->ev_fork, s));
    PD_CUDA(cudaStreamWaitEvent(md->side, md->ev_fork, 0));
    if ((rc = mesh_transform_packed(md->m, c->xq, c->nsmax, c->counts + W_NS, energy, md->side, md->ev_spread,
                                    md->ev_r2c)))
        return rc;
    PD_CUDA(cudaEventRecord(md->ev_join, md->side));
    return PD_OK;
}

// The learned correction forks onto the third stream once the step's coordinates are final
// (after the drift); the join waits for it before the closing gather.
static int fork_learned(pd_md *md, cudaStream_t s) {
    if (!md->learned) return PD_OK;
    pd_md_state &st = md->st;
    int rc;
    PD_CUDA(cudaEventRecord(md->ev_fork2, s));
    PD_CUDA(cudaStreamWaitEvent(md->side2, md->ev_fork2, 0));
    if ((rc = learned_correction_launch(md->learned, md->net, st.x, st.y, st.z, st.q, st.type, nullptr, md->side2)))
        return rc;
    PD_CUDA(cudaEventRecord(md->ev_join2, md->side2));
    return PD_OK;
}

// Closing part of a step: the pair pass (the mesh transform already forked), then the join.
static int enqueue_forces(pd_md *md, int energy, float half_dt, cudaStream_t s) {
    pd_cluster *c = md->c;
    pd_mesh *m = md->m;
    pd_md_state &st = md->st;
    int rc;
    if (m && md->pair_wait) PD_CUDA(cudaStreamWaitEvent(s, md->pair_wait == 1 ? md->ev_spread : md->ev_r2c, 0));
    if ((rc = cluster_pairs_launch(c, energy, s))) return rc;
    if (m) {
        PD_CUDA(cudaStreamWaitEvent(s, md->ev_join, 0));
        if (md->learned) PD_CUDA(cudaStreamWaitEvent(s, md->ev_join2, 0));
        rc = mesh_gather_join(m, c, c->xq, c->perm, c->counts + W_NS, c->nsmax, st.fx, st.fy, st.fz, st.vx, st.vy,
                              st.vz, st.inv_mass, st.inv_mass_uniform, half_dt, st.epot, st.vir6, st.vglobal6, st.q,
                              md->half_c_self,
                              md->learned ? (md->net ? learned_corr(md->learned) : learned_radial(md->learned))
                                          : nullptr,
                              energy, s);
        if (rc) return rc;
    } else {
        const int blocks = (c->nslot + 255) / 256;
        if (energy)
            k_scatter_kick<true><<<blocks, 256, 0, s>>>(c->perm, c->nslot, c->counts, c->fc, c->vc, c->xq,
                                                        md->half_c_self, st.fx, st.fy, st.fz, st.vx, st.vy, st.vz,
                                                        st.inv_mass, st.inv_mass_uniform, half_dt, st.epot, st.vir6);
        else
            k_scatter_kick<false><<<blocks, 256, 0, s>>>(c->perm, c->nslot, c->counts, c->fc, c->vc, c->xq,
                                                         md->half_c_self, st.fx, st.fy, st.fz, st.vx, st.vy, st.vz,
                                                         st.inv_mass, st.inv_mass_uniform, half_dt, st.epot,
                                                         st.vir6);
        PD_LAUNCHED();
    }
    return PD_OK;
}

// One full step, device-decided.  cond = 1 (inside a stream capture): the build and
// prune bodies become IF nodes of the captured graph; otherwise their kernels are
// launched and return at once when the device flags are clear.
// Marks the end of the drift (positions final for this step): an external event node inside a
// capture, so that work outside the graph can wait for it; a plain record otherwise.
static int record_positions(pd_md *md, cudaStream_t s) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    PD_CUDA(cudaStreamIsCapturing(s, &cs));
    if (cs == cudaStreamCaptureStatusActive)
        PD_CUDA(cudaEventRecordWithFlags(md->ev_pos, s, cudaEventRecordExternal));
    else
        PD_CUDA(cudaEventRecord(md->ev_pos, s));
    return PD_OK;
}

static int enqueue_step(pd_md *md, float dt, int energy, cudaStream_t s, int cond) {
    pd_cluster *c = md->c;
    pd_md_state &st = md->st;
    const float hb = (float)(0.5 * c->p.skin), hp = (float)(0.5 * c->p.prune_buffer);
    const float *q = c->p.coulomb ? st.q : nullptr;
    int rc;
    const int kb = (st.n + 255) / 256;
    if (cond) {
        cudaStreamCaptureStatus status;
        cudaGraph_t g = nullptr;
        PD_CUDA(cudaStreamGetCaptureInfo(s, &status, nullptr, &g, nullptr, nullptr));
        cudaGraphConditionalHandle hbuild;
        PD_CUDA(cudaGraphConditionalHandleCreate(&hbuild, g, 0, cudaGraphCondAssignDefault));
        k_kick_drift<true><<<kb, 256, 0, s>>>(st.n, st.x, st.y, st.z, st.vx, st.vy, st.vz, st.fx, st.fy, st.fz,
                                              st.inv_mass, st.inv_mass_uniform, dt, md->L[0], md->L[1], md->L[2], q,
                                              c->slot_of, c->xq, c->ref_build, c->ref_prune, hb * hb, hp * hp,
                                              c->counts, c->p.nstlist, c->p.nstprune, hbuild);
        PD_LAUNCHED();
        if ((rc = record_positions(md, s))) return rc;
        if ((rc = capture_if_body(s, md->body, hbuild, [&](cudaStream_t cs) {
                 return cluster_build_launch(c, st.x, st.y, st.z, q, st.type, 1, cs);
             })))
            return rc;
    } else {
        k_kick_drift<false><<<kb, 256, 0, s>>>(st.n, st.x, st.y, st.z, st.vx, st.vy, st.vz, st.fx, st.fy, st.fz,
                                               st.inv_mass, st.inv_mass_uniform, dt, md->L[0], md->L[1], md->L[2], q,
                                               c->slot_of, c->xq, c->ref_build, c->ref_prune, hb * hb, hp * hp,
                                               c->counts, c->p.nstlist, c->p.nstprune, 0);
        PD_LAUNCHED();
        if ((rc = record_positions(md, s))) return rc;
        if ((rc = cluster_build_launch(c, st.x, st.y, st.z, q, st.type, 1, s))) return rc;
    }
    // the mesh transform forks before the prune, which runs as a flag-gated kernel
    if ((rc = fork_learned(md, s))) return rc;
    if ((rc = fork_mesh(md, energy, s))) return rc;
    if ((rc = cluster_prune_launch(c, 1, s))) return rc;
    return enqueue_forces(md, energy, 0.5f * dt, s);
}

extern "C" {

int pd_md_create(pd_md **out, pd_cluster *c, pd_mesh *m, const pd_md_state *st, double box[3]) {
    PD_CHECK(out && c && st && box, PD_EINVAL, "pd_md_create: null argument");
    *out = nullptr;
    PD_CHECK(st->n == c->n, PD_EINVAL, "pd_md_create: state has %d particles, the list %d", st->n, c->n);
    PD_CHECK(st->x && st->y && st->z && st->vx && st->vy && st->vz && st->fx && st->fy && st->fz, PD_EINVAL,
             "pd_md_create: state arrays missing");
    PD_CHECK(!m || st->q, PD_EINVAL, "pd_md_create: a mesh needs charges");
    PD_CHECK(!m || m->p.nmax >= 0, PD_EINVAL, "bad mesh");
    pd_md *md = new pd_md();
    md->c = c;
    md->m = m;
    md->st = *st;
    for (int d = 0; d < 3; ++d) md->L[d] = (float)box[d];
    md->half_c_self = c->p.coulomb ? 0.5f * c->p.coul_C * c->p.selfc : 0.f;
    // the mesh chain (spread, transforms, solve) is latency-bound and on the step's
    // critical path: its stream takes the highest priority, the pair pass fills in
    int prio_lo = 0, prio_hi = 0;
    cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi);
    if (cudaStreamCreateWithPriority(&md->side, cudaStreamNonBlocking, prio_hi) != cudaSuccess ||
        cudaStreamCreateWithFlags(&md->body, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&md->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&md->ev_spread, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&md->ev_r2c, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&md->ev_join, cudaEventDisableTiming) != cudaSuccess ||
        cudaStreamCreateWithFlags(&md->copy, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&md->ev_pos, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&md->ev_copied, cudaEventDisableTiming) != cudaSuccess ||
        dalloc(&md->esum, 1) != PD_OK) {
        set_error("pd_md_create: stream/event allocation failed");
        pd_md_destroy(md);
        return PD_ECUDA;
    }
    *out = md;
    return PD_OK;
}

int pd_md_destroy(pd_md *md) {
    if (!md) return PD_OK;
    for (int k = 0; k < 2; ++k)
        if (md->exec[k]) cudaGraphExecDestroy(md->exec[k]);
    if (md->ev_fork) cudaEventDestroy(md->ev_fork);
    if (md->ev_spread) cudaEventDestroy(md->ev_spread);
    if (md->ev_r2c) cudaEventDestroy(md->ev_r2c);
    if (md->ev_join) cudaEventDestroy(md->ev_join);
    if (md->ev_pos) cudaEventDestroy(md->ev_pos);
    if (md->ev_copied) cudaEventDestroy(md->ev_copied);
    if (md->copy) cudaStreamDestroy(md->copy);
    if (md->side) cudaStreamDestroy(md->side);
    if (md->body) cudaStreamDestroy(md->body);
    if (md->side2) cudaStreamDestroy(md->side2);
    if (md->ev_fork2) cudaEventDestroy(md->ev_fork2);
    if (md->ev_join2) cudaEventDestroy(md->ev_join2);
    dfree(md->esum);
    delete md;
    return PD_OK;
}

// evaluate_forces_into_f!: eager list maintenance (host boundary) and one force pass without kicks.
int pd_md_evaluate(pd_md *md, int energy, pd_stream_t sp) {
    PD_CHECK(md, PD_EINVAL, "pd_md_evaluate: null handle");
    cudaStream_t s = (cudaStream_t)sp;
    pd_cluster *c = md->c;
    pd_md_state &st = md->st;
    const float *q = c->p.coulomb ? st.q : nullptr;
    int rc, h[W_LEN];
    if ((rc = cluster_decide_launch(c, st.x, st.y, st.z, 0, s))) return rc;
    if ((rc = cluster_read_counts(c, h, s))) return rc;
    if (h[W_BUILD] || !c->have_build) {
        for (int attempt = 0; attempt < 8; ++attempt) {
            if ((rc = cluster_build_launch(c, st.x, st.y, st.z, q, st.type, 0, s))) return rc;
            if ((rc = cluster_read_counts(c, h, s))) return rc;
            if (h[W_ERR] == 0) break;
            if (h[W_ERR] == PD_ENONFINITE) {
                set_error("Cluster-pair list: non-finite coordinates");
                return PD_ENONFINITE;
            }
            if ((rc = pd_cluster_grow(c))) return rc;
            // the graphs captured the old entry storage
            for (int k = 0; k < 2; ++k)
                if (md->exec[k]) {
                    cudaGraphExecDestroy(md->exec[k]);
                    md->exec[k] = nullptr;
                }
        }
        PD_CHECK(h[W_ERR] == 0, PD_ECAPACITY, "outer list still overflows after growth");
        c->have_build = true;
        if ((rc = cluster_set_word(c, W_PRUNE, 1, s))) return rc;
    } else {
        if ((rc = pd_cluster_pack(c, st.x, st.y, st.z, q, st.type, sp))) return rc;
    }
    if ((rc = fork_learned(md, s))) return rc;
    if ((rc = fork_mesh(md, energy, s))) return rc;
    if ((rc = cluster_prune_launch(c, 1, s))) return rc;
    return enqueue_forces(md, energy, 0.f, s);
}

int pd_md_set_learned(pd_md *md, pd_learned *h, pd_mlp *net) {
    PD_CHECK(md, PD_EINVAL, "pd_md_set_learned: null handle");
    PD_CHECK(h || !net, PD_EINVAL, "pd_md_set_learned: a network needs the correction handle");
    PD_CHECK(!h || md->m, PD_EINVAL, "pd_md_set_learned: the correction needs a mesh");
    if (h && !md->side2) {
        int prio_lo = 0, prio_hi = 0;
        cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi);
        PD_CUDA(cudaStreamCreateWithPriority(&md->side2, cudaStreamNonBlocking, prio_hi));
        PD_CUDA(cudaEventCreateWithFlags(&md->ev_fork2, cudaEventDisableTiming));
        PD_CUDA(cudaEventCreateWithFlags(&md->ev_join2, cudaEventDisableTiming));
    }
    md->learned = h;
    md->net = net;
    // captured steps hold the old sequence
    for (int k = 0; k < 2; ++k)
        if (md->exec[k]) {
            cudaGraphExecDestroy(md->exec[k]);
            md->exec[k] = nullptr;
        }
    return PD_OK;
}

int pd_md_set_schedule(pd_md *md, int pair_wait) {
    PD_CHECK(md, PD_EINVAL, "pd_md_set_schedule: null handle");
    PD_CHECK(pair_wait >= 0 && pair_wait <= 2, PD_EINVAL, "pd_md_set_schedule: pair_wait 0, 1 or 2");
    if (md->pair_wait != pair_wait) {
        md->pair_wait = pair_wait;
        for (int k = 0; k < 2; ++k)   // captured steps hold the old dependencies
            if (md->exec[k]) {
                cudaGraphExecDestroy(md->exec[k]);
                md->exec[k] = nullptr;
            }
    }
    return PD_OK;
}

int pd_md_step(pd_md *md, int nsteps, float dt, int energy_last, int use_graph, pd_stream_t sp) {
    PD_CHECK(md, PD_EINVAL, "pd_md_step: null handle");
    PD_CHECK(nsteps >= 0, PD_EINVAL, "pd_md_step: negative step count");
    cudaStream_t s = (cudaStream_t)sp;
    int rc;
    if (!md->c->have_build) {
        if ((rc = pd_md_evaluate(md, 0, sp))) return rc;
    }
    for (int k = 0; k < nsteps; ++k) {
        const int energy = (energy_last && k == nsteps - 1) ? 1 : 0;
        if (!use_graph) {
            if ((rc = enqueue_step(md, dt, energy, s, 0))) return rc;
            continue;
        }
        if (!md->exec[energy] || md->exec_dt[energy] != dt || md->exec_stream[energy] != s ||
            md->exec_epoch[energy] != md->c->shape_epoch || (md->m && md->exec_mepoch[energy] != md->m->epoch)) {
            if (md->exec[energy]) {
                cudaGraphExecDestroy(md->exec[energy]);
                md->exec[energy] = nullptr;
            }
            PD_CHECK(s != nullptr, PD_EINVAL, "pd_md_step: graph replay needs a non-default stream");
            // conditional IF nodes for build / prune; if this driver refuses them, capture the gated kernels
            for (int attempt = 0; attempt < 2 && !md->exec[energy]; ++attempt) {
                const int cond = md->cond_nodes ? 1 : 0;
                cudaGraph_t g = nullptr;
                PD_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
                rc = enqueue_step(md, dt, energy, s, cond);
                cudaError_t e = cudaStreamEndCapture(s, &g);
                // per-node priorities: the mesh branch, captured from the high-priority side stream,
                // keeps its priority inside the graph (the default instantiation drops it)
                if (rc == PD_OK && e == cudaSuccess)
                    e = cudaGraphInstantiateWithFlags(&md->exec[energy], g, cudaGraphInstantiateFlagUseNodePriority);
                if (g) cudaGraphDestroy(g);
                if (rc == PD_OK && e == cudaSuccess) break;
                md->exec[energy] = nullptr;
                cudaGetLastError();
                if (!cond) {
                    if (rc) return rc;
                    PD_CHECK(false, PD_ECUDA, "step capture failed: %s", cudaGetErrorString(e));
                }
                md->cond_nodes = false;
            }
            md->exec_dt[energy] = dt;
            md->exec_stream[energy] = s;
            md->exec_epoch[energy] = md->c->shape_epoch;
            if (md->m) md->exec_mepoch[energy] = md->m->epoch;
        }
        PD_CUDA(cudaGraphLaunch(md->exec[energy], s));
    }
    return PD_OK;
}

int pd_md_step_host(pd_md *md, float *host_xyz, float *host_v, int nsteps, float dt, double *epot_sum, pd_stream_t sp) {
    PD_CHECK(md && host_xyz && host_v, PD_EINVAL, "pd_md_step_host: null argument");
    cudaStream_t s = (cudaStream_t)sp;
    pd_md_state &st = md->st;
    const size_t nb = sizeof(float) * (size_t)st.n;
    float *dx[3] = {st.x, st.y, st.z}, *dv[3] = {st.vx, st.vy, st.vz};
    // copies in: one per array triple when the caller keeps its components in one block, one for the
    // whole state when positions and velocities are adjacent blocks on both sides
    const bool xblock = st.y == st.x + st.n && st.z == st.y + st.n;
    const bool vblock = st.vy == st.vx + st.n && st.vz == st.vy + st.n;
    const bool whole = xblock && vblock && st.vx == st.x + 3 * (size_t)st.n && host_v == host_xyz + 3 * (size_t)st.n;
    if (whole) {
        PD_CUDA(cudaMemcpyAsync(st.x, host_xyz, 6 * nb, cudaMemcpyHostToDevice, s));
    } else {
        for (int d = 0; d < (xblock ? 1 : 3); ++d)
            PD_CUDA(cudaMemcpyAsync(dx[d], host_xyz + (size_t)d * st.n, xblock ? 3 * nb : nb, cudaMemcpyHostToDevice,
                                    s));
        for (int d = 0; d < (vblock ? 1 : 3); ++d)
            PD_CUDA(cudaMemcpyAsync(dv[d], host_v + (size_t)d * st.n, vblock ? 3 * nb : nb, cudaMemcpyHostToDevice,
                                    s));
    }
    int rc = pd_md_step(md, nsteps, dt, epot_sum ? 1 : 0, 1, sp);
    if (rc) return rc;
    if (epot_sum) {
        PD_CUDA(cudaMemsetAsync(md->esum, 0, sizeof(double), s));
        k_sum<<<std::min(1024, (st.n + 255) / 256), 256, 0, s>>>(st.epot, st.n, md->esum);
        PD_LAUNCHED();
        PD_CUDA(cudaMemcpyAsync(epot_sum, md->esum, sizeof(double), cudaMemcpyDeviceToHost, s));
    }
    // positions: final after the last step's drift (ev_pos), copied back while its forces are computed;
    // velocities after the closing kick
    PD_CUDA(cudaStreamWaitEvent(md->copy, md->ev_pos, 0));
    for (int d = 0; d < (xblock ? 1 : 3); ++d)
        PD_CUDA(cudaMemcpyAsync(host_xyz + (size_t)d * st.n, dx[d], xblock ? 3 * nb : nb, cudaMemcpyDeviceToHost,
                                md->copy));
    PD_CUDA(cudaEventRecord(md->ev_copied, md->copy));
    for (int d = 0; d < (vblock ? 1 : 3); ++d)
        PD_CUDA(cudaMemcpyAsync(host_v + (size_t)d * st.n, dv[d], vblock ? 3 * nb : nb, cudaMemcpyDeviceToHost, s));
    PD_CUDA(cudaStreamWaitEvent(s, md->ev_copied, 0));
    PD_CUDA(cudaStreamSynchronize(s));
    return PD_OK;
}

}  // extern "C"
