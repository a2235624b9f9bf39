// Host-side structures of libpdb200 shared by its translation units.
#pragma once

#include <cuda_runtime.h>
#include <cufft.h>
#include <stdint.h>
#include <string>

#include "../../include/pdb200.h"

namespace pdb {

// Thread-local message of the last failure (pd_last_error).
void set_error(const char *fmt, ...);
void count_launch(int n = 1);

#define PD_CUDA(call)                                                                   \
    do {                                                                                \
        cudaError_t e_ = (call);                                                        \
        if (e_ != cudaSuccess) {                                                        \
            ::pdb::set_error("%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_),     \
                             __FILE__, __LINE__);                                       \
            return e_ == cudaErrorMemoryAllocation ? PD_ENOMEM : PD_ECUDA;              \
        }                                                                               \
    } while (0)

#define PD_LAUNCHED()                                                                   \
    do {                                                                                \
        ::pdb::count_launch();                                                          \
        cudaError_t e_ = cudaGetLastError();                                            \
        if (e_ != cudaSuccess) {                                                        \
            ::pdb::set_error("kernel launch failed: %s (%s:%d)", cudaGetErrorString(e_), \
                             __FILE__, __LINE__);                                       \
            return PD_ECUDA;                                                            \
        }                                                                               \
    } while (0)

#define PD_CHECK(cond, code, ...)        \
    do {                                 \
        if (!(cond)) {                   \
            ::pdb::set_error(__VA_ARGS__); \
            return (code);               \
        }                                \
    } while (0)

template <typename T>
int dalloc(T **p, size_t count) {
    *p = nullptr;
    if (count == 0) count = 1;
    cudaError_t e = cudaMalloc((void **)p, count * sizeof(T));
    if (e != cudaSuccess) {
        set_error("cudaMalloc of %zu bytes failed: %s", count * sizeof(T), cudaGetErrorString(e));
        *p = nullptr;
        return PD_ENOMEM;
    }
    return PD_OK;
}
template <typename T>
void dfree(T *&p) {
    if (p) cudaFree((void *)p);
    p = nullptr;
}

// Parameters of the fused pair kernel, passed by value (kernel parameter space).
struct PairParams {
    float Lx, Ly, Lz;
    int lj_kind;
    float c6, c12, lrc2, esh;     // uniform LJ
    int ntypes;
    int coulomb;
    float C, rc2, sx, eshift;
    int ne, nf;
    int has_mesh;                 // excluded pairs beyond r_c remove the mesh's full 1/r (coul_has_mesh)
    int lj_excl;                  // masked pairs also drop their LJ term (bond exclusions)
    float pe[PD_MAX_POLY];
    float pf[PD_MAX_POLY];
};

// Geometry of the cluster list for n particles in a box (the setup! rules, List.jl:874-937).
struct ClusterGeom {
    int ncx, ncy, ncol, nzb, nsmax, nslot, mx, my, ncs;
    long long nbin;
    double rho, rlist;
};
// Argument checks of an engine's parameters (shared by every cluster entry point that takes them).
int cluster_check_params(const pd_cluster_params *p);
// The box checks and geometry rules for n particles and list radius rlist; PD_EINVAL on a bad box.
int cluster_geometry(int n, double rlist, const double box[3], ClusterGeom *g);
// Pair-kernel parameters of an engine (box lengths from box, the rest from p).
void cluster_pair_params(const pd_cluster_params *p, const double box[3], PairParams *pp);

}  // namespace pdb

struct pd_cluster {
    pd_cluster_params p;
    int n = 0;
    double box[3] = {0, 0, 0};
    float L[3] = {0, 0, 0};
    double rlist = 0;
    // geometry of the last setup (List.jl:874-937)
    int ncx = 0, ncy = 0, nzb = 0, mx = 0, my = 0, ncol = 0, nbin = 0, nsmax = 0, nslot = 0, ncs = 0;
    int necap = 0;
    bool grown = false;
    bool have_build = false;
    int nsplit = 1;
    int pair_warps = 2;        // warps per super-cluster part of the pair kernel
    int shape_epoch = 0;       // incremented when the pair-kernel shape changes (captured steps re-capture)
    int num_sms = 148;
    // device buffers
    int *counts = nullptr;     // W_LEN words
    int *bin = nullptr;        // N
    int *bcnt = nullptr;       // nbin, zero between builds
    int *bstart = nullptr;     // nbin + 1
    int *cursor = nullptr;     // nbin
    int *sorted = nullptr;     // N
    int *col_sc_off = nullptr; // ncol + 1
    int *sc_first = nullptr, *sc_n = nullptr, *sc_col = nullptr;  // nsmax
    int *perm = nullptr;       // nslot (-1 padding)
    int *slot_of = nullptr;    // N
    int *order = nullptr;      // N
    float4 *xq = nullptr;      // nslot
    int *ts = nullptr;         // nslot
    float4 *cbc = nullptr, *cbh = nullptr;   // 8 nsmax cluster boxes (centre, half width)
    float4 *sbc = nullptr, *sbh = nullptr;   // nsmax super-cluster boxes
    int *cnt_sc = nullptr;     // nsmax
    int *colcnt = nullptr;     // nsmax * ncs: outer entries per (super-cluster, search column)
    int *scio = nullptr;       // nsmax + 1
    uint32_t *cjo = nullptr;   // necap
    uint2 *cjw = nullptr;      // necap
    int *nw = nullptr;         // nsmax
    float4 *fc = nullptr;      // nslot: force xyz + energy
    float *vc = nullptr;       // 6 nslot
    float4 *ref_build = nullptr, *ref_prune = nullptr;  // N
    float *lj_table = nullptr; // ntypes^2 x 4 (device)
    // Coulomb exceptions (pd_cluster_set_exceptions): CSR rows by particle (both orientations),
    // per outer entry its slot in the exclusion masks (0: none), per working entry the same, the
    // 64-bit pair masks of the flagged entries (8 per entry, one per i-cluster) and the pairs
    // computed outside the tiles: in-list pairs with a nonzero scale (coef = scale) and pairs
    // beyond the list (coef = scale - 1)
    int nexc = 0;              // canonical exception pairs
    int *exo = nullptr;        // N + 1
    int *exj = nullptr;        // 2 nexc
    float *exs = nullptr;      // 2 nexc
    int *xid = nullptr;        // necap
    int *wxid = nullptr;       // necap
    unsigned long long *xmask = nullptr;  // 8 nexc
    int *xpi = nullptr, *xpj = nullptr;   // nexc
    float *xpc = nullptr;      // nexc
    // Bond exclusions (lj_excl): the masks also drop LJ; the corrections restore the LJ term of
    // masked pairs that are not bonded (lr) and the Coulomb potential shift of bonded pairs that
    // carry their full Coulomb term (sh, energy only); storage indices
    int lj_excl = 0;
    int nlr = 0, nsh = 0;
    int *lri = nullptr, *lrj = nullptr;
    int *shi = nullptr, *shj = nullptr;
    pdb::PairParams pp;
};

struct pd_mesh {
    pd_mesh_params p;
    int K1 = 0, K2 = 0, K3 = 0, K1h = 0;
    int nmodes = 0, nnodes = 0;
    double box[3] = {0, 0, 0};
    double ubg = 0.0;          // background energy
    float bg = 0.0f;           // background potential per unit charge
    int nmax_packed = 0;
    float *gridA = nullptr;    // charge grid (kept zero between transforms)
    float *gridB = nullptr;    // potential grid
    float *field[3] = {nullptr, nullptr, nullptr};  // ik field grids
    cufftComplex *spec = nullptr;
    cufftComplex *scratch = nullptr;                // ik
    float *G = nullptr;        // nmodes
    float *Vc = nullptr;       // 6 nmodes (row c: c * nmodes + m)
    double *acc = nullptr;     // 7
    float4 *packed = nullptr;  // particles packed in the caller's order (SoA entry points)
    cufftHandle fwd = 0, bwd = 0;
    bool plans = false;
    void *work = nullptr;
    size_t work_size = 0;
    cudaStream_t plan_stream = nullptr;
    // ESP (prolate split and window): quadrature of the split's transform, window node polynomials
    // ((deg + 1) x H floats) and the per-axis deconvolution or alias tables, all on the device
    bool prolate = false;
    double split_rc = 0.0, bg_coef = 0.0;
    int nquad = 0;
    double *xq = nullptr, *wchi = nullptr;
    float *wpoly = nullptr;
    int wdeg = 0;
    double *wtab[3] = {nullptr, nullptr, nullptr};
    float4 *self_tab = nullptr; // self-force table (T^3 samples of the fractional position), or null
    int self_T = 0;
    int epoch = 0;              // bumped when a change needs captured steps to be captured again
};

namespace pdb {
// Mesh internals used by the step engine.
// ev_spread / ev_r2c (optional) are recorded once the spread / the forward transform are enqueued.
int mesh_transform_packed(pd_mesh *m, const float4 *xq, int nchunks, const int *ns_dev, int energy, cudaStream_t s,
                          cudaEvent_t ev_spread = nullptr, cudaEvent_t ev_r2c = nullptr);
int mesh_gather_join(pd_mesh *m, pd_cluster *c, const float4 *xq, const int *perm, const int *ns_dev, int nchunks,
                     float *fx, float *fy, float *fz, float *vx, float *vy, float *vz, const float *inv_mass,
                     float inv_mass_uniform, float half_dt, float *epot, float *vir6, float *vglobal6, const float *q,
                     float half_c_self, const float4 *extra, int energy, cudaStream_t s);
int mesh_store_virial(pd_mesh *m, float *vglobal6, cudaStream_t s);
// Cluster internals used by the step engine.
int cluster_decide_launch(pd_cluster *c, const float *x, const float *y, const float *z, int fixed, cudaStream_t s);
int cluster_pairs_launch(pd_cluster *c, int energy, cudaStream_t s);
// The pair pass of an engine with exceptions (tiles with exclusion masks, then the pairs outside them).
int cluster_pairs_launch_excl(pd_cluster *c, int energy, cudaStream_t s);
int cluster_build_launch(pd_cluster *c, const float *x, const float *y, const float *z, const float *q,
                         const int *type, int conditional, cudaStream_t s);
int cluster_prune_launch(pd_cluster *c, int conditional, cudaStream_t s);
int cluster_read_counts(pd_cluster *c, int *host, cudaStream_t s);
// Exception pairs computed outside the tiles and the bond-exclusion corrections, added to the slot
// accumulators (part of the pair pass: cluster_pairs_launch runs it after the tiles).
int cluster_exceptions_launch(pd_cluster *c, int energy, cudaStream_t s);
// Frees an engine's exception buffers.
void cluster_free_exceptions(pd_cluster *c);
int cluster_set_word(pd_cluster *c, int word, int value, cudaStream_t s);
// ELL, network and learned-correction internals used by the learned form and the step engine.
int ell_capacity(const pd_ell *e);
int mlp_forward_launch(const pd_mlp *q, const void *X, int n, float *s, const float4 *V, float4 *corr,
                       cudaStream_t st);
int learned_correction_launch(pd_learned *h, const pd_mlp *net, const float *x, const float *y, const float *z,
                              const float *q, const int *type, float4 *corr, cudaStream_t s);
const float4 *learned_corr(const pd_learned *h);
const float4 *learned_radial(const pd_learned *h);
int ell_sort_cells_launch(const int *cell_of, int n, int ncell, int *cell_count, int *cell_off, int *sorted, int *tmp,
                          long long *st, cudaStream_t s);

// Batched meshes of charged replicas (batch_mesh.cu).  Replica r's real grids start at float
// `grid` of the concatenated grids and its half spectrum (and influence function) at complex mode
// `modes`; replicas of one mesh size are adjacent, so one batched cuFFT plan transforms them all.
struct BMeshRep {
    int K1, K2, K3, K1h;
    float Lx, Ly, Lz;
    int nmodes;
    long long grid;
    long long modes;
};

// What the batched mesh kernels read and write.  Particles are processed in chunks of `chunk`
// consecutive cell-order positions of one replica (padded slots: slot_src = -1).
struct BMeshView {
    int order, chunk, nchunk, nrep;
    int tpi;                     // threads per particle of the spread and gather CTAs (2 or 4)
    const BMeshRep *reps;
    const int *chunk_rep;        // nchunk
    const int *slot_src;         // nchunk * chunk: cell-order position or -1
    float4 *mq;                  // nchunk * chunk: (x, y, z, q) of the slot's particle
    int *mid;                    // nchunk * chunk: particle index or -1
    float *gridA, *gridB;        // charge grids (zero between steps), potential grids
    float2 *spec;
    const float *G;
    long long total_nodes, total_modes;
};

struct BMeshKick {
    float *vx, *vy, *vz;
    const float *inv_mass;
    float half_dt;
    int on;
};

// Pack the step's coordinates and charges: xq (cell order, for the pair kernel) and the padded
// chunk slots of the mesh.  Skipped while the rows are invalid (st[E_VALID] == 0).
int bmesh_pack_launch(const BMeshView &v, const float *x, const float *y, const float *z, const float *q,
                      const int *sorted, float4 *xq, const long long *st, cudaStream_t s);
int bmesh_spread_launch(const BMeshView &v, const long long *st, cudaStream_t s);
// spec *= G over every replica's modes; clears the charge grids for the next spread.
int bmesh_solve_launch(const BMeshView &v, const long long *st, cudaStream_t s);
// AD gather joined with the pair forces already stored in f: f += mesh force, the closing half kick
// when kick.on, and with energy epot += q phi / 2 - half_c_self q^2.
int bmesh_gather_launch(const BMeshView &v, float *fx, float *fy, float *fz, float *epot, int energy,
                        const BMeshKick &kick, float half_c_self, const long long *st, cudaStream_t s);

// Append an IF node on handle h to the graph being captured on s, capture body(cs) into its body
// graph on the helper stream cs, and continue s after the node.
template <typename F>
inline int capture_if_body(cudaStream_t s, cudaStream_t cs, cudaGraphConditionalHandle h, F &&body) {
    cudaStreamCaptureStatus status;
    cudaGraph_t g = nullptr;
    const cudaGraphNode_t *deps = nullptr;
    size_t ndeps = 0;
    PD_CUDA(cudaStreamGetCaptureInfo(s, &status, nullptr, &g, &deps, &ndeps));
    PD_CHECK(status == cudaStreamCaptureStatusActive, PD_ESTATE, "conditional node outside a capture");
    cudaGraphNodeParams p = {};
    p.type = cudaGraphNodeTypeConditional;
    p.conditional.handle = h;
    p.conditional.type = cudaGraphCondTypeIf;
    p.conditional.size = 1;
    cudaGraphNode_t node;
    PD_CUDA(cudaGraphAddNode(&node, g, deps, ndeps, &p));
    PD_CUDA(cudaStreamBeginCaptureToGraph(cs, p.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                          cudaStreamCaptureModeRelaxed));
    const int rc = body(cs);
    cudaGraph_t done = nullptr;
    const cudaError_t err = cudaStreamEndCapture(cs, &done);
    if (rc) return rc;
    PD_CHECK(err == cudaSuccess, PD_ECUDA, "conditional body capture failed: %s", cudaGetErrorString(err));
    PD_CUDA(cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies));
    return PD_OK;
}
}  // namespace pdb
