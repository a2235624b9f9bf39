/*
 * pdb200.h — C ABI of libpdb200.so, the B200 (sm_100a) implementation of the
 * per-step force hot path of ParticleDynamics.jl.
 *
 * The ABI is what the reference's Julia host code would `ccall` in place of
 * the bodies of its hot-path kernels.  Every entry point takes plain pointers
 * (caller arrays are DEVICE pointers unless stated otherwise), sizes and a
 * CUDA stream, and returns an int status (PD_OK = 0).  No C++ or torch types
 * cross the boundary.  Handles are not thread-safe: use one handle per stream.
 *
 * Reference paths below are relative to the ParticleDynamics.jl project root.
 *
 * Ownership follows the reference (src/electrostatics/Solver.jl:68-74,
 * src/clusterpairs/List.jl:18-27): the caller owns the particle arrays
 * (structure-of-arrays float32 x, y, z, q, forces, energies) and passes them
 * on every call; the library owns its workspaces, allocates them only in the
 * *_create / *_setup / *_grow / *_set_box calls, and never allocates, frees or
 * synchronises inside the enqueue calls, so enqueue calls can be captured in a
 * CUDA graph.
 *
 * Errors: host argument errors return PD_EINVAL with a message available from
 * pd_last_error().  In-stream failures (outer-list capacity, non-finite
 * coordinates) latch a device error word inside the handle; every later list
 * and pair kernel of that handle then does nothing (as the reference's
 * counts[CL_ERR], src/clusterpairs/List.jl:25-27, Kernels.jl:51) until the
 * host reads the status at a boundary (pd_cluster_status) and grows the list
 * (pd_cluster_grow).  No kernel traps.
 */
#ifndef PDB200_H
#define PDB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* A cudaStream_t passed as an opaque pointer (NULL = the legacy default stream). */
typedef void *pd_stream_t;

enum pd_status_code {
    PD_OK = 0,
    PD_EINVAL = 1,      /* bad argument (ArgumentError in the reference) */
    PD_ENOMEM = 2,      /* device allocation failed */
    PD_ECAPACITY = 3,   /* outer cluster list overflowed; pd_cluster_grow, then rebuild */
    PD_ENONFINITE = 4,  /* non-finite coordinates met by a list build */
    PD_ECUFFT = 5,      /* a cuFFT call failed */
    PD_ECUDA = 6,       /* a CUDA runtime call failed */
    PD_ESTATE = 7,      /* call out of order (e.g. pairs before any build) */
    PD_ENOTSUP = 8      /* valid request this build does not support */
};

/* Library version (major*10000 + minor*100 + patch). */
int pd_version(void);
/* Static text for a status code. */
const char *pd_strerror(int code);
/* Message of the last failure on the calling thread ("" if none). */
const char *pd_last_error(void);
/* Number of kernel launches this library has issued on the calling process. */
uint64_t pd_launch_count(void);

/* ======================================================================
 * Cluster-pair engine: ClusterPairEngine + ClusterPairList
 * (src/clusterpairs/Engine.jl:15-97, src/clusterpairs/List.jl:112-179).
 *
 * Particles are clustered into x-y columns of about one super-cluster edge,
 * sorted by z, cut into super-clusters of 64 and split 2x2x2 into clusters of
 * up to 8.  The outer list holds, per super-cluster, the j-clusters
 * (index >= the i-cluster's) whose bounding-box gap is below r_list = rmax +
 * skin; pruning keeps the 8x8 tiles with a pair inside rmax + prune_buffer.
 * ====================================================================== */
typedef struct pd_cluster pd_cluster;

enum pd_lj_kind {
    PD_LJ_NONE = 0,     /* no van der Waals term */
    PD_LJ_UNIFORM = 1,  /* one (c6, c12, rc2, esh) for every pair */
    PD_LJ_TABLE = 2     /* per type-pair table, ntypes <= 16 (LJ_TABLE_SHARED) */
};

#define PD_MAX_POLY 32
#define PD_MAX_TYPES 16

typedef struct {
    int n;                  /* particles */
    double rmax;            /* largest interaction cutoff */
    double skin;            /* list buffer: r_list = rmax + skin */
    double prune_buffer;    /* r_prune = rmax + prune_buffer, 0 <= prune_buffer <= skin */
    /* Lennard-Jones, pair_force() of src/clusterpairs/PairFunctor.jl:127-156:
     * f = (12 c12 ir6 - 6 c6) ir6 ir2 and e = (c12 ir6 - c6) ir6 - esh inside rc2. */
    int lj_kind;
    float lj_c6, lj_c12, lj_rc2, lj_esh;      /* PD_LJ_UNIFORM */
    int ntypes;                               /* PD_LJ_TABLE: type ids 1..ntypes */
    float lj_table[PD_MAX_TYPES * PD_MAX_TYPES * 4]; /* row-major (c6, c12, rc2, esh), lj_type_table() PairFunctor.jl:166-179 */
    /* Real-space Coulomb as CoulombPolynomial (PairFunctor.jl:21-29): inside rc2,
     * f/r = C qq (1/r^3 - P_f(x)), e = C qq (1/r + P_e(x) - eshift), x = r^2 sx - 1.
     * Monomial coefficients, constant term first (horner(), PairFunctor.jl:104-110). */
    int coulomb;
    float coul_C, coul_rc2, coul_sx, coul_eshift;
    int coul_has_mesh;
    int coul_ne, coul_nf;
    float coul_pe[PD_MAX_POLY], coul_pf[PD_MAX_POLY];
    float selfc;            /* self coefficient: the scatter subtracts 0.5*C*selfc*q^2 */
    /* fixed list intervals (nstlist, nstprune) instead of displacement triggers; 0 = triggers
     * (_decide_kernel!, src/clusterpairs/Engine.jl:301-324) */
    int nstlist, nstprune;
} pd_cluster_params;

typedef struct {
    int superclusters;      /* counts[CL_NS] */
    int outer_entries;      /* counts[CL_NE] */
    int working_entries;    /* entries of the pruned list */
    int error;              /* 0, PD_ECAPACITY or PD_ENONFINITE */
    int required;           /* outer entries needed after PD_ECAPACITY (counts[CL_REQ]) */
    int capacity;           /* outer-entry capacity (necap) */
    int builds, prunes;     /* device-decided totals (CL_NBUILD, CL_NPRUNE) */
    int nsmax, nslot;       /* super-cluster bound and slot count of this geometry */
    int last_build, last_prune; /* decision flags of the last pd_cluster_decide */
    long long tile_bits;    /* live (i-atom, j-half) tile bits of the working list */
    int mask_entries;       /* outer entries holding an exception pair (exclusion masks) */
    int outside_pairs;      /* exception pairs computed outside the tiles (counts[CL_NP]) */
} pd_cluster_stats;

/* ClusterPairEngine(T, N, box; ...) + setup! (Engine.jl:54-97, 130-139).  Copies *p. */
int pd_cluster_create(pd_cluster **out, const pd_cluster_params *p, const double box[3]);
int pd_cluster_destroy(pd_cluster *c);
/* setup!(list, box, rlist, npmax) (List.jl:874-937): size every buffer for this box and
 * request a build.  Host boundary: may reallocate (captured graphs must be recaptured). */
int pd_cluster_setup(pd_cluster *c, const double box[3]);
/* Shape of the pair kernel (no reference counterpart; the autotuner's choice): nsplit CTAs per
 * super-cluster, each splitting the super-cluster's entries, and 1, 2 or 4 warps per CTA taking
 * entries in turn.  Captured steps re-capture after a change. */
int pd_cluster_set_pair_shape(pd_cluster *c, int nsplit, int warps);
int pd_cluster_pair_shape(pd_cluster *c, int *nsplit, int *warps);
/* ensure_capacity!(list) (List.jl:959-969): after PD_ECAPACITY grow the outer-entry storage to
 * 1.5x (first growth) or 1.25x the required entries plus 1024, and request a build. */
int pd_cluster_grow(pd_cluster *c);
/* request_build!(list) (List.jl:1077): the next decision rebuilds. */
int pd_cluster_request_build(pd_cluster *c, pd_stream_t s);
/* enqueue_decide! (Engine.jl:328-335): displacement maxima since the last build/prune and the
 * device decision (build, prune) written to the handle's device flags.  fixed = 1 follows
 * nstlist/nstprune when they are set. */
int pd_cluster_decide(pd_cluster *c, const float *x, const float *y, const float *z, int fixed, pd_stream_t s);
/* build!(list, rx, ry, rz) (List.jl:979-1051) followed by the pack of the force coordinates
 * (_pack!, Engine.jl:117-127) and the first pruning pass.  q and type may be NULL.
 * conditional = 1: every kernel of the build runs only when the device build flag is set
 * (the CL_BUILD conditional graph body of ClusterBackend.jl:110-143). */
int pd_cluster_build(pd_cluster *c, const float *x, const float *y, const float *z,
                     const float *q, const int *type, int conditional, pd_stream_t s);
/* _pack! (Engine.jl:117-127): cluster-ordered force coordinates (centred image) and charges. */
int pd_cluster_pack(pd_cluster *c, const float *x, const float *y, const float *z,
                    const float *q, const int *type, pd_stream_t s);
/* enqueue_prune! (Engine.jl:353-364): distance-only pruning of the outer list to the prune
 * radius (_prune_only_kernel!, Kernels.jl:349-394) and compaction into the working list.
 * conditional = 1: only when the device prune flag is set. */
int pd_cluster_prune(pd_cluster *c, const float *x, const float *y, const float *z, int conditional, pd_stream_t s);
/* enqueue_pairs!(eng, energy, Val(false)) (Engine.jl:213-223): fused LJ + Coulomb pass over the
 * working list (_cluster_pair_kernel!, Kernels.jl:38-202) into the slot accumulators. */
int pd_cluster_pairs(pd_cluster *c, int energy, pd_stream_t s);
/* enqueue_scatter! (Engine.jl:227-257, _scatter_kernel! Kernels.jl:207-240): slot accumulators to
 * storage order, minus the Coulomb self energy, then zero the accumulators.  add = 1 adds to
 * fx/fy/fz/epot (a mesh gather in set mode ran first); vir6 is N x 6 row-major
 * (xx, yy, zz, xy, xz, yz) and is always overwritten.  q may be NULL (uncharged). */
int pd_cluster_scatter(pd_cluster *c, float *fx, float *fy, float *fz, float *epot, float *vir6,
                       const float *q, int energy, int add, pd_stream_t s);
/* compute!(eng, ...) (Engine.jl:185-190): eager update_list! + pairs + scatter.  Reads the
 * device counts on the host after a build and grows/rebuilds on overflow (not capturable). */
int pd_cluster_compute(pd_cluster *c, const float *x, const float *y, const float *z,
                       const float *q, const int *type, float *fx, float *fy, float *fz,
                       float *epot, float *vir6, int energy, pd_stream_t s);
/* Exceptions on the cluster route: Coulomb exclusions and scaled pairs, with optional bond
 * exclusions of the Lennard-Jones term.  Follows normalize_exceptions (src/electrostatics/Spec.jl:
 * 200-227), bond_exclusion_rows (src/clusterpairs/Engine.jl:274-290), the exclusion masks of
 * _exclusion_kernel! (src/clusterpairs/List.jl:634-688), the excluded branch of pair_force
 * (PairFunctor.jl:127-156) and _scaled_pairs_kernel!, _lj_restore_kernel!, _coulomb_shift_kernel!
 * (src/clusterpairs/Kernels.jl:244-339).
 *
 * (pi[k], pj[k], scale[k]): 0-based storage indices and a finite scale >= 0 (0 = excluded).  A pair
 * listed twice must carry the same scale; scale 1 is an ordinary pair and is dropped.  The pair's
 * Coulomb term becomes scale * C qi qj / r: a pair inside the list takes the excluded branch in its
 * tile (minus the mesh part, which is the whole 1/r beyond the real-space cutoff when the engine has
 * a mesh) and the scaled term is added outside the tiles; a pair beyond the list adds (scale - 1) *
 * C qi qj / r outside the tiles.
 * (bi[k], bj[k]): bonded pairs whose LJ term is dropped (the engine needs an LJ term).  The masks
 * cover the union: a bonded pair that is no Coulomb exception keeps its full Coulomb term (scale 1
 * and, energy only, the potential shift of an ordinary pair inside the cutoff); a Coulomb exception
 * that is not bonded keeps its LJ term.
 * n = nbond = 0 removes every exception.  Requests a build; captured steps re-capture.  Host
 * boundary (allocates).  Errors: PD_EINVAL with the reference's messages for out-of-range or
 * self pairs, negative or non-finite scales and conflicting duplicates. */
int pd_cluster_set_exceptions(pd_cluster *c, int n, const int *pi, const int *pj, const double *scale,
                              int nbond, const int *bi, const int *bj);
/* Allocation-free force evaluation.  This entry point has no counterpart in the reference.
 *
 * It serves callers that cannot call cudaMalloc: a plugin inside a host program whose own memory
 * pool has claimed the device memory (CUDA.jl, PyTorch's caching allocator), a host that has
 * sized its device memory to the byte and forbids further allocation, or a real-time loop that
 * must stay out of the allocator (cudaMalloc may synchronise the device).  It does the work of
 * pd_cluster_compute (build, prune, pair pass, scatter) for one small system without a handle,
 * taking every scratch buffer from one static device array of PD_STATIC_SCRATCH_BYTES that each
 * GPU loading the library holds until the process exits.  The caller passes the inputs and the
 * outputs as for pd_cluster_compute; it calls no allocating routine.
 *
 * Limits: 1 <= p->n <= PD_STATIC_MAX_N particles (larger counts return PD_EINVAL with a message);
 * PD_ECAPACITY if the outer list outgrows the array.  The first call on a device looks up the
 * array's device address (cudaGetSymbolAddress) with that device current, so make that first
 * call before any stream capture.  All calls share the array and it keeps the last call's
 * contents (the call clears what must start at zero); calls that overlap on the GPU race.
 * The call reads a device status word back at its end, so it synchronises s.  On PD_ECAPACITY or
 * PD_ENONFINITE the outputs have already been overwritten (they hold no pair forces). */
#define PD_STATIC_SCRATCH_BYTES (4u << 20)
#define PD_STATIC_MAX_N 4096
int pd_cluster_compute_static(const pd_cluster_params *p, const double box[3], const float *x, const float *y,
                              const float *z, const float *q, const int *type, float *fx, float *fy, float *fz,
                              float *epot, float *vir6, int energy, pd_stream_t s);
/* statistics(eng) (Engine.jl:402-412): host read of the device counts (synchronises s). */
int pd_cluster_status(pd_cluster *c, pd_cluster_stats *out, pd_stream_t s);
/* mesh_order(eng) (Engine.jl:394): device pointer to the particles in slot order (n entries). */
const int *pd_cluster_order(pd_cluster *c);
/* Device pointers into the list for tests: perm (nslot, -1 = padding), packed xyzq (nslot x 4),
 * outer offsets (nsmax + 1), outer entries ((cj << 8) | i-cluster mask), working entries
 * (cj, two 8-bit warp masks in bits 0-15 of the second word), working counts (nsmax). */
int pd_cluster_buffers(pd_cluster *c, const int **perm, const float **xq, const int **scio,
                       const uint32_t **cjo, const uint32_t **cjw, const int **nw);

/* ======================================================================
 * Mesh engine: ElectrostaticsSolver / MeshWorkspace (src/electrostatics/Solver.jl:17-158)
 * for SPME (B-spline window, exact deconvolution), P3M with the optimal influence
 * function for analytic (AD) or ik differentiation, and ESP (prolate split and window,
 * optimal AD influence or plain deconvolution).  cuFFT does the transforms.
 * ====================================================================== */
typedef struct pd_mesh pd_mesh;

/* influence kinds :spme, :p3m_ad, :p3m_ik, :esp, :esp_deconvolution (Spec.jl:5) */
enum pd_mesh_kind {
    PD_MESH_SPME = 1, PD_MESH_P3M_AD = 2, PD_MESH_P3M_IK = 3, PD_MESH_ESP = 4, PD_MESH_ESP_DECONV = 5
};

typedef struct {
    int kind;               /* pd_mesh_kind */
    int order;              /* window width P, 3..12: the B-spline order (BSplineWindow, Windows.jl:18-24)
                             * or the prolate window's grid points (ProlateWindow, Windows.jl:38-54) */
    int alias_order;        /* P3M alias sums |n| <= alias_order, 0..6 */
    int mesh[3];            /* K1, K2, K3 (resolve_mesh, Spec.jl:141-146) */
    double alpha;           /* Gaussian split parameter (SPME, P3M; unused by ESP) */
    double C;               /* coulomb_prefactor / relative_permittivity */
    int background;         /* net_charge = :background (Solver.jl:179-185) */
    double qtotal;          /* total charge (background term) */
    int nmax;               /* largest particle count passed to pd_mesh_transform / pd_mesh_gather */
} pd_mesh_params;

int pd_mesh_create(pd_mesh **out, const pd_mesh_params *p, const double box[3]);

/* Prolate split and window of an ESP mesh: what the reference's host setup computes in FP64
 * (ProlateSplit, Splits.jl:37-60; ProlateWindow and its device stencil, Windows.jl:38-135;
 * window_deconvolution / window_alias_table, Windows.jl:367-411).  The influence function is then
 * computed on the device with the exact quadrature of the split's transform
 * (compute_influence!, Influence.jl:190-227). */
#define PD_PROLATE_MAX_QUAD 256
#define PD_PROLATE_MAX_DEG 24
#define PD_PROLATE_MAX_NODES 8
typedef struct {
    double cutoff;          /* r_c of the split: g(k) = 4 pi c_hat(k r_c) / k^2 */
    int nquad;              /* quadrature of c_hat(u) = sum_q wchi[q] cos(u xq[q]), 1..PD_PROLATE_MAX_QUAD */
    double xq[PD_PROLATE_MAX_QUAD];    /* nodes on [0, 1] */
    double wchi[PD_PROLATE_MAX_QUAD];  /* quadrature weights times chi(xq) */
    double background_coefficient;     /* pi r_c^2 m_2 (background energy -C coef Q^2 / V) */
    int deg;                /* degree of the node polynomials, 1..PD_PROLATE_MAX_DEG */
    double poly[PD_PROLATE_MAX_DEG + 1][PD_PROLATE_MAX_NODES];  /* [k][h]: coefficient of tau^k of
                             * node h < ceil(P/2) (ProlatePolyStencil, Windows.jl:63-72) */
    const double *table[3]; /* per axis d: PD_MESH_ESP_DECONV the deconvolution 1/phi_hat^2 (K_d values);
                             * PD_MESH_ESP the alias table phi_hat(theta_m + 2 pi n), (2 alias_order + 1)
                             * values per mode m, m-major (entry m (2 alias_order + 1) + n + alias_order) */
} pd_prolate;
/* ElectrostaticsSolver(spec) for an ESP spec (p->kind PD_MESH_ESP or PD_MESH_ESP_DECONV).  Copies the
 * tables.  The gather is the AD gather with the prolate window; self-force removal is not offered. */
int pd_mesh_create_prolate(pd_mesh **out, const pd_mesh_params *p, const pd_prolate *w, const double box[3]);
int pd_mesh_destroy(pd_mesh *m);
/* refresh_geometry!(solver, box) (Solver.jl:193-209): FP64 influence function and virial
 * coefficients on the device for a new box (compute_influence!, Influence.jl:190-227). */
int pd_mesh_set_box(pd_mesh *m, const double box[3]);
/* mesh_transform!(solver, rx, ry, rz, q, energy, order) (Solver.jl:305-339): spread the n
 * particles order[0..n) (0-based ids; NULL = identity), forward R2C, influence multiply with the
 * FP64 mesh energy/virial reduction, inverse C2R (ik: three field transforms). */
int pd_mesh_transform(pd_mesh *m, const float *x, const float *y, const float *z, const float *q,
                      const int *order, int n, int energy, pd_stream_t s);
/* mesh_gather!(solver, ..., energy, order; set) (Solver.jl:360-378): reciprocal forces (and
 * energies 0.5 q phi + bg q) of the particles of order, added (set = 0) or stored (set = 1, AD
 * only); with energy, vglobal6 (device, 6 floats) receives the mesh virial plus background. */
int pd_mesh_gather(pd_mesh *m, const float *x, const float *y, const float *z, const float *q,
                   const int *order, int n, float *fx, float *fy, float *fz, float *epot,
                   float *vglobal6, int energy, int set, pd_stream_t s);
/* Host read of the FP64 accumulator acc[0..7): mesh energy and the six virial sums. */
int pd_mesh_energy(pd_mesh *m, double out7[7], pd_stream_t s);
/* Copies of the FP32 influence function (nmodes) and virial coefficients (6 x nmodes) to host
 * memory; either pointer may be NULL.  nmodes = (K1/2+1)*K2*K3. */
int pd_mesh_influence(pd_mesh *m, float *G, float *Vc);
/* Mesh dimensions and mode count. */
int pd_mesh_dims(pd_mesh *m, int mesh[3], int *nmodes);
/* Self-force removal (no counterpart in the reference; off by default, so the mesh forces stay the
 * reference's): the AD gather subtracts q_i^2 S(u_i), the force that particle i receives through the
 * mesh from its own charge, interpolated trilinearly from a table of S at table_size^3 fractional
 * grid positions.  The table comes from the mesh's own influence function and is recomputed by
 * pd_mesh_set_box.  table_size 0 turns it off; 4..64 otherwise.  Energies are unchanged.
 * PD_ENOTSUP for ik differentiation. */
int pd_mesh_set_self_force_removal(pd_mesh *m, int table_size);
/* Host copy of the table (4 floats per entry, x fastest: entry (t1 + T (t2 + T t3)) is S at grid
 * coordinates (t1, t2, t3) / T per unit charge squared) and its size T (0 when off); out4 may be NULL. */
int pd_mesh_self_force_table(pd_mesh *m, float *out4, int *table_size);

/* ======================================================================
 * Device step engine: the captured per-step graph of the reference's device engine
 * (cluster_step_parts, src/engine/ClusterBackend.jl:90-220): kick + drift (+ list decision),
 * conditional build and prune, the pair pass in parallel with the mesh transform, then the
 * gather fused with the slot scatter and the closing half kick.
 * ====================================================================== */
typedef struct pd_md pd_md;

typedef struct {
    int n;
    float *x, *y, *z;          /* positions (centred image, wrapped into [-L/2, L/2) by the drift) */
    float *vx, *vy, *vz;
    float *fx, *fy, *fz;       /* forces of the current positions */
    const float *q;            /* charges or NULL */
    const int *type;           /* type ids 1..ntypes or NULL */
    const float *inv_mass;     /* per particle 1/m (device) or NULL: use inv_mass_uniform */
    float inv_mass_uniform;
    float *epot;               /* per-particle potential energy (energy steps) */
    float *vir6;               /* per-particle pair virial, N x 6 (energy steps) */
    float *vglobal6;           /* mesh virial (energy steps), 6 floats */
} pd_md_state;

/* The engine borrows c, m (may be NULL) and the state arrays for its lifetime.  The mesh may use
 * any influence kind: SPME and P3M-AD gather with analytic derivatives, P3M-ik from its three
 * field grids. */
int pd_md_create(pd_md **out, pd_cluster *c, pd_mesh *m, const pd_md_state *st, double box[3]);
int pd_md_destroy(pd_md *md);
/* evaluate_forces_into_f!(st, energy) (src/simulation/ForceEvaluation.jl:40-44): forces (and
 * energies, virials) of the current positions; the list is kept valid (host boundary). */
int pd_md_evaluate(pd_md *md, int energy, pd_stream_t s);
/* nsteps velocity-Verlet NVE steps (NVEFusion.jl:3-27, SimulationCore.jl:581-592) with time
 * step dt; energies on the last step when energy_last = 1.  use_graph = 1 replays one captured
 * CUDA graph per step (captured on the first call); 0 launches the kernels directly. */
int pd_md_step(pd_md *md, int nsteps, float dt, int energy_last, int use_graph, pd_stream_t s);
/* Schedule of the step (no counterpart in the reference; a tuning knob of this build): the pair
 * pass, which runs beside the mesh chain, starts after the prune (pair_wait 0), after the mesh
 * chain's spread (1) or after its forward transform (2).  Later starts leave the critical mesh chain
 * more of the GPU; the forces are the same.  Captured steps are captured again after a change. */
int pd_md_set_schedule(pd_md *md, int pair_wait);
/* Steps through the C ABI with host buffers: copies x, v (pinned host, 3n floats each,
 * [x..., y..., z...]) to the device, runs nsteps, copies them back with the potential energy
 * sum (double) of the last step.  The positions are copied back on an internal stream as soon as
 * the last step's drift has written them (beside the force pass); the call returns when both
 * copies are done.  Used for end-to-end timing. */
int pd_md_step_host(pd_md *md, float *host_xyz, float *host_v, int nsteps, float dt,
                    double *epot_sum, pd_stream_t s);

/* ======================================================================
 * ELL route: cell list + fixed-capacity neighbour rows (the reference's default `CellList`
 * route for LJ / WCA, src/neighbors/DeviceNeighborCUDA.jl, src/neighbors/DenseNeighborCUDA.jl)
 * and the row pair kernels (src/engine/PairTraversal.jl:66-125, src/engine/PairModels.jl:13-49,
 * src/nonbonded/LJELLEngineKernels.jl).  2D and 3D; rows are slot-major (slot t of particle i
 * at t * n + i, _ell_index, src/neighbors/NeighborTypes.jl:31), 0-based ids.
 * ====================================================================== */
typedef struct pd_ell pd_ell;

enum { PD_PAIR_LJ = 1, PD_PAIR_WCA = 2 };

typedef struct {
    int dim;            /* 2 or 3 */
    int n;
    double cutoff;      /* interaction cutoff; the list radius is cutoff + skin */
    double skin;        /* CellList buffer (src/workflow/Forces.jl:33-42) */
    int cap;            /* row capacity (CellList capacity) */
    int interval;       /* initial rebuild interval 1..100 (CellList rebuild_interval) */
    int model;          /* PD_PAIR_LJ or PD_PAIR_WCA (UniformLJ / UniformWCA) */
    float eps, sigma;
    float rc2;          /* pair cutoff squared (WCA: 1.2599211 sigma^2, PairModels.jl:25) */
    float eshift;       /* LJ potential-shift modifier u(r_c), or 0 */
    int lanes;          /* lanes per row in the pair kernel: 1, 2, 4, 8, or 0 to choose from the density */
} pd_ell_params;

typedef struct {
    int valid, error, requested;   /* error: 0, 1 capacity (rows longer than cap), 2 coordinates */
    long long step, last_build, interval, checks, builds;
    long long required;            /* longest row of the last build attempt */
    int cap, lanes, allpairs;      /* allpairs: box below three cells per dimension, rows from all pairs */
} pd_ell_stats;

/* DeviceNeighborWorkspace(T, N, box; cutoff, skin, cap, interval) (DeviceNeighborCUDA.jl:64-88) */
int pd_ell_create(pd_ell **out, const pd_ell_params *p, const double box[3]);
int pd_ell_destroy(pd_ell *e);
/* update_device_neighbors! (DeviceNeighborCUDA.jl:420-427): displacement check and decision, then
 * the rebuild kernels, which return at once unless the device decided to rebuild.  Coordinates
 * must be centred (|x| <= L/2). */
int pd_ell_update(pd_ell *e, const float *x, const float *y, const float *z, pd_stream_t s);
/* request_device_rebuild!: invalidate the list so that the next update rebuilds it. */
int pd_ell_request(pd_ell *e, pd_stream_t s);
/* The row pair kernel: f (stored), with energy = 1 the per-particle energy (half of each pair) and
 * the per-particle half virial (3D: n x 6 xx yy zz xy xz yz; 2D: n x 3 xx yy xy).  z / fz may be
 * NULL in 2D.  No forces are written while the list is invalid. */
int pd_ell_forces(pd_ell *e, const float *x, const float *y, const float *z, float *fx, float *fy, float *fz,
                  float *epot, float *vir, int energy, pd_stream_t s);
/* device_neighbor_status (DeviceNeighborCUDA.jl:624-637): boundary readback. */
int pd_ell_status(pd_ell *e, pd_ell_stats *out);
/* Device pointers of the rows (cap * n ints) and the row lengths (n ints). */
int pd_ell_rows(pd_ell *e, int **rows, int **counts);
/* resize_capacity! + rearm_capacity_rebuild! (DeviceNeighborCUDA.jl:606-620): new row storage of
 * capacity cap, a latched capacity error cleared and a rebuild requested.  Captured graphs that
 * hold the old storage must be re-captured (the step engine does so when its key changes). */
int pd_ell_resize(pd_ell *e, int cap);

/* Step engine on the ELL route (src/engine/Run.jl:162-294, src/engine/Langevin.jl): drift with the
 * list decision fused, the flag-gated rebuild (a conditional graph node when captured), the pair
 * kernel with the closing half kick.  The state's z, vz, fz may be NULL in 2D; q, type and
 * vglobal6 are not used; vir6 holds n x 6 (3D) or n x 3 (2D) values. */
typedef struct pd_ell_md pd_ell_md;
int pd_ell_md_create(pd_ell_md **out, pd_ell *e, const pd_md_state *st);
int pd_ell_md_destroy(pd_ell_md *md);
/* evaluate_forces_into_f! on this route: decision + rebuild at the current positions, forces. */
int pd_ell_md_evaluate(pd_ell_md *md, int energy, pd_stream_t s);
/* nsteps velocity-Verlet NVE steps of size dt. */
int pd_ell_md_step(pd_ell_md *md, int nsteps, float dt, int energy_last, int use_graph, pd_stream_t s);
/* nsteps Langevin BAOAB steps (_baoa_kernel!, Langevin.jl:58-88): friction gamma, temperature kT,
 * noise from Philox4x32-10 keyed on (particle id, device step) and seed (src/engine/Philox.jl). */
int pd_ell_md_langevin(pd_ell_md *md, int nsteps, float dt, float gamma, float kT, unsigned long long seed,
                       int energy_last, int use_graph, pd_stream_t s);
/* Langevin bookkeeping (LangevinData.dq / dU / Ekin, Langevin.jl:25-35): n-float device arrays the
 * Langevin steps accumulate into -- heat exchanged with the bath (dq), work of the forces (dU, the
 * power v.f of every kick) -- and the per-particle kinetic energy after the step (ekin); all three or
 * none (NULL detaches). */
int pd_ell_md_bookkeeping(pd_ell_md *md, float *dq, float *dU, float *ekin);
/* nsteps Langevin BAOA steps (_baoa_kernel!, Langevin.jl:51-80 with kick = 2 dt): B1 with the full
 * dt, A O A, the forces, no trailing half kick. */
int pd_ell_md_baoa(pd_ell_md *md, int nsteps, float dt, float gamma, float kT, unsigned long long seed,
                   int energy_last, int use_graph, pd_stream_t s);
/* nsteps Langevin steps of the Grønbech-Jensen-Farago velocity-Verlet scheme (_gjf_pos_kernel!,
 * _gjf_vel_kernel!, Langevin.jl:164-208): positions from v, f and beta, the forces, then velocities
 * from the old and new forces and the same beta (Philox on particle id and device step). */
int pd_ell_md_gjf(pd_ell_md *md, int nsteps, float dt, float gamma, float kT, unsigned long long seed,
                  int energy_last, int use_graph, pd_stream_t s);

/* ------------------------------------------------------------------------------------------
 * Learned coarse-mesh correction (no reference counterpart: an added form compared with the
 * plain fine-mesh PME above).  PME runs on a 2x coarser mesh; a 32-128-128-1 SiLU network
 * (BF16 tensor cores, FP32 accumulation) maps each particle's local charge descriptors to a
 * scalar s_i, and the force residual is F_i = s_i V_i with
 * V_i = sum_{r_ij < rcut} q_i q_j b(r_ij) (r_i - r_j).
 * ------------------------------------------------------------------------------------------ */
#define PD_LEARNED_MAX_RADIAL 8
typedef struct pd_mlp pd_mlp;
typedef struct pd_learned pd_learned;

/* Network parameters, FP32, concatenated: w1 [128][32], b1 [128], w2 [128][128], b2 [128],
 * w3 [128], b3 [1] (pd_mlp_param_count() floats).  The tensor cores read BF16 copies of w1, w2. */
int pd_mlp_param_count(void);
int pd_mlp_create(pd_mlp **out);
int pd_mlp_destroy(pd_mlp *net);
int pd_mlp_set_params(pd_mlp *net, const float *host);   /* also clears gradients and Adam state */
int pd_mlp_get_params(pd_mlp *net, float *host);
int pd_mlp_get_grads(pd_mlp *net, float *host);
/* Inference over n rows of X (n x 32 BF16, device): s (n floats, may be NULL) and, with V4
 * (n x float4) given, corr4 (n x float4) = (s V.x, s V.y, s V.z, s). */
int pd_mlp_forward(pd_mlp *net, const void *X, int n, float *s, const float *V4, float *corr4, pd_stream_t st);
/* Fused forward + backward over n rows for the loss sum_r (s_r^2 a_r - 2 s_r b_r) scale / 2, i.e.
 * dL/ds_r = scale (s_r a_r - b_r), with ab = n x (a, b) floats; gradients are added to the
 * network's gradient buffers and the loss to its FP64 loss word. */
int pd_mlp_train(pd_mlp *net, const void *X, const float *ab, int n, float scale, pd_stream_t st);
/* Adam on the FP32 parameters with the gradients times grad_scale; clears the gradients and
 * refreshes the BF16 weight copies. */
int pd_mlp_adam(pd_mlp *net, float lr, float beta1, float beta2, float eps, float grad_scale, pd_stream_t st);
int pd_mlp_loss(pd_mlp *net, double *out, int reset);
int pd_mlp_zero_grads(pd_mlp *net, pd_stream_t st);
/* 1 after a tensor-core wait that timed out (latched). */
int pd_mlp_error(pd_mlp *net, int *out);

typedef struct {
    float rcut;                 /* descriptor / residual cutoff (6 A) */
    float skin;                 /* neighbour-row skin */
    int cap;                    /* row capacity */
    float mu0, dmu, sigma;      /* feature Gaussians: centres mu0 + k dmu (k < 16), width sigma */
    int nb;                     /* radial terms of b(r), 1..PD_LEARNED_MAX_RADIAL */
    float nu0, dnu, tau;        /* their centres nu0 + m dnu and width tau */
    float coef[PD_LEARNED_MAX_RADIAL];   /* b(r) = fc(r) sum_m coef[m] exp(-(r - nu_m)^2 / (2 tau^2)) */
} pd_learned_params;

int pd_learned_create(pd_learned **out, const pd_learned_params *p, int n, const double box[3]);
int pd_learned_destroy(pd_learned *h);
int pd_learned_set_radial(pd_learned *h, const float *coef, int nb);
/* Row update (own displacement decision) and descriptors at centred coordinates: X (n x 32 BF16),
 * species 0 = type id 1, species 1 = every other id (1-based type ids; type may be NULL),
 * V4 (n x float4); NULL selects the handle's buffers.  With Vb4 (nb x n x float4) the radial-term
 * vectors V_i^(m) are written instead of V. */
int pd_learned_descriptors(pd_learned *h, const float *x, const float *y, const float *z, const float *q,
                           const int *type, void *X, float *V4, float *Vb4, pd_stream_t st);
/* Descriptors + network: corr4 (n x float4, NULL: the handle's buffer) = (s V, s). */
int pd_learned_correction(pd_learned *h, pd_mlp *net, const float *x, const float *y, const float *z, const float *q,
                          const int *type, float *corr4, pd_stream_t st);
int pd_learned_buffers(pd_learned *h, void **X, float **V4, float **corr4);
int pd_learned_status(pd_learned *h, pd_ell_stats *out);
int pd_learned_resize(pd_learned *h, int cap);
/* Attach (or with NULL detach) the correction to a step engine: every force pass then adds
 * corr = s V to the forces before the closing kick (the descriptors and the network run on a
 * third stream beside the pair pass and the mesh).  net = NULL attaches the radial term alone
 * (corr = V, s = 1: the descriptors run, the network does not). */
int pd_md_set_learned(pd_md *md, pd_learned *h, pd_mlp *net);

/* ------------------------------------------------------------------------------------------
 * Batched replicas (no reference counterpart: the reference steps one system per engine).
 * Hundreds of independent 3D LJ / WCA systems of uneven size, each with its own cubic or
 * orthorhombic box and pair model, concatenated (replica r owns the particles after those of
 * replicas 0..r-1) and stepped together: one launch per stage over all replicas, the NVE step
 * captured into one CUDA graph.  Rows follow the ELL route (radius max r_c + skin, one rebuild
 * decision for the whole batch).
 * ------------------------------------------------------------------------------------------ */
typedef struct pd_batch pd_batch;
typedef struct {
    double box[3];          /* each length above twice the list radius */
    int n;                  /* particles */
    int kind;               /* PD_PAIR_LJ or PD_PAIR_WCA (UniformLJ / UniformWCA, PairModels.jl:13-49) */
    float eps, sigma, rc2;  /* rc2: squared cutoff (WCA: 1.2599211 sigma^2) */
    float eshift;           /* LJ energy shift at the cutoff (0 unshifted); WCA adds eps */
} pd_batch_replica;

int pd_batch_create(pd_batch **out, const pd_batch_replica *reps, int nrep, float skin, int cap, int lanes);
int pd_batch_destroy(pd_batch *b);
int pd_batch_count(pd_batch *b, int *n, int *ncell);
/* Lanes per row of the pair kernel (1, 2, 4, 8), the autotuner's choice. */
int pd_batch_set_lanes(pd_batch *b, int lanes);
/* Displacement decision and the flag-gated rebuild at centred coordinates (all replicas). */
int pd_batch_update(pd_batch *b, const float *x, const float *y, const float *z, pd_stream_t st);
/* Forces (stored) and, with energy, the per-particle energy (half of each pair). */
int pd_batch_forces(pd_batch *b, const float *x, const float *y, const float *z, float *fx, float *fy, float *fz,
                    float *epot, int energy, pd_stream_t st);
int pd_batch_status(pd_batch *b, pd_ell_stats *out);
/* Device pointers of the rows (cap x n ints, slot t of the particle at cell-order position k at
 * t * n + k, entries are cell-order positions), their lengths (n, by position) and the cell order
 * (n particle indices). */
int pd_batch_rows(pd_batch *b, int **rows, int **counts, int **order);

/* Charged replicas (the batched ionic melts): every replica's real-space Coulomb term is the
 * cluster route's fitted polynomial of the Gaussian split (pair_force, PairFunctor.jl:127-156:
 * f/r = C qq (r^-3 - P_f(x)), e = C qq (1/r + P_e(x) - eshift), x = r^2 sx - 1, inside rc2), and
 * selfc = 2 alpha / sqrt(pi) gives the per-particle self energy -C selfc q^2 / 2.  The charges come
 * from the bound state (pd_md_state.q).  rc2 must lie inside the list radius of the batch. */
typedef struct {
    float C, rc2, sx, eshift;
    int ne, nf;                     /* coefficients (<= 16 each), constant term first */
    float pe[PD_MAX_POLY], pf[PD_MAX_POLY];
    float selfc;
} pd_batch_coulomb;
int pd_batch_set_coulomb(pd_batch *b, const pd_batch_coulomb *c);
/* One SPME or P3M-AD mesh per replica (meshes: nrep x (K1, K2, K3), the replica's own box at the
 * shared spacing), B-spline order 4..6, with its FP64 influence function from the single-system
 * setup (compute_influence!, Influence.jl:190-227).  The replicas' meshes are transformed by one
 * batched cuFFT plan per mesh size; spread, influence multiply and gather are one launch each over
 * all replicas.  Neutral replicas only (net_charge = :error).  Host boundary: allocates. */
int pd_batch_set_mesh(pd_batch *b, int kind, int order, double alpha, double C, const int *meshes);
/* Spread tile of the batched meshes, the autotuner's choice: 32 or 64 particles (cell-order
 * neighbours of one replica) per spread / gather CTA, with 2 threads per ion sharing its stencil's
 * z planes, or 4 (tiles of 64).  Host boundary: may reallocate. */
int pd_batch_set_spread_tile(pd_batch *b, int chunk, int threads_per_ion);
/* Batched-mesh sizes: FFT plan groups (mesh sizes), grid nodes and modes of all replicas, the tile
 * size and the number of tiles. */
int pd_batch_mesh_info(pd_batch *b, int *groups, long long *nodes, long long *modes, int *chunk, int *nchunk);
/* Step state (x, v, f, per-particle inverse masses, optional epot) of all replicas, concatenated. */
int pd_batch_bind(pd_batch *b, const pd_md_state *st);
int pd_batch_evaluate(pd_batch *b, int energy, pd_stream_t st);
/* nsteps velocity-Verlet NVE steps: drift (+ decision), IF rebuild, pairs (+ closing half kick). */
int pd_batch_step(pd_batch *b, int nsteps, float dt, int use_graph, pd_stream_t st);

/* FP64 Ewald sum on the GPU (ewald_reference, test/ewald_reference.jl:50-127, restated): rq4 =
 * n x (x, y, z, q) doubles on the device; real space over minimum images within x / alpha
 * (must be below half the smallest box length), reciprocal space within |k| < 2 alpha x,
 * x = sqrt(digits ln 10); parts: 1 real space, 2 reciprocal space, 4 self energy.  F (n x 3
 * doubles, device) is overwritten; E (host, may be NULL) receives the energy. */
int pd_ewald_oracle(int n, const double *rq4, const double box[3], double C, double alpha, double digits, int parts,
                    double *F, double *E);

/* ======================================================================
 * Snapshot I/O: the GSD file layer (version 2.0) that the reference's trajectory writer and
 * restart reader drive through GSDFiles.jl (src/io/GSDIO.jl:104-203, 380-615,
 * src/io/RestartIO.jl:20-511), and a device kernel that packs one frame's per-particle chunks
 * for a single device-to-host copy.  These calls are host file I/O: they take HOST buffers and
 * are not stream-ordered (pd_snapshot_pack is the exception).
 * ====================================================================== */
typedef struct pd_gsd pd_gsd;

/* GSD type codes (RestartIO.jl:27-39) */
enum pd_gsd_type {
    PD_GSD_UINT8 = 1, PD_GSD_UINT16 = 2, PD_GSD_UINT32 = 3, PD_GSD_UINT64 = 4, PD_GSD_INT8 = 5,
    PD_GSD_INT16 = 6, PD_GSD_INT32 = 7, PD_GSD_INT64 = 8, PD_GSD_FLOAT = 9, PD_GSD_DOUBLE = 10,
    PD_GSD_CHARACTER = 11
};
enum pd_gsd_mode { PD_GSD_CREATE = 0, PD_GSD_APPEND = 1, PD_GSD_READ = 2 };

/* One index entry as stored in the file (32 bytes). */
typedef struct {
    uint64_t frame;
    uint64_t N;
    int64_t location;
    uint32_t M;
    uint16_t id;
    uint8_t type;
    uint8_t flags;
} pd_gsd_index_entry;

/* gsd_open(path; application, schema, schema_version, append) (GSDIO.jl:167-175, 140-165):
 * PD_GSD_CREATE truncates or creates the file and writes an empty version-2.0 layout;
 * PD_GSD_APPEND continues an existing file after its last committed frame; PD_GSD_READ reads.
 * schema_version = (major << 16) | minor (HOOMD schema 1.4: 0x00010004).  An invalid magic or a
 * truncated file returns PD_EINVAL (the reference's "Invalid GSD magic", GSDIO.jl:113). */
int pd_gsd_open(const char *path, int mode, const char *application, const char *schema, uint32_t schema_version,
                pd_gsd **out);
/* gsd_close(h) (GSDIO.jl:203).  Chunks written after the last pd_gsd_end_frame are dropped. */
int pd_gsd_close(pd_gsd *h);
/* write_chunk(name; type, N, M, data) (GSDFiles' write_chunk_raw!, GSDIO.jl:307-310): N x M values
 * of `type`, row-major, from host memory, into the frame being written.  A name appears at most
 * once per frame. */
int pd_gsd_write_chunk(pd_gsd *h, const char *name, int type, uint64_t N, uint32_t M, const void *data);
/* end_frame!(h) (GSDIO.jl:599): commits the frame (index entries, new names, header). */
int pd_gsd_end_frame(pd_gsd *h);
/* sync!(h) (GSDIO.jl:600-610): fsync of the file. */
int pd_gsd_flush(pd_gsd *h);
/* nframes(reader) (test/test_io_gsd.jl:90): committed frames. */
uint64_t pd_gsd_nframes(const pd_gsd *h);
/* Header fields: file layer and schema versions, application and schema names (64-byte buffers). */
int pd_gsd_header(const pd_gsd *h, uint32_t *gsd_version, uint32_t *schema_version, char *application,
                  char *schema);
/* _maybe_one(r, entries_for_frame(frame), name) (RestartIO.jl:141-149): *found = 1 and the entry
 * when `frame` holds a chunk `name`, else *found = 0. */
int pd_gsd_find_chunk(const pd_gsd *h, uint64_t frame, const char *name, pd_gsd_index_entry *out, int *found);
/* read_chunk(entry) (RestartIO.jl:41-52): the entry's N x M values into a host buffer of `bytes`. */
int pd_gsd_read_chunk(const pd_gsd *h, const pd_gsd_index_entry *e, void *buf, uint64_t bytes);
/* _entries_for_frame(r, frame) (RestartIO.jl:141): the frame's entries (up to cap); *count = all. */
int pd_gsd_frame_entries(const pd_gsd *h, uint64_t frame, pd_gsd_index_entry *out, int cap, int *count);
/* r.names[id + 1] (RestartIO.jl:227): the name of chunk id into buf (size bytes). */
int pd_gsd_name(const pd_gsd *h, int id, char *buf, int size);

/* One frame's per-particle device arrays (structure of arrays, build order).  z, vz, fz are NULL
 * in 2D; velocities, forces, types and virial rows are optional (NULL = chunk absent).  `type`
 * holds 1-based type ids; `vir` is n x 6 (3D: xx, yy, zz, xy, xz, yz) or n x 3 (2D: xx, yy, xy),
 * row-major. */
typedef struct {
    int n;
    int dim;
    const float *x, *y, *z;
    const float *vx, *vy, *vz;
    const float *fx, *fy, *fz;
    const int *type;
    const float *vir;
} pd_snapshot_src;

/* Byte offsets of the packed chunks inside the staging buffer (~0 = absent), each 16-byte
 * aligned: particles/position (float32 n x 3), particles/velocity (n x 3), particles/force
 * (n x 3), particles/typeid (uint32 n, 0-based), particles/virial (float32 n x virial_columns). */
typedef struct {
    uint64_t position, velocity, force, typeid_, virial;
    int virial_columns;
    uint64_t bytes;
} pd_snapshot_offsets;
int pd_snapshot_layout(const pd_snapshot_src *src, pd_snapshot_offsets *out);
/* Packs the frame into the device buffer dst (16-byte aligned, dst_bytes >= layout.bytes) on
 * stream s, in the chunks' on-disk layout (_soa_to_posmat / _soa_to_velmat / _soa_to_frcmat and
 * the 0-based type ids of GSDIO.jl:228-299, 451-454).  Stream-ordered, allocates nothing. */
int pd_snapshot_pack(const pd_snapshot_src *src, void *dst, uint64_t dst_bytes, pd_stream_t s);

#ifdef __cplusplus
}
#endif
#endif /* PDB200_H */
