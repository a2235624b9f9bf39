// Allocation-free cluster-pair force evaluation (pd_cluster_compute_static).
//
// Some callers cannot call cudaMalloc: a host that has already sized its
// device memory pool to the byte and forbids further allocation, a caller in
// the middle of building a CUDA graph region, or a real-time loop that must
// not enter the allocator.  For them this file keeps one file-scope device
// arena and runs the ordinary build -> prune -> pair -> scatter sequence of
// the cluster-pair engine with every scratch buffer carved out of it.
//
// Properties of the arena (PD_STATIC_SCRATCH_BYTES, 4 MiB): it exists on every
// GPU that loads libpdb200 until the process exits; all calls share it and it
// keeps the contents of the last call, so every buffer that must start at
// zero is cleared by the call itself; two calls whose work overlaps on the GPU
// (different streams, or different host threads) race on it.  The host needs
// the arena's device address, which it obtains once per device with
// cudaGetSymbolAddress on the first call made while that device is current;
// make that first call before any stream capture begins.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>

#include "common.cuh"
#include "internal.hpp"

using namespace pdb;

namespace {

constexpr size_t kArenaBytes = PD_STATIC_SCRATCH_BYTES;
static __device__ __align__(256) unsigned char g_arena[kArenaBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void *g_arena_ptr[kMaxDevices] = {nullptr};

// Device address of g_arena for the current device (set-up on the first call per device).
int arena_address(void **out) {
    int dev = 0;
    PD_CUDA(cudaGetDevice(&dev));
    PD_CHECK(dev >= 0 && dev < kMaxDevices, PD_EINVAL, "device index %d out of range", dev);
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_arena_ptr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_arena);
        PD_CHECK(e == cudaSuccess && p, PD_ECUDA, "cudaGetSymbolAddress of the static scratch failed: %s",
                 cudaGetErrorString(e));
        g_arena_ptr[dev] = p;
    }
    *out = g_arena_ptr[dev];
    return PD_OK;
}

// Bump allocator over the arena (256-byte aligned pieces).
struct Carver {
    unsigned char *base;
    size_t used = 0;
    bool ok = true;
    template <typename T>
    T *take(size_t count) {
        const size_t bytes = ((std::max<size_t>(count, 1) * sizeof(T)) + 255) & ~size_t(255);
        if (used + bytes > kArenaBytes) {
            ok = false;
            return nullptr;
        }
        T *p = reinterpret_cast<T *>(base + used);
        used += bytes;
        return p;
    }
};

}  // namespace

extern "C" int pd_cluster_compute_static(const pd_cluster_params *p, const double box[3], const float *x,
                                         const float *y, const float *z, const float *q, const int *type, float *fx,
                                         float *fy, float *fz, float *epot, float *vir6, int energy, pd_stream_t sp) {
    PD_CHECK(p && box && x && y && z && fx && fy && fz, PD_EINVAL, "pd_cluster_compute_static: null argument");
    PD_CHECK(!energy || epot, PD_EINVAL, "pd_cluster_compute_static: energy needs epot");
    PD_CHECK(p->n >= 1 && p->n <= PD_STATIC_MAX_N, PD_EINVAL,
             "pd_cluster_compute_static: %d particles; the static scratch serves 1..%d", p->n, PD_STATIC_MAX_N);
    PD_CHECK(p->skin >= 0 && p->prune_buffer >= 0 && p->prune_buffer <= p->skin && p->rmax > 0, PD_EINVAL,
             "pd_cluster_compute_static: need rmax > 0 and 0 <= prune_buffer <= skin");
    PD_CHECK(p->lj_kind >= PD_LJ_NONE && p->lj_kind <= PD_LJ_TABLE, PD_EINVAL, "unknown LJ kind %d", p->lj_kind);
    PD_CHECK(p->lj_kind != PD_LJ_TABLE || (p->ntypes >= 1 && p->ntypes <= PD_MAX_TYPES), PD_EINVAL,
             "LJ type table needs 1 <= ntypes <= %d", PD_MAX_TYPES);
    PD_CHECK(!p->coulomb || (p->coul_ne >= 1 && p->coul_ne <= PD_MAX_POLY && p->coul_nf >= 1 &&
                             p->coul_nf <= PD_MAX_POLY),
             PD_EINVAL, "Coulomb polynomial needs 1..%d coefficients", PD_MAX_POLY);
    cudaStream_t s = (cudaStream_t)sp;

    // geometry of this box (the setup! rules, without allocation)
    pd_cluster c;
    c.p = *p;
    c.n = p->n;
    const int N = p->n;
    const double rlist = p->rmax + p->skin;
    const double Lx = (float)box[0], Ly = (float)box[1], Lz = (float)box[2];
    PD_CHECK(std::isfinite(Lx) && std::isfinite(Ly) && std::isfinite(Lz) && Lx > 0 && Ly > 0 && Lz > 0, PD_EINVAL,
             "box lengths must be finite and positive");
    PD_CHECK(std::min(Lx, std::min(Ly, Lz)) > 2 * rlist, PD_EINVAL,
             "cluster-pair list radius %g needs every box length above %g.", rlist, 2 * rlist);
    const double rho = N / (Lx * Ly * Lz);
    const double b = std::cbrt(SUPER / rho);
    c.ncx = std::max(1, (int)std::floor(Lx / b));
    c.ncy = std::max(1, (int)std::floor(Ly / b));
    c.ncol = c.ncx * c.ncy;
    c.nzb = std::max(1, (int)std::nearbyint(Lz * rho * (Lx / c.ncx) * (Ly / c.ncy) / 4));
    const long long nbin = (long long)c.ncol * c.nzb;
    PD_CHECK(nbin <= 4LL * PD_STATIC_MAX_N, PD_EINVAL, "pd_cluster_compute_static: %lld z-bins exceed the static "
             "scratch", nbin);
    c.nbin = (int)nbin;
    c.nsmax = (N + SUPER - 1) / SUPER + c.ncol;
    c.nslot = SUPER * c.nsmax;
    c.mx = (int)std::floor(rlist / (0.98 * Lx / c.ncx)) + 1;
    c.my = (int)std::floor(rlist / (0.98 * Ly / c.ncy)) + 1;
    c.ncs = std::min(2 * c.mx + 1, c.ncx) * std::min(2 * c.my + 1, c.ncy);
    PD_CHECK(c.ncs <= SEARCH_MAX_COLS, PD_EINVAL, "pd_cluster_compute_static: %d search columns exceed %d", c.ncs,
             SEARCH_MAX_COLS);
    for (int d = 0; d < 3; ++d) {
        c.box[d] = box[d];
        c.L[d] = (float)box[d];
    }
    c.rlist = rlist;
    int dev = 0;
    PD_CUDA(cudaGetDevice(&dev));
    PD_CUDA(cudaDeviceGetAttribute(&c.num_sms, cudaDevAttrMultiProcessorCount, dev));
    c.nsplit = std::max(1, std::min(32, (32 * c.num_sms + c.nsmax - 1) / std::max(c.nsmax, 1)));
    PairParams &pp = c.pp;
    memset(&pp, 0, sizeof pp);
    pp.Lx = c.L[0];
    pp.Ly = c.L[1];
    pp.Lz = c.L[2];
    pp.lj_kind = p->lj_kind;
    pp.c6 = p->lj_c6;
    pp.c12 = p->lj_c12;
    pp.lrc2 = p->lj_rc2;
    pp.esh = p->lj_esh;
    pp.ntypes = p->lj_kind == PD_LJ_TABLE ? p->ntypes : 1;
    pp.coulomb = p->coulomb;
    pp.C = p->coul_C;
    pp.rc2 = p->coul_rc2;
    pp.sx = p->coul_sx;
    pp.eshift = p->coul_eshift;
    pp.ne = p->coulomb ? p->coul_ne : 1;
    pp.nf = p->coulomb ? p->coul_nf : 1;
    for (int k = 0; k < PD_MAX_POLY; ++k) {   // coefficients past the fitted length are zero (exact padding)
        pp.pe[k] = k < pp.ne ? p->coul_pe[k] : 0.f;
        pp.pf[k] = k < pp.nf ? p->coul_pf[k] : 0.f;
    }

    // carve every buffer of the list out of the arena
    void *base = nullptr;
    int rc = arena_address(&base);
    if (rc) return rc;
    Carver cv{reinterpret_cast<unsigned char *>(base)};
    c.counts = cv.take<int>(W_LEN);
    c.bin = cv.take<int>(N);
    c.bcnt = cv.take<int>(c.nbin);
    c.bstart = cv.take<int>(c.nbin + 1);
    c.cursor = cv.take<int>(c.nbin);
    c.sorted = cv.take<int>(N);
    c.col_sc_off = cv.take<int>(c.ncol + 1);
    c.sc_first = cv.take<int>(c.nsmax);
    c.sc_n = cv.take<int>(c.nsmax);
    c.sc_col = cv.take<int>(c.nsmax);
    c.perm = cv.take<int>(c.nslot);
    c.slot_of = cv.take<int>(N);
    c.order = cv.take<int>(N);
    c.xq = cv.take<float4>(c.nslot);
    c.ts = cv.take<int>(c.nslot);
    c.cbc = cv.take<float4>(8 * (size_t)c.nsmax);
    c.cbh = cv.take<float4>(8 * (size_t)c.nsmax);
    c.sbc = cv.take<float4>(c.nsmax);
    c.sbh = cv.take<float4>(c.nsmax);
    c.cnt_sc = cv.take<int>(c.nsmax);
    c.colcnt = cv.take<int>((size_t)c.nsmax * c.ncs);
    c.scio = cv.take<int>(c.nsmax + 1);
    c.nw = cv.take<int>(c.nsmax);
    c.fc = cv.take<float4>(c.nslot);
    c.vc = cv.take<float>(6 * (size_t)c.nslot);
    c.ref_build = cv.take<float4>(N);
    c.ref_prune = cv.take<float4>(N);
    c.lj_table = cv.take<float>(PD_MAX_TYPES * PD_MAX_TYPES * 4);
    PD_CHECK(cv.ok, PD_EINVAL, "pd_cluster_compute_static: the list of %d particles exceeds the static scratch", N);
    // what remains holds the outer and working entries (4 + 8 bytes each)
    const size_t left = kArenaBytes - cv.used;
    const size_t necap = left > 1024 ? (left - 1024) / (sizeof(uint32_t) + sizeof(uint2)) : 0;
    PD_CHECK(necap >= 64, PD_EINVAL, "pd_cluster_compute_static: no room left for list entries");
    c.necap = (int)std::min<size_t>(necap, 1u << 30);
    c.cjo = cv.take<uint32_t>(c.necap);
    c.cjw = cv.take<uint2>(c.necap);
    PD_CHECK(cv.ok, PD_EINVAL, "pd_cluster_compute_static: entry storage exceeds the static scratch");

    // the arena keeps the previous call's contents: clear what must start at zero
    PD_CUDA(cudaMemsetAsync(c.counts, 0, W_LEN * sizeof(int), s));
    PD_CUDA(cudaMemsetAsync(c.bcnt, 0, sizeof(int) * (size_t)c.nbin, s));
    PD_CUDA(cudaMemsetAsync(c.fc, 0, sizeof(float4) * (size_t)c.nslot, s));
    PD_CUDA(cudaMemsetAsync(c.vc, 0, sizeof(float) * 6 * (size_t)c.nslot, s));
    PD_CUDA(cudaMemsetAsync(c.nw, 0, sizeof(int) * (size_t)c.nsmax, s));
    PD_CUDA(cudaMemsetAsync(c.scio, 0, sizeof(int) * ((size_t)c.nsmax + 1), s));
    if (p->lj_kind == PD_LJ_TABLE)
        PD_CUDA(cudaMemcpyAsync(c.lj_table, p->lj_table, sizeof(p->lj_table), cudaMemcpyHostToDevice, s));

    if ((rc = cluster_build_launch(&c, x, y, z, p->coulomb ? q : nullptr, type, 0, s))) return rc;
    if ((rc = cluster_set_word(&c, W_PRUNE, 1, s))) return rc;
    if ((rc = cluster_prune_launch(&c, 1, s))) return rc;
    if ((rc = cluster_pairs_launch(&c, energy, s))) return rc;
    if ((rc = pd_cluster_scatter(&c, fx, fy, fz, epot, vir6, q, energy, 0, sp))) return rc;
    // report list failures (a device word read back; no allocation)
    int h[W_LEN];
    if ((rc = cluster_read_counts(&c, h, s))) return rc;
    PD_CHECK(h[W_ERR] != PD_ENONFINITE, PD_ENONFINITE, "Cluster-pair list: non-finite coordinates");
    PD_CHECK(h[W_ERR] != PD_ECAPACITY, PD_ECAPACITY,
             "pd_cluster_compute_static: %d outer entries exceed the %d the static scratch holds", h[W_REQ], c.necap);
    return PD_OK;
}
