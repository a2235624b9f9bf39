// Allocation-free cluster-pair force evaluation (pd_cluster_compute_static).
//
// Some callers cannot call cudaMalloc: a plugin inside a host program whose
// own memory pool has already claimed the device memory (a Julia CUDA.jl
// session, a PyTorch process with its caching allocator), so that a direct
// cudaMalloc fails or escapes the pool's accounting; a host that has sized
// its device memory to the byte and forbids further allocation; or a
// real-time loop that must not enter the allocator, because cudaMalloc can
// synchronise the device and take unbounded time.  For them this file keeps
// one file-scope device arena and runs the ordinary build -> prune -> pair ->
// scatter sequence of the cluster-pair engine with every scratch buffer carved
// out of it.
//
// Properties of the arena (PD_STATIC_SCRATCH_BYTES, 4 MiB): it exists on every
// GPU that loads libpdb200 until the process exits; all calls share it and it
// keeps the contents of the last call, so every buffer that must start at
// zero is cleared by the call itself; two calls whose work overlaps on the GPU
// (different streams, or different host threads) race on it.  The host needs
// the arena's device address, which it obtains once per device with
// cudaGetSymbolAddress on the first call made while that device is current;
// make that first call before any stream capture begins.  The call reads the
// list's status word back at its end, so it synchronises its stream.  On a list
// failure (PD_ECAPACITY, PD_ENONFINITE) the outputs have already been
// overwritten with the empty pair pass's result (no pair forces) when the error
// is returned.
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
    int rc = cluster_check_params(p);
    if (rc) return rc;
    PD_CHECK(p->n <= PD_STATIC_MAX_N, PD_EINVAL,
             "pd_cluster_compute_static: %d particles; the static scratch serves 1..%d", p->n, PD_STATIC_MAX_N);
    cudaStream_t s = (cudaStream_t)sp;

    // geometry of this box: the rules pd_cluster_setup applies, without its allocations
    pd_cluster c;
    c.p = *p;
    c.n = p->n;
    const int N = p->n;
    ClusterGeom g;
    if ((rc = cluster_geometry(N, p->rmax + p->skin, box, &g))) return rc;
    PD_CHECK(g.nbin <= 4LL * PD_STATIC_MAX_N, PD_EINVAL, "pd_cluster_compute_static: %lld z-bins exceed the static "
             "scratch", g.nbin);
    c.ncx = g.ncx;
    c.ncy = g.ncy;
    c.ncol = g.ncol;
    c.nzb = g.nzb;
    c.nbin = (int)g.nbin;
    c.nsmax = g.nsmax;
    c.nslot = g.nslot;
    c.mx = g.mx;
    c.my = g.my;
    c.ncs = g.ncs;
    c.rlist = g.rlist;
    for (int d = 0; d < 3; ++d) {
        c.box[d] = box[d];
        c.L[d] = (float)box[d];
    }
    int dev = 0;
    PD_CUDA(cudaGetDevice(&dev));
    PD_CUDA(cudaDeviceGetAttribute(&c.num_sms, cudaDevAttrMultiProcessorCount, dev));
    c.nsplit = std::max(1, std::min(32, (32 * c.num_sms + c.nsmax - 1) / std::max(c.nsmax, 1)));
    cluster_pair_params(p, box, &c.pp);

    // carve every buffer of the list out of the arena
    void *base = nullptr;
    if ((rc = arena_address(&base))) return rc;
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
