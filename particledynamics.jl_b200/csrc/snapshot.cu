// Device side of the snapshot I/O path: one kernel packs a frame's per-particle chunks in the GSD
// on-disk layout (row-major N x 3 positions, velocities and forces with z = 0 in 2D, 0-based uint32
// type ids, N x 6 or N x 3 virial rows) into one staging buffer, so that a frame leaves the GPU as one
// copy instead of one copy and one synchronisation per array.
//
// The reference gathers each structure-of-arrays component to the host separately, synchronises
// after each, and interleaves on the host (src/io/GSDIO.jl:228-299, the _soa_to_*mat helpers), and
// converts the 1-based type ids to 0-based ones there (GSDIO.jl:451-454).  The particle arrays of
// this library stay in build order (no spatial reordering of the caller's storage), so the
// reference's _unpermuted step (GSDIO.jl:209-220) has nothing to undo here.
#include <algorithm>

#include "common.cuh"
#include "internal.hpp"

namespace {

constexpr uint64_t kAbsent = ~0ull;

// Section offsets in 4-byte words, each section starting on a 16-byte boundary.
struct Words {
    uint64_t pos, vel, frc, tid, vir, total;
    int vrow;
};

inline uint64_t up4(uint64_t w) { return (w + 3) & ~3ull; }

Words layout_words(const pd_snapshot_src &s) {
    Words w{};
    const uint64_t n = (uint64_t)s.n;
    w.vrow = s.dim == 3 ? 6 : 3;
    uint64_t o = 0;
    w.pos = o;
    o = up4(o + 3 * n);
    w.vel = s.vx ? o : kAbsent;
    if (s.vx) o = up4(o + 3 * n);
    w.frc = s.fx ? o : kAbsent;
    if (s.fx) o = up4(o + 3 * n);
    w.tid = s.type ? o : kAbsent;
    if (s.type) o = up4(o + n);
    w.vir = s.vir ? o : kAbsent;
    if (s.vir) o = up4(o + (uint64_t)w.vrow * n);
    w.total = o;
    return w;
}

struct PackArgs {
    const float *x, *y, *z, *vx, *vy, *vz, *fx, *fy, *fz, *vir;
    const int *type;
    uint32_t *dst;
    uint64_t n, pos, vel, frc, tid, vir_at, total;
    int vrow;
};

__device__ __forceinline__ float comp3(const float *a, const float *b, const float *c, uint64_t p, uint64_t k) {
    return k == 0 ? __ldg(a + p) : (k == 1 ? __ldg(b + p) : (c ? __ldg(c + p) : 0.f));
}

// One thread per output word, grid-stride: every store of a warp is contiguous, and each word is
// read once from its source array.
__global__ void __launch_bounds__(256) k_snapshot_pack(PackArgs a) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < a.total; e += stride) {
        uint32_t word = 0;
        if (e < a.pos + 3 * a.n) {
            const uint64_t r = e - a.pos;
            word = __float_as_uint(comp3(a.x, a.y, a.z, r / 3, r % 3));
        } else if (a.vel != kAbsent && e >= a.vel && e < a.vel + 3 * a.n) {
            const uint64_t r = e - a.vel;
            word = __float_as_uint(comp3(a.vx, a.vy, a.vz, r / 3, r % 3));
        } else if (a.frc != kAbsent && e >= a.frc && e < a.frc + 3 * a.n) {
            const uint64_t r = e - a.frc;
            word = __float_as_uint(comp3(a.fx, a.fy, a.fz, r / 3, r % 3));
        } else if (a.tid != kAbsent && e >= a.tid && e < a.tid + a.n) {
            word = (uint32_t)(__ldg(a.type + (e - a.tid)) - 1);
        } else if (a.vir_at != kAbsent && e >= a.vir_at && e < a.vir_at + (uint64_t)a.vrow * a.n) {
            word = __float_as_uint(__ldg(a.vir + (e - a.vir_at)));
        }
        a.dst[e] = word;   // alignment padding between sections is written as zero
    }
}

int check_src(const pd_snapshot_src *s, const char *where) {
    PD_CHECK(s, PD_EINVAL, "%s: null source", where);
    PD_CHECK(s->n >= 0, PD_EINVAL, "%s: negative particle count", where);
    PD_CHECK(s->dim == 2 || s->dim == 3, PD_EINVAL, "%s: dim must be 2 or 3, got %d", where, s->dim);
    PD_CHECK(s->n == 0 || (s->x && s->y && (s->dim == 2 || s->z)), PD_EINVAL, "%s: positions are required", where);
    PD_CHECK(!s->vx || (s->vy && (s->dim == 2 || s->vz)), PD_EINVAL, "%s: velocities need every component", where);
    PD_CHECK(!s->fx || (s->fy && (s->dim == 2 || s->fz)), PD_EINVAL, "%s: forces need every component", where);
    return PD_OK;
}

}  // namespace

extern "C" {

int pd_snapshot_layout(const pd_snapshot_src *s, pd_snapshot_offsets *out) {
    int rc = check_src(s, "pd_snapshot_layout");
    if (rc != PD_OK) return rc;
    PD_CHECK(out, PD_EINVAL, "pd_snapshot_layout: null output");
    const Words w = layout_words(*s);
    auto bytes = [](uint64_t o) { return o == kAbsent ? kAbsent : 4 * o; };
    out->position = bytes(w.pos);
    out->velocity = bytes(w.vel);
    out->force = bytes(w.frc);
    out->typeid_ = bytes(w.tid);
    out->virial = bytes(w.vir);
    out->virial_columns = w.vrow;
    out->bytes = 4 * w.total;
    return PD_OK;
}

int pd_snapshot_pack(const pd_snapshot_src *s, void *dst, uint64_t dst_bytes, pd_stream_t stream) {
    int rc = check_src(s, "pd_snapshot_pack");
    if (rc != PD_OK) return rc;
    const Words w = layout_words(*s);
    PD_CHECK(dst_bytes >= 4 * w.total, PD_EINVAL, "pd_snapshot_pack: the staging buffer holds %llu bytes, the frame "
             "needs %llu", (unsigned long long)dst_bytes, (unsigned long long)(4 * w.total));
    PD_CHECK(dst && ((uintptr_t)dst & 15) == 0, PD_EINVAL, "pd_snapshot_pack: the staging buffer must be 16-byte "
             "aligned device memory");
    if (w.total == 0) return PD_OK;
    PackArgs a{s->x, s->y, s->z, s->vx, s->vy, s->vz, s->fx, s->fy, s->fz, s->vir, s->type, (uint32_t *)dst,
               (uint64_t)s->n, w.pos, w.vel, w.frc, w.tid, w.vir, w.total, w.vrow};
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const uint64_t want = (w.total + 255) / 256;
    const unsigned blocks = (unsigned)std::min<uint64_t>(want, (uint64_t)sms * 8);
    k_snapshot_pack<<<blocks, 256, 0, (cudaStream_t)stream>>>(a);
    PD_LAUNCHED();
    return PD_OK;
}

}  // extern "C"
