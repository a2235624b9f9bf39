// GSD (General Simulation Data) file layer, version 2.0, host side of the snapshot I/O path.
//
// The reference writes and reads its trajectory and restart frames through the third-party
// GSDFiles.jl package (compat "0.1, 0.2", Project.toml:16), driven by src/io/GSDIO.jl and
// src/io/RestartIO.jl.  That package is not part of the reference's sources; this file restates
// the published GSD 2.0 file layer it implements, with the layout the reference itself relies on:
//
//   header, 256 bytes at offset 0 (read field by field in GSDIO.jl:110-135):
//     uint64 magic 0x65DF65DF65DF65DF, uint64 index_location, uint64 index_allocated_entries,
//     uint64 namelist_location, uint64 namelist_allocated_entries (bytes of the name block),
//     uint32 schema_version, uint32 gsd_version ((major << 16) | minor), char application[64],
//     char schema[64], char reserved[80];
//   index entries, 32 bytes each: uint64 frame, uint64 N, int64 location, uint32 M, uint16 id,
//     uint8 type, uint8 flags; the index block holds index_allocated_entries entries, the used ones
//     first, sorted by frame and, inside a frame, by name id; unused entries are zero;
//   the name block: the chunk names as null-terminated strings in id order (GSDIO.jl:145-149
//     rebuilds it the same way), zero-filled to its allocated size;
//   chunk data: N x M values of the entry's type, row-major, anywhere after the header.
//
// Type codes are GSD's (RestartIO.jl:27-39): 1 uint8, 2 uint16, 3 uint32, 4 uint64, 5 int8,
// 6 int16, 7 int32, 8 int64, 9 float32, 10 float64, 11 character.
//
// Frames are committed by pd_gsd_end_frame: the frame's chunk data is already in the file, then its
// index entries are written into the index block (moved to the end of the file with twice the
// capacity when full), the name block likewise, and finally the header.  A reader therefore never
// sees a frame whose index entries point at data that is not yet written.
#include <errno.h>
#include <fcntl.h>
#include <stdio.h>
#include <string.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <string>
#include <unordered_map>
#include <vector>

#include "internal.hpp"

namespace {

constexpr uint64_t kMagic = 0x65DF65DF65DF65DFull;
constexpr uint32_t kGsdVersion = (2u << 16) | 0u;
constexpr uint64_t kInitialIndex = 128;      // entries
constexpr uint64_t kInitialNames = 1024;     // bytes

#pragma pack(push, 1)
struct Header {
    uint64_t magic;
    uint64_t index_location;
    uint64_t index_allocated_entries;
    uint64_t namelist_location;
    uint64_t namelist_allocated_entries;
    uint32_t schema_version;
    uint32_t gsd_version;
    char application[64];
    char schema[64];
    char reserved[80];
};
#pragma pack(pop)
static_assert(sizeof(Header) == 256, "GSD header is 256 bytes");
static_assert(sizeof(pd_gsd_index_entry) == 32, "GSD index entry is 32 bytes");

size_t type_size(int t) {
    switch (t) {
        case PD_GSD_UINT8: case PD_GSD_INT8: case PD_GSD_CHARACTER: return 1;
        case PD_GSD_UINT16: case PD_GSD_INT16: return 2;
        case PD_GSD_UINT32: case PD_GSD_INT32: case PD_GSD_FLOAT: return 4;
        case PD_GSD_UINT64: case PD_GSD_INT64: case PD_GSD_DOUBLE: return 8;
        default: return 0;
    }
}

bool pwrite_all(int fd, const void *buf, size_t n, uint64_t off) {
    const char *p = static_cast<const char *>(buf);
    while (n > 0) {
        ssize_t w = ::pwrite(fd, p, n, (off_t)off);
        if (w < 0) {
            if (errno == EINTR) continue;
            return false;
        }
        p += w;
        n -= (size_t)w;
        off += (uint64_t)w;
    }
    return true;
}

bool pread_all(int fd, void *buf, size_t n, uint64_t off) {
    char *p = static_cast<char *>(buf);
    while (n > 0) {
        ssize_t r = ::pread(fd, p, n, (off_t)off);
        if (r < 0) {
            if (errno == EINTR) continue;
            return false;
        }
        if (r == 0) return false;
        p += r;
        n -= (size_t)r;
        off += (uint64_t)r;
    }
    return true;
}

}  // namespace

struct pd_gsd {
    int fd = -1;
    int mode = 0;
    std::string path;
    Header header{};
    std::vector<pd_gsd_index_entry> index;      // committed entries, file order
    std::vector<pd_gsd_index_entry> pending;    // entries of the frame being written
    std::vector<std::string> names;             // id -> name
    std::unordered_map<std::string, uint16_t> ids;
    uint64_t nframes = 0;
    uint64_t file_end = 0;                      // where the next chunk's data goes
    bool names_dirty = false;
};

namespace {

uint64_t names_bytes(const pd_gsd *h) {
    uint64_t b = 0;
    for (auto &n : h->names) b += n.size() + 1;
    return b;
}

int write_names(pd_gsd *h) {
    uint64_t need = names_bytes(h) + 1;   // a trailing empty string ends the block
    if (need > h->header.namelist_allocated_entries) {
        uint64_t cap = std::max<uint64_t>(h->header.namelist_allocated_entries, kInitialNames);
        while (cap < need) cap *= 2;
        h->header.namelist_location = h->file_end;
        h->header.namelist_allocated_entries = cap;
        h->file_end += cap;
    }
    std::vector<char> blk(h->header.namelist_allocated_entries, 0);
    size_t o = 0;
    for (auto &n : h->names) {
        memcpy(blk.data() + o, n.c_str(), n.size() + 1);
        o += n.size() + 1;
    }
    PD_CHECK(pwrite_all(h->fd, blk.data(), blk.size(), h->header.namelist_location), PD_EINVAL,
             "GSD: writing the name block of %s failed: %s", h->path.c_str(), strerror(errno));
    h->names_dirty = false;
    return PD_OK;
}

int write_header(pd_gsd *h) {
    PD_CHECK(pwrite_all(h->fd, &h->header, sizeof(Header), 0), PD_EINVAL, "GSD: writing the header of %s failed: %s",
             h->path.c_str(), strerror(errno));
    return PD_OK;
}

int load(pd_gsd *h) {
    struct stat sb;
    PD_CHECK(fstat(h->fd, &sb) == 0, PD_EINVAL, "GSD: stat of %s failed: %s", h->path.c_str(), strerror(errno));
    PD_CHECK((uint64_t)sb.st_size >= sizeof(Header), PD_EINVAL, "GSD: %s is too short for a GSD header",
             h->path.c_str());
    PD_CHECK(pread_all(h->fd, &h->header, sizeof(Header), 0), PD_EINVAL, "GSD: reading the header of %s failed",
             h->path.c_str());
    PD_CHECK(h->header.magic == kMagic, PD_EINVAL, "GSD: invalid GSD magic in %s", h->path.c_str());
    PD_CHECK((h->header.gsd_version >> 16) == 2, PD_ENOTSUP,
             "GSD: %s has file layer version %u.%u; this build reads and appends version 2 files", h->path.c_str(),
             h->header.gsd_version >> 16, h->header.gsd_version & 0xffffu);
    const uint64_t fsize = (uint64_t)sb.st_size;
    PD_CHECK(h->header.index_location + h->header.index_allocated_entries * 32 <= fsize &&
                 h->header.namelist_location + h->header.namelist_allocated_entries <= fsize,
             PD_EINVAL, "GSD: the index or name block of %s lies beyond the end of the file", h->path.c_str());
    // names
    std::vector<char> blk(h->header.namelist_allocated_entries + 1, 0);
    PD_CHECK(pread_all(h->fd, blk.data(), h->header.namelist_allocated_entries, h->header.namelist_location), PD_EINVAL,
             "GSD: reading the name block of %s failed", h->path.c_str());
    size_t o = 0;
    while (o < h->header.namelist_allocated_entries && blk[o] != 0) {
        std::string nm(blk.data() + o);
        o += nm.size() + 1;
        PD_CHECK(h->names.size() < 65535, PD_EINVAL, "GSD: %s has more than 65535 chunk names", h->path.c_str());
        h->ids.emplace(nm, (uint16_t)h->names.size());
        h->names.push_back(std::move(nm));
    }
    // index: the used entries come first; the first entry with location 0 ends them
    std::vector<pd_gsd_index_entry> all(h->header.index_allocated_entries);
    if (!all.empty())
        PD_CHECK(pread_all(h->fd, all.data(), all.size() * 32, h->header.index_location), PD_EINVAL,
                 "GSD: reading the index of %s failed", h->path.c_str());
    uint64_t used = 0;
    while (used < all.size() && all[used].location != 0) ++used;
    all.resize(used);
    for (size_t k = 0; k < all.size(); ++k) {
        const pd_gsd_index_entry &e = all[k];
        const size_t ts = type_size(e.type);
        PD_CHECK(ts != 0, PD_EINVAL, "GSD: index entry %zu of %s has unknown type %d", k, h->path.c_str(), (int)e.type);
        PD_CHECK(e.id < h->names.size(), PD_EINVAL, "GSD: index entry %zu of %s names id %d of %zu", k,
                 h->path.c_str(), (int)e.id, h->names.size());
        PD_CHECK(e.location > 0 && (uint64_t)e.location + e.N * (uint64_t)e.M * ts <= fsize, PD_EINVAL,
                 "GSD: index entry %zu of %s points beyond the end of the file", k, h->path.c_str());
        PD_CHECK(k == 0 || e.frame >= all[k - 1].frame, PD_EINVAL, "GSD: the index of %s is not sorted by frame",
                 h->path.c_str());
    }
    h->index = std::move(all);
    h->nframes = h->index.empty() ? 0 : h->index.back().frame + 1;
    h->file_end = fsize;
    return PD_OK;
}

const pd_gsd_index_entry *find(const pd_gsd *h, uint64_t frame, uint16_t id) {
    auto lo = std::lower_bound(h->index.begin(), h->index.end(), frame,
                               [](const pd_gsd_index_entry &e, uint64_t f) { return e.frame < f; });
    for (auto it = lo; it != h->index.end() && it->frame == frame; ++it)
        if (it->id == id) return &*it;
    return nullptr;
}

}  // namespace

extern "C" {

int pd_gsd_open(const char *path, int mode, const char *application, const char *schema, uint32_t schema_version,
                pd_gsd **out) {
    PD_CHECK(out && path, PD_EINVAL, "pd_gsd_open: null argument");
    *out = nullptr;
    PD_CHECK(mode == PD_GSD_CREATE || mode == PD_GSD_APPEND || mode == PD_GSD_READ, PD_EINVAL,
             "pd_gsd_open: unknown mode %d", mode);
    if (mode == PD_GSD_CREATE) {
        PD_CHECK(application && schema, PD_EINVAL, "pd_gsd_open: a new file needs an application and a schema name");
        PD_CHECK(strlen(application) < 64 && strlen(schema) < 64, PD_EINVAL,
                 "pd_gsd_open: application and schema names are limited to 63 bytes");
    }
    pd_gsd *h = new pd_gsd();
    h->mode = mode;
    h->path = path;
    int rc = PD_OK;
    if (mode == PD_GSD_CREATE) {
        h->fd = ::open(path, O_RDWR | O_CREAT | O_TRUNC, 0644);
        if (h->fd < 0) {
            pdb::set_error("pd_gsd_open: cannot create %s: %s", path, strerror(errno));
            delete h;
            return PD_EINVAL;
        }
        memset(&h->header, 0, sizeof(Header));
        h->header.magic = kMagic;
        h->header.gsd_version = kGsdVersion;
        h->header.schema_version = schema_version;
        strncpy(h->header.application, application, 63);
        strncpy(h->header.schema, schema, 63);
        h->header.index_location = sizeof(Header);
        h->header.index_allocated_entries = kInitialIndex;
        h->header.namelist_location = sizeof(Header) + kInitialIndex * 32;
        h->header.namelist_allocated_entries = kInitialNames;
        h->file_end = h->header.namelist_location + kInitialNames;
        std::vector<char> zeros(h->file_end, 0);
        memcpy(zeros.data(), &h->header, sizeof(Header));
        if (!pwrite_all(h->fd, zeros.data(), zeros.size(), 0)) {
            pdb::set_error("pd_gsd_open: writing the initial blocks of %s failed: %s", path, strerror(errno));
            rc = PD_EINVAL;
        }
    } else {
        h->fd = ::open(path, mode == PD_GSD_APPEND ? O_RDWR : O_RDONLY);
        if (h->fd < 0) {
            pdb::set_error("pd_gsd_open: cannot open %s: %s", path, strerror(errno));
            delete h;
            return PD_EINVAL;
        }
        rc = load(h);
    }
    if (rc != PD_OK) {
        ::close(h->fd);
        delete h;
        return rc;
    }
    *out = h;
    return PD_OK;
}

int pd_gsd_write_chunk(pd_gsd *h, const char *name, int type, uint64_t N, uint32_t M, const void *data) {
    PD_CHECK(h && name, PD_EINVAL, "pd_gsd_write_chunk: null argument");
    PD_CHECK(h->mode != PD_GSD_READ, PD_ESTATE, "pd_gsd_write_chunk: %s is open for reading", h->path.c_str());
    const size_t ts = type_size(type);
    PD_CHECK(ts != 0, PD_EINVAL, "pd_gsd_write_chunk: unknown GSD type %d for %s", type, name);
    PD_CHECK(M > 0, PD_EINVAL, "pd_gsd_write_chunk: %s needs M >= 1", name);
    PD_CHECK(N == 0 || data, PD_EINVAL, "pd_gsd_write_chunk: %s has N = %llu and no data", name,
             (unsigned long long)N);
    PD_CHECK(strlen(name) > 0, PD_EINVAL, "pd_gsd_write_chunk: empty chunk name");
    uint16_t id;
    auto it = h->ids.find(name);
    if (it == h->ids.end()) {
        PD_CHECK(h->names.size() < 65535, PD_EINVAL, "pd_gsd_write_chunk: more than 65535 chunk names");
        id = (uint16_t)h->names.size();
        h->ids.emplace(name, id);
        h->names.emplace_back(name);
        h->names_dirty = true;
    } else {
        id = it->second;
    }
    for (auto &e : h->pending)
        PD_CHECK(e.id != id, PD_EINVAL, "pd_gsd_write_chunk: %s is already in frame %llu", name,
                 (unsigned long long)h->nframes);
    const uint64_t bytes = N * (uint64_t)M * ts;
    pd_gsd_index_entry e{};
    e.frame = h->nframes;
    e.N = N;
    e.M = M;
    e.id = id;
    e.type = (uint8_t)type;
    e.flags = 0;
    e.location = (int64_t)h->file_end;
    if (bytes > 0)
        PD_CHECK(pwrite_all(h->fd, data, bytes, h->file_end), PD_EINVAL, "pd_gsd_write_chunk: writing %s failed: %s",
                 name, strerror(errno));
    h->file_end += bytes;
    h->pending.push_back(e);
    return PD_OK;
}

int pd_gsd_end_frame(pd_gsd *h) {
    PD_CHECK(h, PD_EINVAL, "pd_gsd_end_frame: null handle");
    PD_CHECK(h->mode != PD_GSD_READ, PD_ESTATE, "pd_gsd_end_frame: %s is open for reading", h->path.c_str());
    std::sort(h->pending.begin(), h->pending.end(),
              [](const pd_gsd_index_entry &a, const pd_gsd_index_entry &b) { return a.id < b.id; });
    const uint64_t used = h->index.size();
    const uint64_t need = used + h->pending.size();
    bool moved = false;
    if (need > h->header.index_allocated_entries) {
        uint64_t cap = std::max<uint64_t>(h->header.index_allocated_entries, kInitialIndex);
        while (cap < need) cap *= 2;
        h->header.index_location = h->file_end;
        h->header.index_allocated_entries = cap;
        h->file_end += cap * 32;
        moved = true;
    }
    h->index.insert(h->index.end(), h->pending.begin(), h->pending.end());
    h->pending.clear();
    int rc;
    if (moved) {
        std::vector<pd_gsd_index_entry> blk(h->header.index_allocated_entries);
        memset(blk.data(), 0, blk.size() * 32);
        std::copy(h->index.begin(), h->index.end(), blk.begin());
        PD_CHECK(pwrite_all(h->fd, blk.data(), blk.size() * 32, h->header.index_location), PD_EINVAL,
                 "pd_gsd_end_frame: writing the index of %s failed: %s", h->path.c_str(), strerror(errno));
    } else if (need > used) {
        PD_CHECK(pwrite_all(h->fd, h->index.data() + used, (need - used) * 32, h->header.index_location + used * 32),
                 PD_EINVAL, "pd_gsd_end_frame: writing the index of %s failed: %s", h->path.c_str(), strerror(errno));
    }
    if (h->names_dirty && (rc = write_names(h)) != PD_OK) return rc;
    if ((rc = write_header(h)) != PD_OK) return rc;
    h->nframes += 1;
    return PD_OK;
}

int pd_gsd_flush(pd_gsd *h) {
    PD_CHECK(h, PD_EINVAL, "pd_gsd_flush: null handle");
    if (h->mode != PD_GSD_READ)
        PD_CHECK(::fsync(h->fd) == 0, PD_EINVAL, "pd_gsd_flush: fsync of %s failed: %s", h->path.c_str(),
                 strerror(errno));
    return PD_OK;
}

int pd_gsd_close(pd_gsd *h) {
    if (!h) return PD_OK;
    int rc = PD_OK;
    if (h->mode != PD_GSD_READ && !h->pending.empty()) {
        // chunks written after the last end_frame belong to no committed frame: drop them
        h->pending.clear();
    }
    if (h->fd >= 0 && ::close(h->fd) != 0) {
        pdb::set_error("pd_gsd_close: closing %s failed: %s", h->path.c_str(), strerror(errno));
        rc = PD_EINVAL;
    }
    delete h;
    return rc;
}

uint64_t pd_gsd_nframes(const pd_gsd *h) { return h ? h->nframes : 0; }

int pd_gsd_header(const pd_gsd *h, uint32_t *gsd_version, uint32_t *schema_version, char *application,
                  char *schema) {
    PD_CHECK(h, PD_EINVAL, "pd_gsd_header: null handle");
    if (gsd_version) *gsd_version = h->header.gsd_version;
    if (schema_version) *schema_version = h->header.schema_version;
    if (application) {
        memcpy(application, h->header.application, 64);
        application[63] = 0;
    }
    if (schema) {
        memcpy(schema, h->header.schema, 64);
        schema[63] = 0;
    }
    return PD_OK;
}

int pd_gsd_find_chunk(const pd_gsd *h, uint64_t frame, const char *name, pd_gsd_index_entry *out, int *found) {
    PD_CHECK(h && name && out && found, PD_EINVAL, "pd_gsd_find_chunk: null argument");
    *found = 0;
    auto it = h->ids.find(name);
    if (it == h->ids.end()) return PD_OK;
    const pd_gsd_index_entry *e = find(h, frame, it->second);
    if (e) {
        *out = *e;
        *found = 1;
    }
    return PD_OK;
}

int pd_gsd_read_chunk(const pd_gsd *h, const pd_gsd_index_entry *e, void *buf, uint64_t bytes) {
    PD_CHECK(h && e && buf, PD_EINVAL, "pd_gsd_read_chunk: null argument");
    const size_t ts = type_size(e->type);
    PD_CHECK(ts != 0, PD_EINVAL, "pd_gsd_read_chunk: unknown GSD type %d", (int)e->type);
    const uint64_t need = e->N * (uint64_t)e->M * ts;
    PD_CHECK(bytes >= need, PD_EINVAL, "pd_gsd_read_chunk: the buffer holds %llu bytes, the chunk %llu",
             (unsigned long long)bytes, (unsigned long long)need);
    if (need == 0) return PD_OK;
    PD_CHECK(pread_all(h->fd, buf, need, (uint64_t)e->location), PD_EINVAL, "pd_gsd_read_chunk: reading %s failed",
             h->path.c_str());
    return PD_OK;
}

int pd_gsd_frame_entries(const pd_gsd *h, uint64_t frame, pd_gsd_index_entry *out, int cap, int *count) {
    PD_CHECK(h && count, PD_EINVAL, "pd_gsd_frame_entries: null argument");
    auto lo = std::lower_bound(h->index.begin(), h->index.end(), frame,
                               [](const pd_gsd_index_entry &e, uint64_t f) { return e.frame < f; });
    int n = 0;
    for (auto it = lo; it != h->index.end() && it->frame == frame; ++it, ++n)
        if (out && n < cap) out[n] = *it;
    *count = n;
    return PD_OK;
}

int pd_gsd_name(const pd_gsd *h, int id, char *buf, int size) {
    PD_CHECK(h && buf && size > 0, PD_EINVAL, "pd_gsd_name: null argument");
    PD_CHECK(id >= 0 && (size_t)id < h->names.size(), PD_EINVAL, "pd_gsd_name: id %d of %zu names", id,
             h->names.size());
    const std::string &s = h->names[(size_t)id];
    PD_CHECK((int)s.size() < size, PD_EINVAL, "pd_gsd_name: the buffer is too short for %s", s.c_str());
    memcpy(buf, s.c_str(), s.size() + 1);
    return PD_OK;
}

}  // extern "C"
