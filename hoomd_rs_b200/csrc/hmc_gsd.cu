// GSD files: the file layer of hoomd-gsd (hoomd-gsd/src/file_layer.rs) and the HOOMD schema
// frame writer (hoomd-gsd/src/hoomd.rs, hoomd-microstate/src/append.rs), behind the
// hmc_gsd_* entry points of include/hmc.h.
//
// The on-disk format and the order of file operations follow the reference, so the same
// calls write byte-identical files:
//   * header (256 bytes, native byte order): magic 0x65df65df65df65df, index location,
//     index allocated entries, name list location, name list allocated entries (u64 each),
//     schema version and GSD version as (major << 16 | minor) u32, application at byte 48 and
//     schema at byte 112, both null-terminated (file_layer.rs:755-832);
//   * index entries (32 bytes): frame, rows, location (u64), columns (u32), name id (u16),
//     type (u8), flags (u8) (file_layer.rs:893-925); entries are sorted by (frame, id) and the
//     first entry with location 0 ends the index (file_layer.rs:1362-1408);
//   * a new file holds the header, 128 zeroed index entries and a 1024-byte zeroed name list
//     (file_layer.rs:1077-1116);
//   * chunk data goes to a write buffer that is flushed to the end of the file once it holds
//     at least the maximum write buffer size (file_layer.rs:1936-2015); sync writes the data,
//     then the new names, then the index entries of completed frames, growing the name list
//     or the index by doubling into a copy at the end of the file and rewriting the header
//     (file_layer.rs:2213-2436).
// Chunks larger than the write buffer are written from the caller's memory right after the
// buffered bytes: the file receives the same bytes in the same order as when they pass
// through the buffer.
#include <errno.h>
#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <chrono>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <unordered_map>
#include <unordered_set>
#include <vector>

#include "../../include/hmc.h"
#include "hmc_host.h"

namespace {

constexpr uint64_t kNameSize = 64;
constexpr uint64_t kEntrySize = 32;
constexpr uint64_t kHeaderSize = 256;
constexpr uint64_t kMagic = 0x65df65df65df65dfull;
constexpr uint16_t kGsdMajor = 2, kGsdMinor = 1;
constexpr uint64_t kInitialIndexEntries = 128;
constexpr uint64_t kInitialNameListBytes = 1024;
constexpr uint64_t kInitialMaximumWriteBuffer = 1024 * 1024;
constexpr uint32_t kMaxNames = 65535;  // ids are u16 and u16::MAX is never assigned
constexpr double kDefaultAutoSyncSeconds = 10.0;

struct Entry {
    uint64_t frame;
    uint64_t n;
    uint64_t location;
    uint32_t m;
    uint16_t id;
    uint8_t type;
    uint8_t flags;
};
static_assert(sizeof(Entry) == kEntrySize, "index entries are 32 bytes");

bool entry_less(const Entry& a, const Entry& b) { return a.frame != b.frame ? a.frame < b.frame : a.id < b.id; }

uint64_t type_size(uint8_t t) {
    switch (t) {
        case HMC_GSD_U8: case HMC_GSD_I8: case HMC_GSD_STRING: return 1;
        case HMC_GSD_U16: case HMC_GSD_I16: return 2;
        case HMC_GSD_U32: case HMC_GSD_I32: case HMC_GSD_F32: return 4;
        case HMC_GSD_U64: case HMC_GSD_I64: case HMC_GSD_F64: return 8;
        default: return 0;
    }
}

thread_local hmc_gsd_error g_gsd_error = HMC_GSD_OK;

hmc_status gsd_fail(hmc_status st, hmc_gsd_error kind, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_gsd_error = kind;
    return hmc::report_error(st, buf);
}

hmc_status ok() {
    g_gsd_error = HMC_GSD_OK;
    return HMC_OK;
}

// Strict UTF-8 validation (what String::from_utf8 accepts).
bool valid_utf8(const unsigned char* s, size_t n) {
    size_t i = 0;
    while (i < n) {
        unsigned char c = s[i];
        if (c < 0x80) { ++i; continue; }
        size_t len;
        uint32_t cp;
        if ((c & 0xE0) == 0xC0) { len = 2; cp = c & 0x1F; }
        else if ((c & 0xF0) == 0xE0) { len = 3; cp = c & 0x0F; }
        else if ((c & 0xF8) == 0xF0) { len = 4; cp = c & 0x07; }
        else return false;
        if (i + len > n) return false;
        for (size_t k = 1; k < len; ++k) {
            if ((s[i + k] & 0xC0) != 0x80) return false;
            cp = (cp << 6) | (s[i + k] & 0x3F);
        }
        if ((len == 2 && cp < 0x80) || (len == 3 && cp < 0x800) || (len == 4 && (cp < 0x10000 || cp > 0x10FFFF)) ||
            (cp >= 0xD800 && cp <= 0xDFFF))
            return false;
        i += len;
    }
    return true;
}

struct Header {
    uint64_t magic = kMagic;
    uint64_t index_location = 0;
    uint64_t index_allocated = 0;
    uint64_t namelist_location = 0;
    uint64_t namelist_allocated = 0;
    uint16_t schema_major = 0, schema_minor = 0;
    uint16_t gsd_major = kGsdMajor, gsd_minor = kGsdMinor;
    std::string application, schema;

    void encode(unsigned char* b) const {
        std::memset(b, 0, kHeaderSize);
        std::memcpy(b + 0, &magic, 8);
        std::memcpy(b + 8, &index_location, 8);
        std::memcpy(b + 16, &index_allocated, 8);
        std::memcpy(b + 24, &namelist_location, 8);
        std::memcpy(b + 32, &namelist_allocated, 8);
        uint32_t sv = (uint32_t)schema_major << 16 | schema_minor;
        uint32_t gv = (uint32_t)gsd_major << 16 | gsd_minor;
        std::memcpy(b + 40, &sv, 4);
        std::memcpy(b + 44, &gv, 4);
        std::memcpy(b + 48, application.data(), application.size());
        std::memcpy(b + 112, schema.data(), schema.size());
    }
};

}  // namespace

struct hmc_gsd {
    int fd = -1;
    bool writable = false;
    Header h;
    uint64_t file_len = 0;
    // chunk names
    std::unordered_map<std::string, uint16_t> name_id;
    std::vector<std::string> names;  // by id
    uint64_t name_insert = 0;        // bytes of the name list in use
    std::vector<char> name_buffer;   // new names not yet in the file
    // index
    std::vector<Entry> entries;      // the entries in the file, in file order
    std::vector<Entry> buffered;     // entries not yet in the file (completed frames, then the open frame)
    size_t pending = 0;              // entries of the open frame (at the end of `buffered`)
    std::unordered_set<uint16_t> frame_names;
    // data
    std::vector<unsigned char> data;
    bool data_flushed = false;
    uint64_t buffer_frame = 0;
    uint64_t file_frame = 0;
    uint64_t max_buffer = kInitialMaximumWriteBuffer;
    // HOOMD schema frame state (hoomd.rs Frame)
    bool frame_open = false;
    bool have_particles_n = false;
    uint32_t particles_n = 0;
    double auto_sync_delay = kDefaultAutoSyncSeconds;
    std::chrono::steady_clock::time_point last_auto_sync = std::chrono::steady_clock::now();
};

namespace {

hmc_status io_fail(const char* what) {
    return gsd_fail(HMC_IO_ERROR, HMC_GSD_IO, "GSD %s: %s", what, std::strerror(errno));
}

hmc_status write_all(int fd, const void* p, uint64_t n, uint64_t offset) {
    const char* c = (const char*)p;
    while (n > 0) {
        ssize_t w = pwrite(fd, c, n > (1ull << 30) ? (1ull << 30) : n, (off_t)offset);
        if (w < 0) {
            if (errno == EINTR) continue;
            return io_fail("write");
        }
        c += w;
        n -= (uint64_t)w;
        offset += (uint64_t)w;
    }
    return HMC_OK;
}

hmc_status read_all(int fd, void* p, uint64_t n, uint64_t offset) {
    char* c = (char*)p;
    while (n > 0) {
        ssize_t r = pread(fd, c, n > (1ull << 30) ? (1ull << 30) : n, (off_t)offset);
        if (r < 0) {
            if (errno == EINTR) continue;
            return io_fail("read");
        }
        if (r == 0) return gsd_fail(HMC_IO_ERROR, HMC_GSD_IO, "GSD read: unexpected end of file");
        c += r;
        n -= (uint64_t)r;
        offset += (uint64_t)r;
    }
    return HMC_OK;
}

hmc_status file_sync(int fd) { return fsync(fd) == 0 ? HMC_OK : io_fail("fsync"); }

#define GSD_TRY(x)                       \
    do {                                 \
        hmc_status st_ = (x);            \
        if (st_ != HMC_OK) return st_;   \
    } while (0)

hmc_status write_header(hmc_gsd* f) {
    unsigned char b[kHeaderSize];
    f->h.encode(b);
    return write_all(f->fd, b, kHeaderSize, 0);
}

hmc_status read_entry(hmc_gsd* f, uint64_t i, Entry* e) {
    return read_all(f->fd, e, kEntrySize, f->h.index_location + i * kEntrySize);
}

bool entry_valid(const hmc_gsd* f, const Entry& e) {
    const uint64_t sz = type_size(e.type);
    if (sz == 0) return false;
    // rows * columns * size must fit in the file (no overflow: each factor is checked)
    if (e.m != 0 && e.n > (UINT64_MAX / e.m) / sz) return false;
    const uint64_t total = e.n * (uint64_t)e.m * sz;
    if (e.location > f->file_len || total > f->file_len - e.location) return false;
    if (e.frame >= f->h.index_allocated) return false;
    if (e.id >= f->names.size()) return false;
    if (e.flags != 0) return false;
    return true;
}

// GsdFile::from_file (file_layer.rs:1118-1206).
hmc_status load(hmc_gsd* f) {
    unsigned char b[kHeaderSize];
    GSD_TRY(read_all(f->fd, b, kHeaderSize, 0));
    Header& h = f->h;
    std::memcpy(&h.magic, b + 0, 8);
    if (h.magic != kMagic)
        return gsd_fail(HMC_IO_ERROR, HMC_GSD_INVALID_FILE_IDENTIFIER, "invalid file identifier %llu",
                        (unsigned long long)h.magic);
    std::memcpy(&h.index_location, b + 8, 8);
    std::memcpy(&h.index_allocated, b + 16, 8);
    std::memcpy(&h.namelist_location, b + 24, 8);
    std::memcpy(&h.namelist_allocated, b + 32, 8);
    uint32_t sv, gv;
    std::memcpy(&sv, b + 40, 4);
    std::memcpy(&gv, b + 44, 4);
    {
        const unsigned char* a = b + 48;
        size_t n = 0;
        while (48 + n < kHeaderSize && a[n]) ++n;
        if (!valid_utf8(a, n)) return gsd_fail(HMC_IO_ERROR, HMC_GSD_INVALID_STRING, "invalid application");
        h.application.assign((const char*)a, n);
        const unsigned char* s = b + 112;
        n = 0;
        while (112 + n < 178 && s[n]) ++n;
        if (!valid_utf8(s, n)) return gsd_fail(HMC_IO_ERROR, HMC_GSD_INVALID_STRING, "invalid schema");
        h.schema.assign((const char*)s, n);
    }
    h.schema_major = (uint16_t)(sv >> 16);
    h.schema_minor = (uint16_t)(sv & 0xffff);
    h.gsd_major = (uint16_t)(gv >> 16);
    h.gsd_minor = (uint16_t)(gv & 0xffff);
    if (h.gsd_major != 2)
        return gsd_fail(HMC_IO_ERROR, HMC_GSD_UNSUPPORTED_VERSION, "unsupported GSD file version (%u, %u)",
                        h.gsd_major, h.gsd_minor);
    struct stat st;
    if (fstat(f->fd, &st) != 0) return io_fail("stat");
    f->file_len = (uint64_t)st.st_size;
    const uint64_t L = f->file_len;
    if (h.index_allocated == 0 || h.index_location > L || h.index_allocated > (L - h.index_location) / kEntrySize)
        return gsd_fail(HMC_IO_ERROR, HMC_GSD_INDEX_OUT_OF_BOUNDS, "index out of bounds (location=%llu)",
                        (unsigned long long)h.index_location);
    if (h.namelist_allocated == 0 || h.namelist_location > L ||
        h.namelist_allocated > (L - h.namelist_location) / kNameSize)
        return gsd_fail(HMC_IO_ERROR, HMC_GSD_NAME_LIST_OUT_OF_BOUNDS, "name list out of bounds (location=%llu)",
                        (unsigned long long)h.namelist_location);
    std::vector<unsigned char> nl(h.namelist_allocated * kNameSize);
    GSD_TRY(read_all(f->fd, nl.data(), nl.size(), h.namelist_location));
    if (nl.back() != 0) return gsd_fail(HMC_IO_ERROR, HMC_GSD_NAME_LIST_NOT_TERMINATED, "name list not terminated");
    // decode_name_map (file_layer.rs:1208-1242)
    size_t pos = 0;
    while (pos < nl.size() && nl[pos] != 0) {
        size_t end = pos;
        while (end < nl.size() && nl[end]) ++end;
        if (!valid_utf8(nl.data() + pos, end - pos))
            return gsd_fail(HMC_IO_ERROR, HMC_GSD_INVALID_STRING, "invalid chunk name");
        std::string name((const char*)nl.data() + pos, end - pos);
        const size_t id = f->names.size();
        if (!f->name_id.emplace(name, (uint16_t)id).second)
            return gsd_fail(HMC_IO_ERROR, HMC_GSD_DUPLICATE_CHUNK_NAME, "duplicate chunk name in the name list");
        if (id == kMaxNames) return gsd_fail(HMC_IO_ERROR, HMC_GSD_NAME_LIST_OVERFLOW, "too many chunk names");
        f->names.push_back(std::move(name));
        f->name_insert += (end - pos) + 1;
        pos = end + 1;
    }
    // count_index_entries (file_layer.rs:1362-1408): binary search for the first location 0
    Entry first;
    GSD_TRY(read_entry(f, 0, &first));
    uint64_t count = 0;
    if (first.location != 0) {
        if (!entry_valid(f, first))
            return gsd_fail(HMC_IO_ERROR, HMC_GSD_CORRUPT_INDEX_ENTRY, "corrupt index entry 0");
        uint64_t l = 0, r = h.index_allocated;
        for (;;) {
            const uint64_t m = l + (r - l) / 2;
            Entry em, el;
            GSD_TRY(read_entry(f, m, &em));
            GSD_TRY(read_entry(f, l, &el));
            if (em.location != 0) {
                if (!entry_valid(f, em) || em.frame < el.frame)
                    return gsd_fail(HMC_IO_ERROR, HMC_GSD_CORRUPT_INDEX_ENTRY, "corrupt index entry %llu",
                                    (unsigned long long)m);
                l = m;
            } else {
                r = m;
            }
            if (r - l == 1) break;
        }
        count = r;
    }
    f->entries.resize(count);
    if (count) GSD_TRY(read_all(f->fd, f->entries.data(), count * kEntrySize, h.index_location));
    if (count) {
        f->file_frame = f->entries.back().frame + 1;
        f->buffer_frame = f->file_frame;
    }
    // a writable 2.0 file is upgraded to 2.1
    if (f->writable && h.gsd_major == kGsdMajor && h.gsd_minor < kGsdMinor) {
        h.gsd_minor = kGsdMinor;
        GSD_TRY(write_header(f));
    }
    return HMC_OK;
}

// GsdFile::initialize_file (file_layer.rs:1077-1116).
hmc_status initialize(hmc_gsd* f, const char* application, const char* schema, uint16_t major, uint16_t minor) {
    const size_t la = std::strlen(application), ls = std::strlen(schema);
    if (la > kNameSize - 1)
        return gsd_fail(HMC_INVALID_ARGUMENT, HMC_GSD_NAME_TOO_LONG, "the name `%s` is too long", application);
    if (ls > kNameSize - 1)
        return gsd_fail(HMC_INVALID_ARGUMENT, HMC_GSD_NAME_TOO_LONG, "the name `%s` is too long", schema);
    Header h;
    h.application = application;
    h.schema = schema;
    h.schema_major = major;
    h.schema_minor = minor;
    h.index_location = kHeaderSize;
    h.index_allocated = kInitialIndexEntries;
    h.namelist_location = kHeaderSize + kEntrySize * kInitialIndexEntries;
    h.namelist_allocated = kInitialNameListBytes / kNameSize;
    unsigned char b[kHeaderSize];
    h.encode(b);
    GSD_TRY(write_all(f->fd, b, kHeaderSize, 0));
    if (ftruncate(f->fd, (off_t)(kHeaderSize + kEntrySize * kInitialIndexEntries + kInitialNameListBytes)) != 0)
        return io_fail("set_len");
    return file_sync(f->fd);
}

hmc_status flush_data(hmc_gsd* f, bool* wrote) {
    *wrote = false;
    if (f->data.empty()) return HMC_OK;
    GSD_TRY(write_all(f->fd, f->data.data(), f->data.size(), f->file_len));
    f->file_len += f->data.size();
    f->data.clear();
    *wrote = true;
    return HMC_OK;
}

// expand_name_list_to / expand_index_to (file_layer.rs:2331-2436): the region grows by
// doubling until it exceeds `needed` bytes and moves to the end of the file.
hmc_status relocate(hmc_gsd* f, uint64_t* location, uint64_t* allocated, uint64_t unit, uint64_t used_bytes,
                    uint64_t needed) {
    uint64_t size = *allocated * unit;
    while (size <= needed) size *= 2;
    const uint64_t new_allocated = (size + unit - 1) / unit;
    size = new_allocated * unit;
    const uint64_t at = f->file_len;
    std::vector<unsigned char> old(used_bytes);
    if (used_bytes) GSD_TRY(read_all(f->fd, old.data(), used_bytes, *location));
    if (used_bytes) GSD_TRY(write_all(f->fd, old.data(), used_bytes, at));
    if (ftruncate(f->fd, (off_t)(at + size)) != 0) return io_fail("set_len");
    f->file_len = at + size;
    GSD_TRY(file_sync(f->fd));
    *location = at;
    *allocated = new_allocated;
    GSD_TRY(write_header(f));
    return file_sync(f->fd);
}

hmc_status flush_names(hmc_gsd* f) {
    if (f->name_buffer.empty()) return HMC_OK;
    const uint64_t need = f->name_insert + f->name_buffer.size();
    if (need > f->h.namelist_allocated * kNameSize)
        GSD_TRY(relocate(f, &f->h.namelist_location, &f->h.namelist_allocated, kNameSize, f->name_insert, need));
    GSD_TRY(write_all(f->fd, f->name_buffer.data(), f->name_buffer.size(), f->h.namelist_location + f->name_insert));
    f->name_insert += f->name_buffer.size();
    f->name_buffer.clear();
    return HMC_OK;
}

// GsdFile::sync_all (file_layer.rs:2269-2329).
hmc_status sync_all(hmc_gsd* f) {
    if (!f->writable) return gsd_fail(HMC_INVALID_ARGUMENT, HMC_GSD_NOT_WRITABLE, "file opened in read-only mode");
    bool wrote;
    GSD_TRY(flush_data(f, &wrote));
    if (wrote || f->data_flushed) {
        f->data_flushed = false;
        GSD_TRY(file_sync(f->fd));
    }
    GSD_TRY(flush_names(f));
    const size_t k = f->buffered.size() - f->pending;
    if (k > 0) {
        const uint64_t n = f->entries.size();
        if (n + k > f->h.index_allocated)
            GSD_TRY(relocate(f, &f->h.index_location, &f->h.index_allocated, kEntrySize, n * kEntrySize,
                             (n + k) * kEntrySize));
        std::sort(f->buffered.begin(), f->buffered.begin() + k, entry_less);
        GSD_TRY(write_all(f->fd, f->buffered.data(), k * kEntrySize, f->h.index_location + n * kEntrySize));
        f->entries.insert(f->entries.end(), f->buffered.begin(), f->buffered.begin() + k);
        f->buffered.erase(f->buffered.begin(), f->buffered.begin() + k);
        GSD_TRY(file_sync(f->fd));
    }
    f->file_frame = f->buffer_frame;
    return HMC_OK;
}

hmc_status get_id(hmc_gsd* f, const std::string& name, uint16_t* id) {
    auto it = f->name_id.find(name);
    if (it != f->name_id.end()) {
        *id = it->second;
        return HMC_OK;
    }
    if (f->names.size() >= kMaxNames)
        return gsd_fail(HMC_INVALID_ARGUMENT, HMC_GSD_NAME_LIST_OVERFLOW, "too many chunk names");
    *id = (uint16_t)f->names.size();
    f->names.push_back(name);
    f->name_id.emplace(name, *id);
    f->name_buffer.insert(f->name_buffer.end(), name.begin(), name.end());
    f->name_buffer.push_back(0);
    return HMC_OK;
}

// GsdFile::write_details (file_layer.rs:1936-2015). `parts` are consecutive pieces of the
// chunk's bytes (one piece for a plain chunk).
struct Piece {
    const void* p;
    uint64_t n;
};
hmc_status write_details(hmc_gsd* f, const char* name, uint32_t columns, uint8_t type, uint64_t rows,
                         const Piece* parts, int n_parts) {
    if (!f->writable) return gsd_fail(HMC_INVALID_ARGUMENT, HMC_GSD_NOT_WRITABLE, "file opened in read-only mode");
    const uint64_t location = f->file_len + f->data.size();
    uint16_t id;
    GSD_TRY(get_id(f, name, &id));
    if (!f->frame_names.insert(id).second)
        return gsd_fail(HMC_INVALID_ARGUMENT, HMC_GSD_DUPLICATE_CHUNK_NAME,
                        "chunk `%s` has already been written in frame %llu", name,
                        (unsigned long long)f->buffer_frame);
    uint64_t bytes = 0;
    for (int i = 0; i < n_parts; ++i) bytes += parts[i].n;
    if (f->data.size() + bytes >= f->max_buffer && bytes >= f->max_buffer / 2) {
        // a large chunk: the buffered bytes, then the chunk straight from the caller's memory
        bool wrote;
        GSD_TRY(flush_data(f, &wrote));
        for (int i = 0; i < n_parts; ++i) {
            GSD_TRY(write_all(f->fd, parts[i].p, parts[i].n, f->file_len));
            f->file_len += parts[i].n;
        }
        f->data_flushed = true;
    } else {
        for (int i = 0; i < n_parts; ++i) {
            const unsigned char* c = (const unsigned char*)parts[i].p;
            f->data.insert(f->data.end(), c, c + parts[i].n);
        }
    }
    Entry e{f->buffer_frame, rows, location, columns, id, type, 0};
    f->buffered.push_back(e);
    f->pending += 1;
    if (f->data.size() >= f->max_buffer) {
        bool wrote;
        GSD_TRY(flush_data(f, &wrote));
        f->data_flushed = true;
    }
    return HMC_OK;
}

hmc_status end_frame(hmc_gsd* f) {
    if (!f->writable) return gsd_fail(HMC_INVALID_ARGUMENT, HMC_GSD_NOT_WRITABLE, "file opened in read-only mode");
    f->buffer_frame += 1;
    f->pending = 0;
    f->frame_names.clear();
    return HMC_OK;
}

// GsdFile::find_chunk (file_layer.rs:1437-1470).
bool find_chunk(const hmc_gsd* f, uint64_t frame, const char* name, Entry* out) {
    if (frame >= f->file_frame || f->entries.empty()) return false;
    auto it = f->name_id.find(name);
    if (it == f->name_id.end()) return false;
    const Entry key{frame, 0, 0, 0, it->second, 0, 0};
    auto p = std::lower_bound(f->entries.begin(), f->entries.end(), key, entry_less);
    if (p == f->entries.end() || p->frame != frame || p->id != it->second) return false;
    *out = *p;
    return true;
}

hmc_status open_fd(const char* path, int flags, int* fd) {
    *fd = ::open(path, flags | O_CLOEXEC, 0644);
    if (*fd < 0) return gsd_fail(HMC_IO_ERROR, HMC_GSD_IO, "I/O error while creating or opening `%s`: %s", path,
                                 std::strerror(errno));
    return HMC_OK;
}

hmc_status create_file(const char* path, const char* application, const char* schema, uint16_t major,
                       uint16_t minor, int exclusive, hmc_gsd** out) {
    if (!path || !application || !schema || !out)
        return gsd_fail(HMC_INVALID_ARGUMENT, HMC_GSD_OK, "NULL argument");
    *out = nullptr;
    int fd;
    GSD_TRY(open_fd(path, O_RDWR | O_CREAT | (exclusive ? O_EXCL : O_TRUNC), &fd));
    hmc_gsd* f = new hmc_gsd();
    f->fd = fd;
    f->writable = true;
    hmc_status st = initialize(f, application, schema, major, minor);
    if (st == HMC_OK) st = load(f);
    if (st != HMC_OK) {
        ::close(fd);
        delete f;
        return st;
    }
    *out = f;
    return ok();
}

// Frame::validate_particles_chunk (hoomd.rs:413-437).
hmc_status validate_particles(hmc_gsd* f, uint64_t rows, const char* name) {
    if (f->have_particles_n) {
        if (rows != f->particles_n)
            return gsd_fail(HMC_INVALID_ARGUMENT, HMC_GSD_INCONSISTENT_LENGTH,
                            "The length of data chunk %s does not match previously written particles chunks", name);
        return HMC_OK;
    }
    if (rows > UINT32_MAX)
        return gsd_fail(HMC_INVALID_ARGUMENT, HMC_GSD_CHUNK_TOO_LARGE, "cannot write %llu entries to data chunk %s",
                        (unsigned long long)rows, name);
    const uint32_t n = (uint32_t)rows;
    Piece p{&n, 4};
    GSD_TRY(write_details(f, "particles/N", 1, HMC_GSD_U32, 1, &p, 1));
    f->have_particles_n = true;
    f->particles_n = n;
    return HMC_OK;
}

hmc_status append_frame(hmc_gsd* f, uint64_t step) {
    Piece p{&step, 8};
    GSD_TRY(write_details(f, "configuration/step", 1, HMC_GSD_U64, 1, &p, 1));
    f->frame_open = true;
    f->have_particles_n = false;
    return HMC_OK;
}

}  // namespace

extern "C" {

hmc_gsd_error hmc_gsd_last_error(void) { return g_gsd_error; }

hmc_status hmc_gsd_create(const char* path, const char* application, const char* schema, uint16_t schema_major,
                          uint16_t schema_minor, int exclusive, hmc_gsd** out) {
    return create_file(path, application, schema, schema_major, schema_minor, exclusive, out);
}

hmc_status hmc_gsd_create_hoomd(const char* path, const char* application, int exclusive, hmc_gsd** out) {
    // HoomdGsdFile::create / create_new (hoomd.rs:180-260): schema "hoomd", version (1, 4)
    return create_file(path, application ? application : "hoomd-rs-b200", "hoomd", 1, 4, exclusive, out);
}

hmc_status hmc_gsd_open(const char* path, int writable, hmc_gsd** out) {
    if (!path || !out) return gsd_fail(HMC_INVALID_ARGUMENT, HMC_GSD_OK, "NULL argument");
    *out = nullptr;
    int fd;
    GSD_TRY(open_fd(path, writable ? O_RDWR : O_RDONLY, &fd));
    hmc_gsd* f = new hmc_gsd();
    f->fd = fd;
    f->writable = writable != 0;
    hmc_status st = load(f);
    if (st != HMC_OK) {
        ::close(fd);
        delete f;
        return st;
    }
    *out = f;
    return ok();
}

hmc_status hmc_gsd_close(hmc_gsd* f) {
    if (!f) return ok();
    hmc_status st = HMC_OK;
    if (f->writable) {
        if (f->frame_open) {
            // an open HOOMD frame ends when it is dropped (hoomd.rs:781-790)
            end_frame(f);
            f->frame_open = false;
        }
        st = sync_all(f);
    }
    ::close(f->fd);
    delete f;
    return st == HMC_OK ? ok() : st;
}

hmc_status hmc_gsd_write_chunk(hmc_gsd* f, const char* name, uint32_t type, uint64_t rows, uint32_t columns,
                               const void* data) {
    if (!f || !name) return gsd_fail(HMC_INVALID_ARGUMENT, HMC_GSD_OK, "NULL argument");
    const uint64_t sz = type_size((uint8_t)type);
    if (sz == 0 || type > 255) return gsd_fail(HMC_INVALID_ARGUMENT, HMC_GSD_INVALID_TYPE, "unknown GSD type %u", type);
    if (columns == 0)
        return gsd_fail(HMC_INVALID_ARGUMENT, HMC_GSD_INVALID_COLUMNS,
                        "the number of columns must be greater than zero and fit in a u32, got 0");
    if (type == HMC_GSD_STRING && columns != 1)
        return gsd_fail(HMC_INVALID_ARGUMENT, HMC_GSD_INVALID_COLUMNS, "string chunks have one column");
    if (rows > (UINT64_MAX / columns) / sz) return gsd_fail(HMC_INVALID_ARGUMENT, HMC_GSD_OK, "chunk too large");
    const uint64_t bytes = rows * columns * sz;
    if (bytes && !data) return gsd_fail(HMC_INVALID_ARGUMENT, HMC_GSD_OK, "NULL data");
    Piece p{data, bytes};
    GSD_TRY(write_details(f, name, columns, (uint8_t)type, rows, &p, 1));
    return ok();
}

hmc_status hmc_gsd_write_strings(hmc_gsd* f, const char* name, const char* const* strings, uint64_t count) {
    if (!f || !name || (count && !strings)) return gsd_fail(HMC_INVALID_ARGUMENT, HMC_GSD_OK, "NULL argument");
    // write_strings_array (file_layer.rs:1854-1900): columns = longest + 1, i8, zero padded
    size_t longest = 0;
    for (uint64_t i = 0; i < count; ++i) {
        if (!strings[i]) return gsd_fail(HMC_INVALID_ARGUMENT, HMC_GSD_OK, "NULL string");
        longest = std::max(longest, std::strlen(strings[i]));
    }
    if (longest + 1 > UINT32_MAX)
        return gsd_fail(HMC_INVALID_ARGUMENT, HMC_GSD_INVALID_COLUMNS, "string too long");
    const uint32_t columns = (uint32_t)(longest + 1);
    std::vector<char> buf(count * columns, 0);
    for (uint64_t i = 0; i < count; ++i) std::memcpy(buf.data() + i * columns, strings[i], std::strlen(strings[i]));
    Piece p{buf.data(), buf.size()};
    GSD_TRY(write_details(f, name, columns, HMC_GSD_I8, count, &p, 1));
    return ok();
}

hmc_status hmc_gsd_end_frame(hmc_gsd* f) {
    if (!f) return gsd_fail(HMC_INVALID_ARGUMENT, HMC_GSD_OK, "NULL file");
    GSD_TRY(end_frame(f));
    return ok();
}

hmc_status hmc_gsd_sync(hmc_gsd* f) {
    if (!f) return gsd_fail(HMC_INVALID_ARGUMENT, HMC_GSD_OK, "NULL file");
    GSD_TRY(sync_all(f));
    f->last_auto_sync = std::chrono::steady_clock::now();
    return ok();
}

hmc_status hmc_gsd_set_maximum_write_buffer_size(hmc_gsd* f, uint64_t bytes) {
    if (!f) return gsd_fail(HMC_INVALID_ARGUMENT, HMC_GSD_OK, "NULL file");
    f->max_buffer = bytes;
    return ok();
}

hmc_status hmc_gsd_get_info(hmc_gsd* f, hmc_gsd_info* out) {
    if (!f || !out) return gsd_fail(HMC_INVALID_ARGUMENT, HMC_GSD_OK, "NULL argument");
    std::memset(out, 0, sizeof(*out));
    out->n_frames = f->file_frame;
    out->buffer_frame = f->buffer_frame;
    out->file_length = f->file_len;
    out->index_entries = f->entries.size();
    out->index_allocated_entries = f->h.index_allocated;
    out->namelist_allocated_entries = f->h.namelist_allocated;
    out->n_names = (uint32_t)f->names.size();
    out->schema_major = f->h.schema_major;
    out->schema_minor = f->h.schema_minor;
    out->gsd_major = f->h.gsd_major;
    out->gsd_minor = f->h.gsd_minor;
    out->writable = f->writable ? 1 : 0;
    out->maximum_write_buffer_size = f->max_buffer;
    std::snprintf(out->application, sizeof(out->application), "%s", f->h.application.c_str());
    std::snprintf(out->schema, sizeof(out->schema), "%s", f->h.schema.c_str());
    return ok();
}

hmc_status hmc_gsd_name(hmc_gsd* f, uint32_t id, char* buffer, uint64_t capacity) {
    if (!f || !buffer) return gsd_fail(HMC_INVALID_ARGUMENT, HMC_GSD_OK, "NULL argument");
    if (id >= f->names.size()) return gsd_fail(HMC_INVALID_ARGUMENT, HMC_GSD_OK, "no name with id %u", id);
    const std::string& s = f->names[id];
    if (s.size() + 1 > capacity) return gsd_fail(HMC_INVALID_ARGUMENT, HMC_GSD_OK, "buffer too small");
    std::memcpy(buffer, s.c_str(), s.size() + 1);
    return ok();
}

hmc_status hmc_gsd_find_chunk(hmc_gsd* f, uint64_t frame, const char* name, hmc_gsd_chunk* out, int* found) {
    if (!f || !name || !found) return gsd_fail(HMC_INVALID_ARGUMENT, HMC_GSD_OK, "NULL argument");
    Entry e;
    *found = find_chunk(f, frame, name, &e) ? 1 : 0;
    if (*found && out) {
        out->frame = e.frame;
        out->rows = e.n;
        out->location = e.location;
        out->columns = e.m;
        out->id = e.id;
        out->type = e.type;
        out->flags = e.flags;
    }
    return ok();
}

hmc_status hmc_gsd_read_chunk(hmc_gsd* f, uint64_t frame, const char* name, uint32_t type, uint32_t columns,
                              void* out, uint64_t capacity, uint64_t* rows) {
    if (!f || !name) return gsd_fail(HMC_INVALID_ARGUMENT, HMC_GSD_OK, "NULL argument");
    Entry e;
    if (!find_chunk(f, frame, name, &e))
        return gsd_fail(HMC_INVALID_ARGUMENT, HMC_GSD_CHUNK_NOT_FOUND, "chunk `%s` not found in frame %llu", name,
                        (unsigned long long)frame);
    // iter_scalars / iter_arrays / read_string (file_layer.rs:1507-1673): columns first, then type
    if (e.m != columns)
        return gsd_fail(HMC_INVALID_ARGUMENT, HMC_GSD_INVALID_COLUMNS, "expected to read %u columns, found %u",
                        columns, e.m);
    if (e.type != type)
        return gsd_fail(HMC_INVALID_ARGUMENT, HMC_GSD_INVALID_TYPE, "expected type %u, found %u", type, e.type);
    const uint64_t bytes = e.n * (uint64_t)e.m * type_size(e.type);
    if (rows) *rows = e.n;
    if (bytes > capacity) return gsd_fail(HMC_INVALID_ARGUMENT, HMC_GSD_OK, "buffer too small (%llu bytes needed)",
                                          (unsigned long long)bytes);
    if (bytes && !out) return gsd_fail(HMC_INVALID_ARGUMENT, HMC_GSD_OK, "NULL output");
    if (bytes) GSD_TRY(read_all(f->fd, out, bytes, e.location));
    if (type == HMC_GSD_STRING && !valid_utf8((const unsigned char*)out, bytes))
        return gsd_fail(HMC_IO_ERROR, HMC_GSD_INVALID_STRING, "invalid string");
    return ok();
}

hmc_status hmc_gsd_append_frame(hmc_gsd* f, uint64_t step) {
    if (!f) return gsd_fail(HMC_INVALID_ARGUMENT, HMC_GSD_OK, "NULL file");
    GSD_TRY(append_frame(f, step));
    return ok();
}

hmc_status hmc_gsd_frame_particles(hmc_gsd* f, const char* name, uint32_t type, uint64_t rows, uint32_t columns,
                                   const void* data) {
    if (!f || !name) return gsd_fail(HMC_INVALID_ARGUMENT, HMC_GSD_OK, "NULL argument");
    GSD_TRY(validate_particles(f, rows, name));
    return hmc_gsd_write_chunk(f, name, type, rows, columns, data);
}

hmc_status hmc_gsd_frame_end(hmc_gsd* f) {
    if (!f) return gsd_fail(HMC_INVALID_ARGUMENT, HMC_GSD_OK, "NULL file");
    // Frame::end (hoomd.rs:766-778)
    GSD_TRY(end_frame(f));
    f->frame_open = false;
    const double since =
        std::chrono::duration<double>(std::chrono::steady_clock::now() - f->last_auto_sync).count();
    if (since >= f->auto_sync_delay) {
        GSD_TRY(sync_all(f));
        f->last_auto_sync = std::chrono::steady_clock::now();
    }
    return ok();
}

hmc_status hmc_gsd_set_auto_sync_delay(hmc_gsd* f, double seconds) {
    if (!f || !(seconds >= 0.0)) return gsd_fail(HMC_INVALID_ARGUMENT, HMC_GSD_OK, "bad argument");
    f->auto_sync_delay = seconds;
    return ok();
}

hmc_status hmc_gsd_append_system(hmc_gsd* f, hmc_system* sys) {
    if (!f || !sys) return gsd_fail(HMC_INVALID_ARGUMENT, HMC_GSD_OK, "NULL argument");
    if (!f->writable) return gsd_fail(HMC_INVALID_ARGUMENT, HMC_GSD_NOT_WRITABLE, "file opened in read-only mode");
    hmc::GsdFrameView v;
    hmc_status st = hmc::system_gsd_frame(sys, &v);
    if (st != HMC_OK) {
        g_gsd_error = HMC_GSD_OK;
        return st;
    }
    // AppendMicrostate::append_microstate (append.rs:115-129): step, position, orientation,
    // dimensions, box
    GSD_TRY(append_frame(f, v.step));
    GSD_TRY(validate_particles(f, v.n, "particles/position"));
    Piece pos{v.position, v.n * 12};
    GSD_TRY(write_details(f, "particles/position", 3, HMC_GSD_F32, v.n, &pos, 1));
    if (v.orientation) {
        Piece ori{v.orientation, v.n * 16};
        GSD_TRY(write_details(f, "particles/orientation", 4, HMC_GSD_F32, v.n, &ori, 1));
    }
    const uint8_t dims = (uint8_t)v.dim;
    Piece pd{&dims, 1};
    GSD_TRY(write_details(f, "configuration/dimensions", 1, HMC_GSD_U8, 1, &pd, 1));
    // Hypercuboid::to_gsd_box (hoomd-geometry/src/shape/cuboid.rs:377-418), cast to f32
    float box[6] = {(float)v.L[0], (float)v.L[1], v.dim == 3 ? (float)v.L[2] : 0.0f, 0.0f, 0.0f, 0.0f};
    Piece pb{box, sizeof(box)};
    GSD_TRY(write_details(f, "configuration/box", 1, HMC_GSD_F32, 6, &pb, 1));
    return ok();
}

}  // extern "C"
