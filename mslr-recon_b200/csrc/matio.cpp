// matio.cpp — MAT v7.3 (HDF5) reader and writer for run_recon's files.
//
// The reference loads its coil maps with MAT.jl (matread, scripts/
// reconstruct.jl:88), its zero-filled k-space with HDF5.jl (h5read, :95) and
// saves its results with MAT.jl (matwrite(...; compress=true), :242-260).
// Both packages sit on libhdf5, which this image does not have; this file
// reads and writes the HDF5 structures of such files directly, from the
// published HDF5 file-format specification.  Host code only: the bulk
// copies, chunk decompression and chunk compression run on a pool of host
// threads over a memory-mapped file (reads) or positioned writes (writes).
#include "mslr_io.h"

#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>
#include <zlib.h>

#include <algorithm>
#include <array>
#include <atomic>
#include <cstdio>
#include <cstring>
#include <ctime>
#include <functional>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

namespace {

thread_local std::string g_err;

struct IoError {
    int code;
    std::string msg;
};

[[noreturn]] void fail(int code, const std::string& m) { throw IoError{code, m}; }

constexpr uint64_t UNDEF = ~0ull;
const uint8_t HDF5_SIG[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};

uint64_t le(const uint8_t* p, int n) {
    uint64_t v = 0;
    for (int i = n - 1; i >= 0; --i) v = (v << 8) | p[i];
    return v;
}

size_t pad8(size_t n) { return (n + 7) & ~size_t(7); }

int n_threads(int n) {
    if (n > 0) return n;
    unsigned h = std::thread::hardware_concurrency();
    return h ? int(h) : 1;
}

// Run f(i) for i in [0, n) on up to `threads` threads; the first error wins.
template <class F>
void parallel_for(int64_t n, int threads, F&& f) {
    int t = int(std::min<int64_t>(n_threads(threads), n));
    if (t <= 1) {
        for (int64_t i = 0; i < n; ++i) f(i);
        return;
    }
    std::atomic<int64_t> next{0};
    std::atomic<bool> stop{false};
    std::mutex mu;
    IoError first{0, ""};
    auto work = [&] {
        try {
            for (;;) {
                if (stop.load(std::memory_order_relaxed)) break;
                int64_t i = next.fetch_add(1);
                if (i >= n) break;
                f(i);
            }
        } catch (const IoError& e) {
            std::lock_guard<std::mutex> g(mu);
            if (!stop.exchange(true)) first = e;
        } catch (const std::exception& e) {
            std::lock_guard<std::mutex> g(mu);
            if (!stop.exchange(true)) first = IoError{MSLRIO_ERR_IO, e.what()};
        }
    };
    std::vector<std::thread> pool;
    for (int i = 1; i < t; ++i) pool.emplace_back(work);
    work();
    for (auto& th : pool) th.join();
    if (stop.load() && first.code) throw first;
}

// Bounded little-endian cursor over file bytes.
struct Cur {
    const uint8_t* p;
    const uint8_t* e;
    void need(size_t n) const {
        if (size_t(e - p) < n) fail(MSLRIO_ERR_FORMAT, "truncated HDF5 structure");
    }
    uint64_t u(int n) {
        need(size_t(n));
        uint64_t v = le(p, n);
        p += n;
        return v;
    }
    void skip(size_t n) {
        need(n);
        p += n;
    }
    const uint8_t* take(size_t n) {
        need(n);
        const uint8_t* q = p;
        p += n;
        return q;
    }
    size_t left() const { return size_t(e - p); }
};

int64_t prod(const int64_t* d, int r) {
    int64_t n = 1;
    for (int i = 0; i < r; ++i) n *= d[i];
    return n;
}

// Bytes of an array of dims d (r of them) with es-byte elements, failing
// rather than wrapping when the file's sizes are absurd.
size_t array_bytes(const int64_t* d, int r, size_t es) {
    unsigned __int128 n = es;
    for (int i = 0; i < r; ++i) {
        if (d[i] < 0) fail(MSLRIO_ERR_FORMAT, "negative dimension");
        n *= uint64_t(d[i]);
        if (n > (unsigned __int128)(uint64_t(1) << 62)) fail(MSLRIO_ERR_FORMAT, "dataset size overflows");
    }
    return size_t(n);
}

int dtype_size(int code) {
    switch (code) {
        case MSLRIO_I8: case MSLRIO_U8: return 1;
        case MSLRIO_I16: case MSLRIO_U16: return 2;
        case MSLRIO_I32: case MSLRIO_U32: case MSLRIO_F32: return 4;
        case MSLRIO_I64: case MSLRIO_U64: case MSLRIO_F64: case MSLRIO_C64: case MSLRIO_REF: return 8;
        case MSLRIO_C128: return 16;
        default: return 0;
    }
}

// Copy the box `ext` between a chunk buffer (dims cd) and the full array
// (dims dd) at offset `off`; to_array selects the direction.  Trailing
// dimensions the box covers completely in both arrays are merged into one
// run, so whole-plane chunks move as a single memcpy.
void copy_box(uint8_t* chunk, const int64_t* cd, uint8_t* arr, const int64_t* dd, const int64_t* off,
              const int64_t* ext, int rank, size_t es, bool to_array) {
    if (rank == 0) {
        if (to_array) memcpy(arr, chunk, es); else memcpy(chunk, arr, es);
        return;
    }
    for (int d = 0; d < rank; ++d)
        if (ext[d] <= 0) return;
    int k = rank - 1;               // dims k.. form one contiguous run in both
    size_t run = size_t(ext[k]) * es;
    while (k > 0 && ext[k] == cd[k] && ext[k] == dd[k]) {
        --k;
        run *= size_t(ext[k]);
    }
    int64_t cs[MSLRIO_MAX_RANK], as[MSLRIO_MAX_RANK];
    cs[rank - 1] = int64_t(es);
    as[rank - 1] = int64_t(es);
    for (int d = rank - 2; d >= 0; --d) {
        cs[d] = cs[d + 1] * cd[d + 1];
        as[d] = as[d + 1] * dd[d + 1];
    }
    int64_t abase = 0;
    for (int d = 0; d < rank; ++d) abase += off[d] * as[d];
    int64_t idx[MSLRIO_MAX_RANK] = {0};
    for (;;) {
        int64_t co = 0, ao = abase;
        for (int d = 0; d < k; ++d) {
            co += idx[d] * cs[d];
            ao += idx[d] * as[d];
        }
        if (to_array) memcpy(arr + ao, chunk + co, run); else memcpy(chunk + co, arr + ao, run);
        int d = k - 1;
        while (d >= 0 && ++idx[d] == ext[d]) idx[d--] = 0;
        if (d < 0) break;
    }
}

void parallel_copy(uint8_t* dst, const uint8_t* src, size_t n, int threads) {
    const size_t blk = size_t(64) << 20;
    int64_t nb = int64_t((n + blk - 1) / blk);
    parallel_for(nb, threads, [&](int64_t i) {
        size_t o = size_t(i) * blk;
        memcpy(dst + o, src + o, std::min(blk, n - o));
    });
}

void parallel_zero(uint8_t* dst, size_t n, int threads) {
    const size_t blk = size_t(64) << 20;
    int64_t nb = int64_t((n + blk - 1) / blk);
    parallel_for(nb, threads, [&](int64_t i) {
        size_t o = size_t(i) * blk;
        memset(dst + o, 0, std::min(blk, n - o));
    });
}

// ───────────────────────────── reader ─────────────────────────────

struct DType {
    int cls = -1;
    uint32_t size = 0;
    int code = 0;          // MSLRIO_* or 0 when not supported
    std::string why;       // why not supported
};

struct Space {
    int rank = 0;
    int64_t dims[MSLRIO_MAX_RANK] = {0};
    bool null = false;
};

struct Filter {
    int id;
    std::vector<uint32_t> cd;
};

struct Msg {
    uint16_t type;
    uint8_t flags;
    const uint8_t* p;
    size_t n;
};

struct ChunkRec {
    uint64_t addr;
    uint64_t size;
    uint32_t mask;
    int64_t off[MSLRIO_MAX_RANK];
};

}  // namespace

struct mslrio_file {
    int fd = -1;
    const uint8_t* map = nullptr;
    size_t size = 0;
    uint64_t base = 0;      // absolute offset that file addresses are relative to
    int so = 8, sl = 8;     // sizes of offsets and lengths
    uint64_t root = UNDEF;  // root group's object-header address

    Cur at(uint64_t addr) const {
        if (addr == UNDEF || addr >= size || base + addr >= size)
            fail(MSLRIO_ERR_FORMAT, "address outside the file");
        return Cur{map + base + addr, map + size};
    }
    Cur at(uint64_t addr, uint64_t len) const {
        Cur c = at(addr);
        if (len > c.left()) fail(MSLRIO_ERR_FORMAT, "structure runs past the end of the file");
        c.e = c.p + len;
        return c;
    }

    // ── object headers ──
    void v1_block(Cur c, std::vector<Msg>& out, std::vector<std::pair<uint64_t, uint64_t>>& cont) const {
        while (c.left() >= 8) {
            uint16_t type = uint16_t(c.u(2));
            size_t n = size_t(c.u(2));
            uint8_t fl = uint8_t(c.u(1));
            c.skip(3);
            const uint8_t* d = c.take(n);
            if (type == 0x10) {
                Cur m{d, d + n};
                uint64_t a = m.u(so), l = m.u(sl);
                cont.emplace_back(a, l);
            } else {
                out.push_back(Msg{type, fl, d, n});
            }
        }
    }
    void v2_block(Cur c, bool crt, std::vector<Msg>& out, std::vector<std::pair<uint64_t, uint64_t>>& cont) const {
        size_t hdr = crt ? 6 : 4;
        while (c.left() >= hdr) {
            uint16_t type = uint16_t(c.u(1));
            size_t n = size_t(c.u(2));
            uint8_t fl = uint8_t(c.u(1));
            if (crt) c.skip(2);
            const uint8_t* d = c.take(n);
            if (type == 0x10) {
                Cur m{d, d + n};
                uint64_t a = m.u(so), l = m.u(sl);
                cont.emplace_back(a, l);
            } else {
                out.push_back(Msg{type, fl, d, n});
            }
        }
    }
    std::vector<Msg> header(uint64_t addr) const {
        std::vector<Msg> out;
        std::vector<std::pair<uint64_t, uint64_t>> cont;
        Cur c = at(addr);
        c.need(4);
        if (memcmp(c.p, "OHDR", 4) == 0) {
            c.skip(4);
            if (c.u(1) != 2) fail(MSLRIO_ERR_FORMAT, "object header: unknown version");
            uint8_t fl = uint8_t(c.u(1));
            if (fl & 0x20) c.skip(16);
            if (fl & 0x10) c.skip(4);
            uint64_t n0 = c.u(1 << (fl & 3));
            c.need(n0);
            v2_block(Cur{c.p, c.p + n0}, (fl & 0x04) != 0, out, cont);
            for (size_t i = 0; i < cont.size(); ++i) {
                if (i > 4096) fail(MSLRIO_ERR_FORMAT, "object header: too many continuation blocks");
                Cur k = at(cont[i].first, cont[i].second);
                if (k.left() < 8 || memcmp(k.p, "OCHK", 4) != 0)
                    fail(MSLRIO_ERR_FORMAT, "object header: bad continuation block");
                v2_block(Cur{k.p + 4, k.e - 4}, (fl & 0x04) != 0, out, cont);
            }
        } else {
            if (c.u(1) != 1) fail(MSLRIO_ERR_FORMAT, "object header: unknown version");
            c.skip(1);
            c.u(2);        // message count
            c.u(4);        // reference count
            uint64_t hsize = c.u(4);
            c.skip(4);     // prefix padded to 16 bytes
            c.need(hsize);
            v1_block(Cur{c.p, c.p + hsize}, out, cont);
            for (size_t i = 0; i < cont.size(); ++i) {
                if (i > 4096) fail(MSLRIO_ERR_FORMAT, "object header: too many continuation blocks");
                v1_block(at(cont[i].first, cont[i].second), out, cont);
            }
        }
        return out;
    }

    // ── datatypes, dataspaces ──
    DType dtype(Cur& c, int depth = 0) const {
        if (depth > 8) fail(MSLRIO_ERR_FORMAT, "datatype nested too deeply");
        DType t;
        uint8_t b0 = uint8_t(c.u(1));
        int ver = b0 >> 4;
        t.cls = b0 & 15;
        uint32_t bf = uint32_t(c.u(3));
        t.size = uint32_t(c.u(4));
        switch (t.cls) {
            case 0: {  // fixed point
                c.skip(4);
                bool be = bf & 1, sg = (bf & 8) != 0;
                if (be) { t.why = "big-endian integers"; break; }
                switch (t.size) {
                    case 1: t.code = sg ? MSLRIO_I8 : MSLRIO_U8; break;
                    case 2: t.code = sg ? MSLRIO_I16 : MSLRIO_U16; break;
                    case 4: t.code = sg ? MSLRIO_I32 : MSLRIO_U32; break;
                    case 8: t.code = sg ? MSLRIO_I64 : MSLRIO_U64; break;
                    default: t.why = "integer of unusual size";
                }
                break;
            }
            case 1: {  // IEEE float
                c.skip(12);
                if ((bf & 1) || (bf & 0x40)) { t.why = "big-endian or VAX floats"; break; }
                if (t.size == 4) t.code = MSLRIO_F32;
                else if (t.size == 8) t.code = MSLRIO_F64;
                else t.why = "float of unusual size";
                break;
            }
            case 3:  // fixed-length string
                t.code = MSLRIO_STR;
                break;
            case 6: {  // compound: complex numbers only
                int nm = int(bf & 0xffff);
                std::vector<std::string> names;
                std::vector<uint64_t> offs;
                std::vector<DType> mt;
                for (int m = 0; m < nm; ++m) {
                    const uint8_t* s = c.p;
                    size_t len = 0;
                    while (len < c.left() && s[len]) ++len;
                    if (len == c.left()) fail(MSLRIO_ERR_FORMAT, "compound member name not terminated");
                    names.emplace_back(reinterpret_cast<const char*>(s), len);
                    c.skip(ver < 3 ? pad8(len + 1) : len + 1);
                    if (ver < 3) {
                        offs.push_back(c.u(4));
                        if (ver == 1) c.skip(28);   // dimensionality, permutation, dims
                    } else {
                        int nb = 1;
                        while (nb < 8 && (uint64_t(1) << (8 * nb)) <= t.size) ++nb;
                        offs.push_back(c.u(nb));
                    }
                    mt.push_back(dtype(c, depth + 1));
                }
                auto is = [&](int i, const char* a, const char* b, const char* cc) {
                    return names[i] == a || names[i] == b || names[i] == cc;
                };
                if (nm == 2 && mt[0].code == mt[1].code && (mt[0].code == MSLRIO_F32 || mt[0].code == MSLRIO_F64) &&
                    offs[0] == 0 && offs[1] == mt[0].size && t.size == 2 * mt[0].size &&
                    is(0, "real", "r", "re") && is(1, "imag", "i", "im"))
                    t.code = mt[0].code == MSLRIO_F32 ? MSLRIO_C64 : MSLRIO_C128;
                else
                    t.why = "compound type other than a complex pair";
                break;
            }
            case 7:
                if ((bf & 15) == 0 && t.size == uint32_t(so)) t.code = MSLRIO_REF;
                else t.why = "region references";
                break;
            default:
                t.why = "datatype class " + std::to_string(t.cls);
        }
        return t;
    }

    Space space(Cur c) const {
        Space s;
        int ver = int(c.u(1));
        s.rank = int(c.u(1));
        int fl = int(c.u(1));
        if (s.rank > MSLRIO_MAX_RANK) fail(MSLRIO_ERR_UNSUPPORTED, "rank above 32");
        if (ver == 1) {
            c.skip(5);
        } else if (ver == 2) {
            int type = int(c.u(1));
            if (type == 2) s.null = true;
        } else {
            fail(MSLRIO_ERR_FORMAT, "dataspace: unknown version");
        }
        for (int d = 0; d < s.rank; ++d) s.dims[d] = int64_t(c.u(sl));
        (void)fl;
        return s;
    }

    // ── groups ──
    std::string heap_name(uint64_t heap, uint64_t off) const {
        Cur h = at(heap);
        h.need(8);
        if (memcmp(h.p, "HEAP", 4) != 0) fail(MSLRIO_ERR_FORMAT, "bad local heap");
        h.skip(8);
        uint64_t dsize = h.u(sl);
        h.u(sl);
        uint64_t daddr = h.u(so);
        if (off >= dsize) fail(MSLRIO_ERR_FORMAT, "name offset outside the local heap");
        Cur d = at(daddr + off, dsize - off);
        size_t n = 0;
        while (n < d.left() && d.p[n]) ++n;
        return std::string(reinterpret_cast<const char*>(d.p), n);
    }

    void group_btree(uint64_t node, uint64_t heap, std::vector<std::pair<std::string, uint64_t>>& out,
                     int depth) const {
        if (depth > 64) fail(MSLRIO_ERR_FORMAT, "group B-tree too deep");
        Cur c = at(node);
        c.need(8);
        if (memcmp(c.p, "TREE", 4) != 0) fail(MSLRIO_ERR_FORMAT, "bad group B-tree node");
        c.skip(4);
        if (c.u(1) != 0) fail(MSLRIO_ERR_FORMAT, "group B-tree node of the wrong type");
        int level = int(c.u(1));
        int n = int(c.u(2));
        c.skip(2 * size_t(so));
        for (int i = 0; i < n; ++i) {
            c.u(sl);
            uint64_t child = c.u(so);
            if (level > 0) {
                group_btree(child, heap, out, depth + 1);
                continue;
            }
            Cur s = at(child);
            s.need(8);
            if (memcmp(s.p, "SNOD", 4) != 0) fail(MSLRIO_ERR_FORMAT, "bad symbol table node");
            s.skip(6);
            int nsym = int(s.u(2));
            for (int k = 0; k < nsym; ++k) {
                uint64_t name = s.u(so);
                uint64_t oh = s.u(so);
                s.skip(24);
                out.emplace_back(heap_name(heap, name), oh);
            }
        }
    }

    bool is_group(const std::vector<Msg>& msgs) const {
        for (auto& m : msgs)
            if (m.type == 0x11 || m.type == 0x06 || m.type == 0x02 || m.type == 0x0A) return true;
        return false;
    }

    // One link message body (header message 0x06, or an object of a group's
    // fractal heap): hard links are kept, soft and external links skipped.
    void link_body(Cur c, std::vector<std::pair<std::string, uint64_t>>& out) const {
        if (c.u(1) != 1) fail(MSLRIO_ERR_FORMAT, "link message: unknown version");
        int fl = int(c.u(1));
        int ltype = (fl & 0x08) ? int(c.u(1)) : 0;
        if (fl & 0x04) c.skip(8);
        if (fl & 0x10) c.skip(1);
        size_t nl = size_t(c.u(1 << (fl & 3)));
        const uint8_t* nm = c.take(nl);
        if (ltype != 0) return;
        out.emplace_back(std::string(reinterpret_cast<const char*>(nm), nl), c.u(so));
    }

    // ── dense link storage: fractal heap + version-2 B-tree name index ──
    static int log2u(uint64_t v) {
        int r = -1;
        while (v) {
            v >>= 1;
            ++r;
        }
        return r;
    }
    struct FHeap {
        int id_len = 0, flags = 0, width = 0, max_heap_bits = 0, rows = 0, off_bytes = 0, len_bytes = 0;
        uint64_t max_obj = 0, start = 0, max_direct = 0, root = UNDEF;
    };
    FHeap fheap(uint64_t addr) const {
        FHeap h;
        Cur c = at(addr);
        c.need(5);
        if (memcmp(c.p, "FRHP", 4) != 0) fail(MSLRIO_ERR_FORMAT, "bad fractal heap header");
        c.skip(4);
        if (c.u(1) != 0) fail(MSLRIO_ERR_FORMAT, "fractal heap: unknown version");
        h.id_len = int(c.u(2));
        int filt = int(c.u(2));
        h.flags = int(c.u(1));
        h.max_obj = c.u(4);
        c.u(sl);                 // next huge object id
        c.u(so);                 // huge-object B-tree
        c.u(sl);                 // free space in managed blocks
        c.u(so);                 // free-space manager
        for (int i = 0; i < 8; ++i) c.u(sl);   // managed / allocated / iterator / counts and sizes
        h.width = int(c.u(2));
        h.start = c.u(sl);
        h.max_direct = c.u(sl);
        h.max_heap_bits = int(c.u(2));
        c.u(2);                  // starting rows of the root indirect block
        h.root = c.u(so);
        h.rows = int(c.u(2));
        if (filt) fail(MSLRIO_ERR_UNSUPPORTED, "filtered fractal heaps are not supported");
        if (h.width <= 0 || h.start == 0 || h.max_direct < h.start || h.max_heap_bits <= 0 || h.max_heap_bits > 64)
            fail(MSLRIO_ERR_FORMAT, "fractal heap: bad doubling table");
        h.off_bytes = (h.max_heap_bits + 7) / 8;
        h.len_bytes = std::min((log2u(h.max_direct) + 7) / 8, log2u(h.max_obj) / 8 + 1);
        return h;
    }
    // Bytes of one managed or tiny heap object named by its heap ID.
    Cur fh_object(const FHeap& h, const uint8_t* id) const {
        int type = (id[0] >> 4) & 3;
        if (type == 2) {
            size_t n = size_t(id[0] & 0x0F) + 1;
            if (1 + n > size_t(h.id_len)) fail(MSLRIO_ERR_FORMAT, "tiny heap object too long");
            return Cur{id + 1, id + 1 + n};
        }
        if (type != 0) fail(MSLRIO_ERR_UNSUPPORTED, "huge fractal-heap objects are not supported");
        if (1 + h.off_bytes + h.len_bytes > h.id_len) fail(MSLRIO_ERR_FORMAT, "heap ID too short");
        uint64_t off = le(id + 1, h.off_bytes), n = le(id + 1 + h.off_bytes, h.len_bytes);
        if (h.rows == 0) return at(h.root + off, n);
        Cur ib = at(h.root);
        ib.need(4);
        if (memcmp(ib.p, "FHIB", 4) != 0) fail(MSLRIO_ERR_FORMAT, "bad fractal heap indirect block");
        ib.skip(5 + size_t(so) + size_t(h.off_bytes));
        int direct_rows = log2u(h.max_direct) - log2u(h.start) + 2;
        uint64_t base = 0;
        for (int r = 0; r < h.rows; ++r) {
            uint64_t bs = r == 0 ? h.start : h.start << (r - 1);
            for (int col = 0; col < h.width; ++col) {
                uint64_t child = ib.u(so);
                if (off >= base && off < base + bs) {
                    if (r >= direct_rows)
                        fail(MSLRIO_ERR_UNSUPPORTED, "nested fractal-heap indirect blocks are not supported");
                    if (child == UNDEF || off - base + n > bs) fail(MSLRIO_ERR_FORMAT, "heap object outside its block");
                    return at(child + (off - base), n);
                }
                base += bs;
            }
        }
        fail(MSLRIO_ERR_FORMAT, "heap offset outside the heap");
    }
    void dense_links(uint64_t heap_addr, uint64_t bt2, std::vector<std::pair<std::string, uint64_t>>& out) const {
        FHeap h = fheap(heap_addr);
        Cur c = at(bt2);
        c.need(4);
        if (memcmp(c.p, "BTHD", 4) != 0) fail(MSLRIO_ERR_FORMAT, "bad v2 B-tree header");
        c.skip(4);
        if (c.u(1) != 0) fail(MSLRIO_ERR_FORMAT, "v2 B-tree: unknown version");
        if (c.u(1) != 5) fail(MSLRIO_ERR_FORMAT, "link name index of the wrong type");
        uint64_t node = c.u(4);
        size_t rs = size_t(c.u(2));
        int depth = int(c.u(2));
        c.skip(2);
        uint64_t root = c.u(so);
        int nroot = int(c.u(2));
        if (rs < 4 + size_t(h.id_len)) fail(MSLRIO_ERR_FORMAT, "v2 B-tree records too small");
        if (depth > 1) fail(MSLRIO_ERR_UNSUPPORTED, "v2 B-tree name indexes deeper than one level");
        auto records = [&](Cur& k, int n) {
            for (int i = 0; i < n; ++i) {
                const uint8_t* r = k.take(rs);
                Cur obj = fh_object(h, r + 4);
                link_body(obj, out);
            }
        };
        if (root == UNDEF) return;
        Cur k = at(root);
        k.need(6);
        if (depth == 0) {
            if (memcmp(k.p, "BTLF", 4) != 0) fail(MSLRIO_ERR_FORMAT, "bad v2 B-tree leaf");
            k.skip(6);
            records(k, nroot);
            return;
        }
        if (memcmp(k.p, "BTIN", 4) != 0) fail(MSLRIO_ERR_FORMAT, "bad v2 B-tree internal node");
        k.skip(6);
        records(k, nroot);
        uint64_t leaf_max = (node - 10) / rs;
        int nb = log2u(leaf_max) / 8 + 1;
        for (int i = 0; i <= nroot; ++i) {
            uint64_t child = k.u(so);
            int n = int(k.u(nb));
            Cur l = at(child);
            l.need(6);
            if (memcmp(l.p, "BTLF", 4) != 0) fail(MSLRIO_ERR_FORMAT, "bad v2 B-tree leaf");
            l.skip(6);
            records(l, n);
        }
    }

    std::vector<std::pair<std::string, uint64_t>> members(uint64_t addr) const {
        std::vector<std::pair<std::string, uint64_t>> out;
        auto msgs = header(addr);
        if (!is_group(msgs)) fail(MSLRIO_ERR_ARG, "not a group");
        for (auto& m : msgs) {
            Cur c{m.p, m.p + m.n};
            if (m.type == 0x11) {
                uint64_t bt = c.u(so), heap = c.u(so);
                group_btree(bt, heap, out, 0);
            } else if (m.type == 0x06) {
                link_body(c, out);
            } else if (m.type == 0x02) {
                c.skip(1);
                int fl = int(c.u(1));
                if (fl & 1) c.skip(8);
                uint64_t fh = c.u(so);
                uint64_t bt2 = c.u(so);
                if (fh != UNDEF) dense_links(fh, bt2, out);
            }
        }
        return out;
    }

    uint64_t lookup(const char* path) const {
        if (!path) fail(MSLRIO_ERR_ARG, "null path");
        uint64_t cur = root;
        std::string p(path);
        size_t i = 0;
        while (i < p.size()) {
            while (i < p.size() && p[i] == '/') ++i;
            if (i >= p.size()) break;
            size_t j = p.find('/', i);
            if (j == std::string::npos) j = p.size();
            std::string name = p.substr(i, j - i);
            bool found = false;
            for (auto& m : members(cur))
                if (m.first == name) {
                    cur = m.second;
                    found = true;
                    break;
                }
            if (!found) fail(MSLRIO_ERR_NOTFOUND, "no object named '" + std::string(path) + "'");
            i = j;
        }
        return cur;
    }

    // ── datasets ──
    struct Dataset {
        DType t;
        Space s;
        int layout = -1;
        uint64_t addr = UNDEF, size = 0;     // contiguous / compact / index address
        const uint8_t* compact = nullptr;
        int cdims_n = 0;
        int64_t cdims[MSLRIO_MAX_RANK + 1] = {0};
        int index = 0;                        // 0 v1 B-tree, 1 single, 2 implicit, 3 fixed array
        uint64_t single_size = 0;
        uint32_t single_mask = 0;
        bool single_filtered = false;
        std::vector<Filter> filters;
        std::string mclass;
        int int_decode = -1, empty = 0;
    };

    void attribute(Cur c, Dataset& ds) const {
        int ver = int(c.u(1));
        if (ver < 1 || ver > 3) fail(MSLRIO_ERR_FORMAT, "attribute: unknown version");
        c.skip(1);
        size_t nl = size_t(c.u(2)), tl = size_t(c.u(2)), sl_ = size_t(c.u(2));
        if (ver == 3) c.skip(1);
        const uint8_t* nm = c.take(ver == 1 ? pad8(nl) : nl);
        std::string name(reinterpret_cast<const char*>(nm), strnlen(reinterpret_cast<const char*>(nm), nl));
        Cur tc{c.take(ver == 1 ? pad8(tl) : tl), nullptr};
        tc.e = tc.p + (ver == 1 ? pad8(tl) : tl);
        Cur sc{c.take(ver == 1 ? pad8(sl_) : sl_), nullptr};
        sc.e = sc.p + (ver == 1 ? pad8(sl_) : sl_);
        if (name != "MATLAB_class" && name != "MATLAB_int_decode" && name != "MATLAB_empty") return;
        DType t = dtype(tc);
        Space s = space(sc);
        if (s.rank > 1 || (s.rank == 1 && s.dims[0] != 1)) return;
        c.need(t.size);
        if (name == "MATLAB_class" && t.code == MSLRIO_STR) {
            ds.mclass.assign(reinterpret_cast<const char*>(c.p), strnlen(reinterpret_cast<const char*>(c.p), t.size));
        } else if (t.cls == 0 && t.size <= 8) {
            int v = int(le(c.p, int(t.size)));
            if (name == "MATLAB_int_decode") ds.int_decode = v;
            if (name == "MATLAB_empty") ds.empty = v;
        }
    }

    void layout_msg(Cur c, Dataset& ds) const {
        int ver = int(c.u(1));
        if (ver == 1 || ver == 2) {
            int nd = int(c.u(1));
            ds.layout = int(c.u(1));
            c.skip(5);
            if (nd > MSLRIO_MAX_RANK + 1) fail(MSLRIO_ERR_UNSUPPORTED, "layout rank above 32");
            if (ds.layout != 0) ds.addr = c.u(so);
            ds.cdims_n = nd;
            for (int d = 0; d < nd; ++d) ds.cdims[d] = int64_t(c.u(4));
            if (ds.layout == 0) {
                ds.size = c.u(4);
                ds.compact = c.take(ds.size);
            } else if (ds.layout == 1) {
                ds.size = uint64_t(prod(ds.cdims, nd));
            }
            ds.index = 0;
        } else if (ver == 3 || ver == 4) {
            ds.layout = int(c.u(1));
            if (ds.layout == 0) {
                ds.size = c.u(2);
                ds.compact = c.take(ds.size);
            } else if (ds.layout == 1) {
                ds.addr = c.u(so);
                ds.size = c.u(sl);
            } else if (ds.layout == 2) {
                if (ver == 3) {
                    int nd = int(c.u(1));
                    if (nd > MSLRIO_MAX_RANK + 1) fail(MSLRIO_ERR_UNSUPPORTED, "layout rank above 32");
                    ds.addr = c.u(so);
                    ds.cdims_n = nd;
                    for (int d = 0; d < nd; ++d) ds.cdims[d] = int64_t(c.u(4));
                    ds.index = 0;
                } else {
                    int fl = int(c.u(1));
                    int nd = int(c.u(1));
                    int enc = int(c.u(1));
                    if (nd > MSLRIO_MAX_RANK + 1 || enc < 1 || enc > 8)
                        fail(MSLRIO_ERR_UNSUPPORTED, "layout: unusual chunk dimensions");
                    ds.cdims_n = nd;
                    for (int d = 0; d < nd; ++d) ds.cdims[d] = int64_t(c.u(enc));
                    int it = int(c.u(1));
                    if (it == 1) {
                        ds.index = 1;
                        if (fl & 2) {
                            ds.single_filtered = true;
                            ds.single_size = c.u(sl);
                            ds.single_mask = uint32_t(c.u(4));
                        }
                    } else if (it == 2) {
                        ds.index = 2;
                    } else if (it == 3) {
                        ds.index = 3;
                        c.skip(1);
                    } else {
                        fail(MSLRIO_ERR_UNSUPPORTED,
                             it == 4 ? "extensible-array chunk index is not supported"
                                     : "version-2 B-tree chunk index is not supported");
                    }
                    ds.addr = c.u(so);
                }
            } else {
                fail(MSLRIO_ERR_UNSUPPORTED, "virtual dataset layout is not supported");
            }
        } else {
            fail(MSLRIO_ERR_FORMAT, "layout: unknown version");
        }
    }

    void filters_msg(Cur c, Dataset& ds) const {
        int ver = int(c.u(1));
        int nf = int(c.u(1));
        if (ver == 1) c.skip(6);
        else if (ver != 2) fail(MSLRIO_ERR_FORMAT, "filter pipeline: unknown version");
        for (int i = 0; i < nf; ++i) {
            Filter f;
            f.id = int(c.u(2));
            size_t nl = (ver == 1 || f.id >= 256) ? size_t(c.u(2)) : 0;
            c.u(2);
            int nv = int(c.u(2));
            c.skip(ver == 1 ? pad8(nl) : nl);
            for (int v = 0; v < nv; ++v) f.cd.push_back(uint32_t(c.u(4)));
            if (ver == 1 && (nv & 1)) c.skip(4);
            ds.filters.push_back(f);
        }
    }

    Dataset dataset(uint64_t addr) const {
        Dataset ds;
        bool have_t = false, have_s = false;
        for (auto& m : header(addr)) {
            Cur c{m.p, m.p + m.n};
            switch (m.type) {
                case 0x01:
                    if (m.flags & 2) fail(MSLRIO_ERR_UNSUPPORTED, "shared dataspace");
                    ds.s = space(c);
                    have_s = true;
                    break;
                case 0x03:
                    if (m.flags & 2) fail(MSLRIO_ERR_UNSUPPORTED, "committed (shared) datatype");
                    ds.t = dtype(c);
                    have_t = true;
                    break;
                case 0x08: layout_msg(c, ds); break;
                case 0x0B: filters_msg(c, ds); break;
                case 0x0C: attribute(c, ds); break;
                case 0x07: fail(MSLRIO_ERR_UNSUPPORTED, "external data storage");
                default: break;
            }
        }
        if (!have_t || !have_s || ds.layout < 0) fail(MSLRIO_ERR_FORMAT, "object is not a dataset");
        return ds;
    }

    void btree_chunks(uint64_t node, int nd, std::vector<ChunkRec>& out, int depth) const {
        if (depth > 64) fail(MSLRIO_ERR_FORMAT, "chunk B-tree too deep");
        Cur c = at(node);
        c.need(8);
        if (memcmp(c.p, "TREE", 4) != 0) fail(MSLRIO_ERR_FORMAT, "bad chunk B-tree node");
        c.skip(4);
        if (c.u(1) != 1) fail(MSLRIO_ERR_FORMAT, "chunk B-tree node of the wrong type");
        int level = int(c.u(1));
        int n = int(c.u(2));
        c.skip(2 * size_t(so));
        for (int i = 0; i < n; ++i) {
            ChunkRec r;
            r.size = c.u(4);
            r.mask = uint32_t(c.u(4));
            for (int d = 0; d < nd; ++d) {
                uint64_t v = c.u(8);
                if (d < MSLRIO_MAX_RANK) r.off[d] = int64_t(v);
            }
            r.addr = c.u(so);
            if (level > 0) btree_chunks(r.addr, nd, out, depth + 1);
            else out.push_back(r);
        }
    }

    void fixed_array_chunks(const Dataset& ds, int rank, const int64_t* grid, std::vector<ChunkRec>& out) const {
        Cur h = at(ds.addr);
        h.need(4);
        if (memcmp(h.p, "FAHD", 4) != 0) fail(MSLRIO_ERR_FORMAT, "bad fixed-array header");
        h.skip(5);
        int client = int(h.u(1));
        int esz = int(h.u(1));
        if (esz < so || (client == 1 && (esz - so - 4 < 1 || esz - so - 4 > 8)))
            fail(MSLRIO_ERR_FORMAT, "fixed array: bad entry size");
        int pbits = int(h.u(1));
        uint64_t nmax = h.u(sl);
        uint64_t dblk = h.u(so);
        Cur d = at(dblk);
        d.need(4);
        if (memcmp(d.p, "FADB", 4) != 0) fail(MSLRIO_ERR_FORMAT, "bad fixed-array data block");
        d.skip(6);
        d.u(so);
        uint64_t per_page = pbits < 63 ? (uint64_t(1) << pbits) : UNDEF;
        bool paged = nmax > per_page;
        if (paged) {
            uint64_t npages = (nmax + per_page - 1) / per_page;
            d.skip((npages + 7) / 8);
            d.skip(4);   // prefix checksum
        }
        int64_t ntot = prod(grid, rank);
        for (uint64_t i = 0; i < nmax && int64_t(i) < ntot; ++i) {
            if (paged && i > 0 && i % per_page == 0) d.skip(4);   // page checksum
            ChunkRec r;
            r.addr = d.u(so);
            r.mask = 0;
            r.size = 0;
            if (client == 1) {
                r.size = d.u(esz - so - 4);
                r.mask = uint32_t(d.u(4));
            } else if (esz != so) {
                d.skip(size_t(esz - so));
            }
            if (r.addr == UNDEF) continue;
            int64_t rem = int64_t(i);
            for (int k = rank - 1; k >= 0; --k) {
                r.off[k] = (rem % grid[k]) * ds.cdims[k];
                rem /= grid[k];
            }
            out.push_back(r);
        }
    }

    void decode_chunk(const Dataset& ds, const ChunkRec& r, size_t chunk_bytes, std::vector<uint8_t>& buf,
                      std::vector<uint8_t>& tmp) const {
        Cur c = at(r.addr, r.size);
        buf.assign(c.p, c.p + r.size);
        for (int i = int(ds.filters.size()) - 1; i >= 0; --i) {
            if (r.mask & (1u << i)) continue;
            const Filter& f = ds.filters[size_t(i)];
            if (f.id == 1) {
                tmp.resize(chunk_bytes);
                uLongf n = uLongf(chunk_bytes);
                int rc = uncompress(tmp.data(), &n, buf.data(), uLong(buf.size()));
                if (rc != Z_OK) fail(MSLRIO_ERR_FORMAT, "deflate: corrupt chunk (zlib " + std::to_string(rc) + ")");
                tmp.resize(n);
                buf.swap(tmp);
            } else if (f.id == 2) {
                size_t es = f.cd.empty() ? 1 : f.cd[0];
                if (es > 1) {
                    size_t ne = buf.size() / es;
                    tmp.resize(buf.size());
                    for (size_t b = 0; b < es; ++b)
                        for (size_t e = 0; e < ne; ++e) tmp[e * es + b] = buf[b * ne + e];
                    std::copy(buf.begin() + long(ne * es), buf.end(), tmp.begin() + long(ne * es));
                    buf.swap(tmp);
                }
            } else if (f.id == 3) {
                if (buf.size() < 4) fail(MSLRIO_ERR_FORMAT, "fletcher32: chunk too short");
                buf.resize(buf.size() - 4);
            } else {
                fail(MSLRIO_ERR_UNSUPPORTED, "filter " + std::to_string(f.id) + " is not supported");
            }
        }
        if (buf.size() != chunk_bytes) fail(MSLRIO_ERR_FORMAT, "chunk decodes to the wrong size");
    }

    void read(uint64_t addr, uint8_t* dst, size_t dst_bytes, int threads) const {
        Dataset ds = dataset(addr);
        if (!ds.t.code) fail(MSLRIO_ERR_UNSUPPORTED, "datatype not supported: " + ds.t.why);
        size_t es = ds.t.size;
        int rank = ds.s.rank;
        size_t n = ds.s.null ? 0 : array_bytes(ds.s.dims, rank, es);
        if (n != dst_bytes) fail(MSLRIO_ERR_ARG, "destination size does not match the dataset");
        if (n == 0) return;
        if (ds.layout == 0) {
            if (ds.size < n) fail(MSLRIO_ERR_FORMAT, "compact data too short");
            memcpy(dst, ds.compact, n);
            return;
        }
        if (ds.layout == 1) {
            if (ds.addr == UNDEF) {
                parallel_zero(dst, n, threads);
                return;
            }
            if (ds.size < n) fail(MSLRIO_ERR_FORMAT, "contiguous data too short");
            Cur c = at(ds.addr, n);
            parallel_copy(dst, c.p, n, threads);
            return;
        }
        // chunked
        if (ds.cdims_n != rank + 1 && ds.cdims_n != rank) fail(MSLRIO_ERR_FORMAT, "chunk rank mismatch");
        int64_t grid[MSLRIO_MAX_RANK];
        for (int d = 0; d < rank; ++d) {
            if (ds.cdims[d] <= 0) fail(MSLRIO_ERR_FORMAT, "zero chunk dimension");
            grid[d] = (ds.s.dims[d] + ds.cdims[d] - 1) / ds.cdims[d];
        }
        size_t chunk_bytes = array_bytes(ds.cdims, rank, es);
        if (chunk_bytes >= (size_t(1) << 32)) fail(MSLRIO_ERR_FORMAT, "chunk of 4 GiB or more");
        int64_t ntot = prod(grid, rank);
        std::vector<ChunkRec> recs;
        if (ds.addr != UNDEF) {
            if (ds.index == 0) {
                btree_chunks(ds.addr, ds.cdims_n, recs, 0);
            } else if (ds.index == 1) {
                ChunkRec r;
                r.addr = ds.addr;
                r.size = ds.single_filtered ? ds.single_size : chunk_bytes;
                r.mask = ds.single_mask;
                for (int d = 0; d < rank; ++d) r.off[d] = 0;
                recs.push_back(r);
            } else if (ds.index == 2) {
                for (int64_t i = 0; i < ntot; ++i) {
                    ChunkRec r;
                    r.addr = ds.addr + uint64_t(i) * chunk_bytes;
                    r.size = chunk_bytes;
                    r.mask = 0;
                    int64_t rem = i;
                    for (int k = rank - 1; k >= 0; --k) {
                        r.off[k] = (rem % grid[k]) * ds.cdims[k];
                        rem /= grid[k];
                    }
                    recs.push_back(r);
                }
            } else {
                fixed_array_chunks(ds, rank, grid, recs);
            }
        }
        for (auto& r : recs) {
            if (r.addr == UNDEF) continue;
            if (ds.filters.empty() && ds.index != 1) r.size = chunk_bytes;
            for (int d = 0; d < rank; ++d)
                if (r.off[d] < 0 || r.off[d] >= ds.s.dims[d] || r.off[d] % ds.cdims[d])
                    fail(MSLRIO_ERR_FORMAT, "chunk offset outside the dataset");
        }
        if (int64_t(recs.size()) < ntot) parallel_zero(dst, n, threads);
        parallel_for(int64_t(recs.size()), threads, [&](int64_t i) {
            thread_local std::vector<uint8_t> a, b;
            const ChunkRec& r = recs[size_t(i)];
            if (r.addr == UNDEF) return;
            decode_chunk(ds, r, chunk_bytes, a, b);
            int64_t ext[MSLRIO_MAX_RANK];
            for (int d = 0; d < rank; ++d) ext[d] = std::min(ds.cdims[d], ds.s.dims[d] - r.off[d]);
            copy_box(a.data(), ds.cdims, dst, ds.s.dims, r.off, ext, rank, es, true);
        });
    }

    void info(uint64_t addr, mslrio_info* o) const {
        memset(o, 0, sizeof(*o));
        o->addr = addr;
        o->matlab_int_decode = -1;
        auto msgs = header(addr);
        if (is_group(msgs)) {
            o->dtype = MSLRIO_GROUP;
            o->layout = -1;
            for (auto& m : msgs)
                if (m.type == 0x0C) {
                    Dataset tmp;
                    attribute(Cur{m.p, m.p + m.n}, tmp);
                    snprintf(o->matlab_class, sizeof(o->matlab_class), "%s", tmp.mclass.c_str());
                }
            return;
        }
        Dataset ds = dataset(addr);
        if (!ds.t.code) fail(MSLRIO_ERR_UNSUPPORTED, "datatype not supported: " + ds.t.why);
        o->dtype = ds.t.code;
        o->elem_size = int32_t(ds.t.size);
        o->rank = ds.s.null ? 1 : ds.s.rank;
        for (int d = 0; d < ds.s.rank; ++d) o->dims[d] = ds.s.null ? 0 : ds.s.dims[d];
        o->layout = ds.layout;
        if (ds.layout == 2)
            for (int d = 0; d < ds.s.rank; ++d) o->chunk[d] = ds.cdims[d];
        o->n_filters = int32_t(ds.filters.size());
        o->matlab_int_decode = ds.int_decode;
        o->matlab_empty = ds.empty;
        snprintf(o->matlab_class, sizeof(o->matlab_class), "%s", ds.mclass.c_str());
    }
};

// ───────────────────────────── writer ─────────────────────────────

namespace {

struct WGroup {
    std::string name;
    std::vector<std::pair<std::string, uint64_t>> members;
};

// Little-endian byte builder.
struct Buf {
    std::vector<uint8_t> b;
    void u(uint64_t v, int n) {
        for (int i = 0; i < n; ++i) b.push_back(uint8_t(v >> (8 * i)));
    }
    void bytes(const void* p, size_t n) {
        const uint8_t* q = static_cast<const uint8_t*>(p);
        b.insert(b.end(), q, q + n);
    }
    void zeros(size_t n) { b.insert(b.end(), n, 0); }
    void pad_to8() {
        while (b.size() % 8) b.push_back(0);
    }
};

constexpr int GROUP_K = 16;   // group internal-node K (superblock 0 value)
constexpr int CHUNK_K = 32;   // chunk B-tree K (fixed at 32 by superblock 0)

void datatype_bytes(Buf& m, int code) {
    auto fixed = [&](int size, bool sg) {
        m.u(0x10 | 0, 1);
        m.u(sg ? 0x08 : 0x00, 1);
        m.u(0, 2);
        m.u(uint64_t(size), 4);
        m.u(0, 2);
        m.u(uint64_t(8 * size), 2);
    };
    auto flt = [&](int size) {
        m.u(0x10 | 1, 1);
        m.u(0x20, 1);                       // little-endian, implied leading mantissa bit
        m.u(size == 4 ? 31 : 63, 1);        // sign bit position
        m.u(0, 1);
        m.u(uint64_t(size), 4);
        m.u(0, 2);
        m.u(uint64_t(8 * size), 2);
        if (size == 4) {
            m.u(23, 1); m.u(8, 1); m.u(0, 1); m.u(23, 1); m.u(127, 4);
        } else {
            m.u(52, 1); m.u(11, 1); m.u(0, 1); m.u(52, 1); m.u(1023, 4);
        }
    };
    switch (code) {
        case MSLRIO_I8: fixed(1, true); break;
        case MSLRIO_U8: fixed(1, false); break;
        case MSLRIO_I16: fixed(2, true); break;
        case MSLRIO_U16: fixed(2, false); break;
        case MSLRIO_I32: fixed(4, true); break;
        case MSLRIO_U32: fixed(4, false); break;
        case MSLRIO_I64: fixed(8, true); break;
        case MSLRIO_U64: fixed(8, false); break;
        case MSLRIO_F32: flt(4); break;
        case MSLRIO_F64: flt(8); break;
        case MSLRIO_C64:
        case MSLRIO_C128: {
            int fs = code == MSLRIO_C64 ? 4 : 8;
            m.u(0x10 | 6, 1);
            m.u(2, 1);                      // two members
            m.u(0, 2);
            m.u(uint64_t(2 * fs), 4);
            const char* names[2] = {"real", "imag"};
            for (int i = 0; i < 2; ++i) {
                Buf nm;
                nm.bytes(names[i], strlen(names[i]) + 1);
                nm.pad_to8();
                m.bytes(nm.b.data(), nm.b.size());
                m.u(uint64_t(i * fs), 4);   // byte offset
                m.u(0, 1);                  // dimensionality
                m.zeros(3 + 4 + 4 + 16);
                flt(fs);
            }
            break;
        }
        case MSLRIO_REF:
            m.u(0x10 | 7, 1);
            m.u(0, 3);                      // object reference
            m.u(8, 4);
            break;
        default: fail(MSLRIO_ERR_ARG, "unknown element type");
    }
}

void message(Buf& h, int type, const Buf& body, int flags = 0) {
    Buf b = body;
    b.pad_to8();
    h.u(uint64_t(type), 2);
    h.u(b.b.size(), 2);
    h.u(uint64_t(flags), 1);
    h.zeros(3);
    h.bytes(b.b.data(), b.b.size());
}

void scalar_space(Buf& s) {
    s.u(1, 1); s.u(0, 1); s.u(0, 1); s.zeros(5);
}

void attr_string(Buf& h, const char* name, const std::string& v) {
    Buf a, t, s;
    t.u(0x10 | 3, 1); t.u(0, 3); t.u(v.size(), 4);           // null-terminated ASCII
    scalar_space(s);
    size_t nl = strlen(name) + 1;
    a.u(1, 1); a.u(0, 1); a.u(nl, 2); a.u(t.b.size(), 2); a.u(s.b.size(), 2);
    Buf nm; nm.bytes(name, nl); nm.pad_to8();
    a.bytes(nm.b.data(), nm.b.size());
    t.pad_to8(); a.bytes(t.b.data(), t.b.size());
    s.pad_to8(); a.bytes(s.b.data(), s.b.size());
    a.bytes(v.data(), v.size());
    message(h, 0x0C, a);
}

void attr_int(Buf& h, const char* name, int64_t v, int size, bool sg) {
    Buf a, t, s;
    t.u(0x10 | 0, 1); t.u(sg ? 0x08 : 0, 1); t.u(0, 2); t.u(uint64_t(size), 4); t.u(0, 2); t.u(uint64_t(8 * size), 2);
    scalar_space(s);
    size_t nl = strlen(name) + 1;
    a.u(1, 1); a.u(0, 1); a.u(nl, 2); a.u(t.b.size(), 2); a.u(s.b.size(), 2);
    Buf nm; nm.bytes(name, nl); nm.pad_to8();
    a.bytes(nm.b.data(), nm.b.size());
    t.pad_to8(); a.bytes(t.b.data(), t.b.size());
    s.pad_to8(); a.bytes(s.b.data(), s.b.size());
    a.u(uint64_t(v), size);
    message(h, 0x0C, a);
}

}  // namespace

struct mslrio_writer {
    int fd = -1;
    std::string path;
    uint64_t base = 0;                    // absolute offset of the superblock
    std::atomic<uint64_t> end{0};         // next free file address (relative)
    std::vector<WGroup> groups;           // [0] is the root group

    static constexpr uint64_t SUPERBLOCK_BYTES = 96;

    uint64_t alloc(uint64_t n) {
        uint64_t a = end.fetch_add((n + 7) & ~uint64_t(7));
        return a;
    }
    void put(uint64_t addr, const void* p, size_t n) const {
        const uint8_t* q = static_cast<const uint8_t*>(p);
        uint64_t off = base + addr;
        while (n) {
            ssize_t w = pwrite(fd, q, std::min<size_t>(n, size_t(1) << 30), off_t(off));
            if (w <= 0) fail(MSLRIO_ERR_IO, "write failed: " + std::string(strerror(errno)));
            q += w;
            off += uint64_t(w);
            n -= size_t(w);
        }
    }
    uint64_t put_new(const Buf& b) {
        uint64_t a = alloc(b.b.size());
        put(a, b.b.data(), b.b.size());
        return a;
    }

    WGroup& group(const std::string& name) {
        for (auto& g : groups)
            if (g.name == name) return g;
        groups.push_back(WGroup{name, {}});
        return groups.back();
    }

    // Version-1 B-tree over the chunks (already in row-major order).
    uint64_t chunk_btree(const std::vector<std::vector<uint64_t>>& offs, const std::vector<uint64_t>& addrs,
                         const std::vector<uint32_t>& sizes, const std::vector<uint32_t>& masks, int rank,
                         const int64_t* cdims, size_t es) {
        int nd = rank + 1;
        size_t keysz = 8 + 8 * size_t(nd);
        size_t node_bytes = 24 + size_t(2 * CHUNK_K + 1) * keysz + size_t(2 * CHUNK_K) * 8;
        struct Key {
            uint32_t size, mask;
            std::vector<uint64_t> off;
        };
        std::vector<Key> keys;
        for (size_t i = 0; i < addrs.size(); ++i) keys.push_back(Key{sizes[i], masks[i], offs[i]});
        Key endk{0, 0, offs.back()};
        for (int d = 0; d < rank; ++d) endk.off[size_t(d)] += uint64_t(cdims[d]);
        endk.off[size_t(rank)] = es;
        std::vector<uint64_t> child = addrs;
        int level = 0;
        for (;;) {
            size_t n = child.size();
            size_t nn = (n + 2 * CHUNK_K - 1) / (2 * CHUNK_K);
            std::vector<uint64_t> up_addr;
            std::vector<Key> up_key;
            for (size_t j = 0; j < nn; ++j) {
                size_t lo = j * 2 * CHUNK_K, hi = std::min(n, lo + 2 * CHUNK_K);
                Buf b;
                b.bytes("TREE", 4);
                b.u(1, 1);
                b.u(uint64_t(level), 1);
                b.u(hi - lo, 2);
                b.u(UNDEF, 8);
                b.u(UNDEF, 8);
                auto put_key = [&](const Key& k) {
                    b.u(k.size, 4);
                    b.u(k.mask, 4);
                    for (int d = 0; d < nd; ++d) b.u(k.off[size_t(d)], 8);
                };
                for (size_t i = lo; i < hi; ++i) {
                    put_key(keys[i]);
                    b.u(child[i], 8);
                }
                put_key(hi < n ? keys[hi] : endk);
                b.zeros(node_bytes - b.b.size());
                up_addr.push_back(put_new(b));
                up_key.push_back(keys[lo]);
            }
            if (nn == 1) return up_addr[0];
            child.swap(up_addr);
            keys.swap(up_key);
            ++level;
        }
    }

    uint64_t write(const char* name, int dtype, int rank, const int64_t* dims, const void* data,
                   const char* mclass, int int_decode, int empty, int level, int64_t chunk_bytes, int threads) {
        if (!name || !*name) fail(MSLRIO_ERR_ARG, "empty dataset name");
        std::string full(name), gname, vname = full;
        size_t slash = full.find('/');
        if (slash != std::string::npos) {
            gname = full.substr(0, slash);
            vname = full.substr(slash + 1);
            if (gname.empty() || vname.empty() || vname.find('/') != std::string::npos)
                fail(MSLRIO_ERR_ARG, "names may hold one level of group: 'grp/var'");
        }
        int es = dtype_size(dtype);
        if (!es) fail(MSLRIO_ERR_ARG, "unknown element type");
        if (rank < 0 || rank > MSLRIO_MAX_RANK || (rank > 0 && !dims)) fail(MSLRIO_ERR_ARG, "bad rank");
        for (int d = 0; d < rank; ++d)
            if (dims[d] < 0) fail(MSLRIO_ERR_ARG, "negative dimension");
        if (level < 0 || level > 9) fail(MSLRIO_ERR_ARG, "deflate level outside 0-9");
        size_t nbytes = size_t(prod(dims, rank)) * size_t(es);
        if (nbytes && !data) fail(MSLRIO_ERR_ARG, "null data");
        const uint8_t* src = static_cast<const uint8_t*>(data);
        for (auto& g : groups)
            if (g.name == gname)
                for (auto& m : g.members)
                    if (m.first == vname) fail(MSLRIO_ERR_ARG, "duplicate name '" + full + "'");

        Buf layout, filters;
        bool chunked = level > 0 && nbytes > 0 && rank > 0;
        if (!chunked) {
            uint64_t a = UNDEF;
            if (nbytes) {
                a = alloc(nbytes);
                const size_t blk = size_t(64) << 20;
                int64_t nb = int64_t((nbytes + blk - 1) / blk);
                parallel_for(nb, threads, [&](int64_t i) {
                    size_t o = size_t(i) * blk;
                    put(a + o, src + o, std::min(blk, nbytes - o));
                });
            }
            layout.u(3, 1); layout.u(1, 1); layout.u(a, 8); layout.u(nbytes, 8);
        } else {
            int64_t target = chunk_bytes > 0 ? chunk_bytes : (int64_t(4) << 20);
            int64_t cd[MSLRIO_MAX_RANK];
            for (int d = 0; d < rank; ++d) cd[d] = dims[d];
            for (int d = 0; d < rank; ++d) {
                int64_t inner = prod(dims + d + 1, rank - d - 1) * es;
                if (inner >= target) {
                    cd[d] = 1;
                    continue;
                }
                cd[d] = std::min<int64_t>(dims[d], std::max<int64_t>(1, target / inner));
                break;
            }
            for (int d = 0; d < rank; ++d)
                if (cd[d] > 0xffffffffll) fail(MSLRIO_ERR_ARG, "chunk dimension too large");
            size_t cbytes = size_t(prod(cd, rank)) * size_t(es);
            int64_t grid[MSLRIO_MAX_RANK];
            for (int d = 0; d < rank; ++d) grid[d] = (dims[d] + cd[d] - 1) / cd[d];
            int64_t nch = prod(grid, rank);
            std::vector<std::vector<uint64_t>> offs(static_cast<size_t>(nch), std::vector<uint64_t>(static_cast<size_t>(rank) + 1, 0));
            std::vector<uint64_t> addrs(static_cast<size_t>(nch));
            std::vector<uint32_t> sizes(static_cast<size_t>(nch)), masks(static_cast<size_t>(nch));
            parallel_for(nch, threads, [&](int64_t i) {
                thread_local std::vector<uint8_t> raw, z;
                int64_t off[MSLRIO_MAX_RANK], ext[MSLRIO_MAX_RANK];
                int64_t rem = i;
                bool edge = false;
                for (int d = rank - 1; d >= 0; --d) {
                    off[d] = (rem % grid[d]) * cd[d];
                    rem /= grid[d];
                    ext[d] = std::min(cd[d], dims[d] - off[d]);
                    edge |= ext[d] != cd[d];
                }
                raw.resize(cbytes);
                if (edge) memset(raw.data(), 0, cbytes);
                copy_box(raw.data(), cd, const_cast<uint8_t*>(src), dims, off, ext, rank, size_t(es), false);
                uLongf zn = compressBound(uLong(cbytes));
                z.resize(zn);
                int rc = compress2(z.data(), &zn, raw.data(), uLong(cbytes), level);
                if (rc != Z_OK) fail(MSLRIO_ERR_IO, "zlib compress failed");
                const uint8_t* out = z.data();
                size_t on = zn;
                uint32_t mask = 0;
                if (on >= cbytes) {      // does not shrink: store raw, deflate marked skipped
                    out = raw.data();
                    on = cbytes;
                    mask = 1;
                }
                uint64_t a = alloc(on);
                put(a, out, on);
                size_t k = size_t(i);
                addrs[k] = a;
                sizes[k] = uint32_t(on);
                masks[k] = mask;
                for (int d = 0; d < rank; ++d) offs[k][size_t(d)] = uint64_t(off[d]);
            });
            uint64_t bt = chunk_btree(offs, addrs, sizes, masks, rank, cd, size_t(es));
            layout.u(3, 1); layout.u(2, 1); layout.u(uint64_t(rank) + 1, 1); layout.u(bt, 8);
            for (int d = 0; d < rank; ++d) layout.u(uint64_t(cd[d]), 4);
            layout.u(uint64_t(es), 4);
            filters.u(1, 1); filters.u(1, 1); filters.zeros(6);
            filters.u(1, 2);               // deflate
            filters.u(8, 2);               // name length
            filters.u(1, 2);               // optional
            filters.u(1, 2);               // one client value
            filters.bytes("deflate\0", 8);
            filters.u(uint64_t(level), 4);
            filters.zeros(4);
        }

        Buf msgs, sp, dt, fill;
        sp.u(1, 1); sp.u(uint64_t(rank), 1); sp.u(0, 1); sp.zeros(5);
        for (int d = 0; d < rank; ++d) sp.u(uint64_t(dims[d]), 8);
        message(msgs, 0x01, sp);
        datatype_bytes(dt, dtype);
        message(msgs, 0x03, dt, 1);
        fill.u(2, 1); fill.u(chunked ? 3 : 1, 1); fill.u(2, 1); fill.u(0, 1);
        message(msgs, 0x05, fill, 1);
        message(msgs, 0x08, layout);
        if (chunked) message(msgs, 0x0B, filters, 1);
        if (mclass && *mclass) attr_string(msgs, "MATLAB_class", mclass);
        if (int_decode >= 0) attr_int(msgs, "MATLAB_int_decode", int_decode, 4, true);
        if (empty) attr_int(msgs, "MATLAB_empty", 1, 1, false);
        const int nmsgs = 4 + (chunked ? 1 : 0) + ((mclass && *mclass) ? 1 : 0) + (int_decode >= 0 ? 1 : 0) +
                          (empty ? 1 : 0);
        uint64_t oh = object_header(msgs, nmsgs);
        group(gname).members.emplace_back(vname, oh);
        return oh;
    }

    uint64_t object_header(const Buf& msgs, int nmsgs) {
        Buf h;
        h.u(1, 1); h.u(0, 1); h.u(uint64_t(nmsgs), 2); h.u(1, 4); h.u(msgs.b.size(), 4); h.zeros(4);
        h.bytes(msgs.b.data(), msgs.b.size());
        return put_new(h);
    }

    // Local heap, one symbol-table node and a one-leaf B-tree for a group;
    // returns {object header, B-tree, heap} addresses.
    std::array<uint64_t, 3> write_group(WGroup& g, int leaf_k) {
        std::sort(g.members.begin(), g.members.end(),
                  [](const std::pair<std::string, uint64_t>& a, const std::pair<std::string, uint64_t>& b) {
                      return strcmp(a.first.c_str(), b.first.c_str()) < 0;
                  });
        Buf data;
        data.zeros(8);                      // offset 0: the empty name
        std::vector<uint64_t> name_off;
        for (auto& m : g.members) {
            name_off.push_back(data.b.size());
            data.bytes(m.first.c_str(), m.first.size() + 1);
            data.pad_to8();
        }
        uint64_t heap_data = put_new(data);
        Buf heap;
        heap.bytes("HEAP", 4); heap.u(0, 4); heap.u(data.b.size(), 8); heap.u(1, 8); heap.u(heap_data, 8);
        uint64_t heap_addr = put_new(heap);

        uint64_t snod = UNDEF;
        if (!g.members.empty()) {
            Buf s;
            s.bytes("SNOD", 4); s.u(1, 1); s.u(0, 1); s.u(g.members.size(), 2);
            for (size_t i = 0; i < g.members.size(); ++i) {
                s.u(name_off[i], 8); s.u(g.members[i].second, 8); s.u(0, 4); s.u(0, 4); s.zeros(16);
            }
            s.zeros(size_t(2 * leaf_k - int(g.members.size())) * 40);
            snod = put_new(s);
        }
        Buf t;
        t.bytes("TREE", 4); t.u(0, 1); t.u(0, 1); t.u(g.members.empty() ? 0 : 1, 2); t.u(UNDEF, 8); t.u(UNDEF, 8);
        t.u(0, 8);
        if (!g.members.empty()) {
            t.u(snod, 8);
            t.u(name_off.back(), 8);
        }
        t.zeros(24 + size_t(2 * GROUP_K + 1) * 8 + size_t(2 * GROUP_K) * 8 - t.b.size());
        uint64_t tree = put_new(t);
        Buf stab, msgs;
        stab.u(tree, 8); stab.u(heap_addr, 8);
        message(msgs, 0x11, stab);
        return {object_header(msgs, 1), tree, heap_addr};
    }

    void finish() {
        size_t most = 1;
        for (auto& g : groups) most = std::max(most, g.members.size() + (g.name.empty() ? groups.size() : 0));
        int leaf_k = std::max<int>(4, int((most + 1) / 2));
        if (leaf_k > 0xffff) fail(MSLRIO_ERR_ARG, "too many variables in one group");
        for (size_t i = 1; i < groups.size(); ++i) {
            auto r = write_group(groups[i], leaf_k);
            groups[0].members.emplace_back(groups[i].name, r[0]);
        }
        auto root = write_group(groups[0], leaf_k);
        uint64_t eof = base + end.load();
        Buf sb;
        sb.bytes(HDF5_SIG, 8);
        sb.u(0, 1); sb.u(0, 1); sb.u(0, 1); sb.u(0, 1); sb.u(0, 1); sb.u(8, 1); sb.u(8, 1); sb.u(0, 1);
        sb.u(uint64_t(leaf_k), 2); sb.u(GROUP_K, 2); sb.u(0, 4);
        sb.u(base, 8); sb.u(UNDEF, 8); sb.u(eof, 8); sb.u(UNDEF, 8);
        sb.u(0, 8); sb.u(root[0], 8); sb.u(1, 4); sb.u(0, 4); sb.u(root[1], 8); sb.u(root[2], 8);
        if (sb.b.size() != SUPERBLOCK_BYTES) fail(MSLRIO_ERR_IO, "internal: superblock size");
        put(0, sb.b.data(), sb.b.size());
        if (ftruncate(fd, off_t(eof)) != 0) fail(MSLRIO_ERR_IO, "truncate failed");
    }
};

namespace {

int guard(const std::function<void()>& f) {
    try {
        f();
        return MSLRIO_OK;
    } catch (const IoError& e) {
        g_err = e.msg;
        return e.code;
    } catch (const std::bad_alloc&) {
        g_err = "out of host memory";
        return MSLRIO_ERR_IO;
    } catch (const std::exception& e) {
        g_err = e.what();
        return MSLRIO_ERR_IO;
    }
}

void matlab_header(int fd) {
    char text[117];
    time_t now = time(nullptr);
    struct tm tmv;
    gmtime_r(&now, &tmv);
    char date[25];
    if (strftime(date, sizeof(date), "%a %b %e %H:%M:%S %Y", &tmv) == 0) date[0] = 0;
    snprintf(text, sizeof(text), "MATLAB 7.3 MAT-file, Platform: GLNXA64, Created on: %s HDF5 schema 1.00 .", date);
    uint8_t ub[512];
    memset(ub, 0, sizeof(ub));
    memset(ub, ' ', 116);
    memcpy(ub, text, strlen(text));
    ub[124] = 0x00;      // version 0x0200, stored as written by MATLAB
    ub[125] = 0x02;
    ub[126] = 'I';       // endian indicator
    ub[127] = 'M';
    if (pwrite(fd, ub, sizeof(ub), 0) != ssize_t(sizeof(ub))) fail(MSLRIO_ERR_IO, "write failed");
}

}  // namespace

extern "C" {

int mslrio_open(const char* path, mslrio_file** out) {
    return guard([&] {
        if (!path || !out) fail(MSLRIO_ERR_ARG, "null argument");
        *out = nullptr;
        int fd = ::open(path, O_RDONLY | O_CLOEXEC);
        if (fd < 0) fail(MSLRIO_ERR_IO, std::string("cannot open ") + path + ": " + strerror(errno));
        struct stat st;
        if (fstat(fd, &st) != 0 || st.st_size < 8) {
            ::close(fd);
            fail(MSLRIO_ERR_FORMAT, std::string(path) + " is not an HDF5 file");
        }
        size_t size = size_t(st.st_size);
        void* m = mmap(nullptr, size, PROT_READ, MAP_SHARED, fd, 0);
        if (m == MAP_FAILED) {
            ::close(fd);
            fail(MSLRIO_ERR_IO, std::string("mmap failed: ") + strerror(errno));
        }
        madvise(m, size, MADV_WILLNEED);
        auto f = new mslrio_file;
        f->fd = fd;
        f->map = static_cast<const uint8_t*>(m);
        f->size = size;
        try {
            uint64_t off = UNDEF;
            for (uint64_t o = 0; o + 8 <= size; o = o ? o * 2 : 512)
                if (memcmp(f->map + o, HDF5_SIG, 8) == 0) {
                    off = o;
                    break;
                }
            if (off == UNDEF) fail(MSLRIO_ERR_FORMAT, std::string(path) + " is not an HDF5 file (no superblock)");
            Cur c{f->map + off + 8, f->map + size};
            int ver = int(c.u(1));
            if (ver == 0 || ver == 1) {
                c.skip(4);
                f->so = int(c.u(1));
                f->sl = int(c.u(1));
                c.skip(1 + 2 + 2 + 4);
                if (ver == 1) c.skip(4);
            } else if (ver == 2 || ver == 3) {
                f->so = int(c.u(1));
                f->sl = int(c.u(1));
                c.skip(1);
            } else {
                fail(MSLRIO_ERR_UNSUPPORTED, "superblock version " + std::to_string(ver));
            }
            auto ok = [](int s) { return s == 2 || s == 4 || s == 8; };
            if (!ok(f->so) || !ok(f->sl)) fail(MSLRIO_ERR_FORMAT, "bad offset / length sizes");
            c.u(f->so);            // stored base address: addresses are taken relative to the superblock
            f->base = off;
            if (ver <= 1) {
                c.skip(3 * size_t(f->so));
                c.u(f->so);        // root entry: link name offset
                f->root = c.u(f->so);
            } else {
                c.skip(2 * size_t(f->so));
                f->root = c.u(f->so);
            }
            f->header(f->root);
        } catch (...) {
            munmap(const_cast<uint8_t*>(f->map), f->size);
            ::close(f->fd);
            delete f;
            throw;
        }
        *out = f;
    });
}

int mslrio_close(mslrio_file* f) {
    if (!f) return MSLRIO_OK;
    munmap(const_cast<uint8_t*>(f->map), f->size);
    ::close(f->fd);
    delete f;
    return MSLRIO_OK;
}

int mslrio_userblock(const mslrio_file* f, uint64_t* bytes) {
    return guard([&] {
        if (!f || !bytes) fail(MSLRIO_ERR_ARG, "null argument");
        *bytes = f->base;
    });
}

int mslrio_group_count(mslrio_file* f, const char* group, int32_t* n) {
    return guard([&] {
        if (!f || !n) fail(MSLRIO_ERR_ARG, "null argument");
        *n = int32_t(f->members(f->lookup(group ? group : "/")).size());
    });
}

int mslrio_group_name(mslrio_file* f, const char* group, int32_t i, char* buf, size_t cap) {
    return guard([&] {
        if (!f || !buf || !cap) fail(MSLRIO_ERR_ARG, "null argument");
        auto m = f->members(f->lookup(group ? group : "/"));
        if (i < 0 || size_t(i) >= m.size()) fail(MSLRIO_ERR_ARG, "member index out of range");
        if (m[size_t(i)].first.size() + 1 > cap) fail(MSLRIO_ERR_ARG, "name buffer too small");
        memcpy(buf, m[size_t(i)].first.c_str(), m[size_t(i)].first.size() + 1);
    });
}

int mslrio_lookup(mslrio_file* f, const char* path, uint64_t* addr) {
    return guard([&] {
        if (!f || !addr) fail(MSLRIO_ERR_ARG, "null argument");
        *addr = f->lookup(path);
    });
}

int mslrio_info_at(mslrio_file* f, uint64_t addr, mslrio_info* info) {
    return guard([&] {
        if (!f || !info) fail(MSLRIO_ERR_ARG, "null argument");
        f->info(addr, info);
    });
}

int mslrio_read_at(mslrio_file* f, uint64_t addr, void* dst, size_t dst_bytes, int32_t nthreads) {
    return guard([&] {
        if (!f || (!dst && dst_bytes)) fail(MSLRIO_ERR_ARG, "null argument");
        f->read(addr, static_cast<uint8_t*>(dst), dst_bytes, nthreads);
    });
}

int mslrio_create(const char* path, int32_t matlab, mslrio_writer** out) {
    return guard([&] {
        if (!path || !out) fail(MSLRIO_ERR_ARG, "null argument");
        *out = nullptr;
        int fd = ::open(path, O_RDWR | O_CREAT | O_TRUNC | O_CLOEXEC, 0644);
        if (fd < 0) fail(MSLRIO_ERR_IO, std::string("cannot create ") + path + ": " + strerror(errno));
        auto w = new mslrio_writer;
        w->fd = fd;
        w->path = path;
        w->base = matlab ? 512 : 0;
        w->end = mslrio_writer::SUPERBLOCK_BYTES;
        w->groups.push_back(WGroup{"", {}});
        try {
            if (matlab) matlab_header(fd);
        } catch (...) {
            ::close(fd);
            unlink(path);
            delete w;
            throw;
        }
        *out = w;
    });
}

int mslrio_write(mslrio_writer* w, const char* name, int32_t dtype, int32_t rank, const int64_t* dims,
                 const void* data, const char* matlab_class, int32_t matlab_int_decode, int32_t matlab_empty,
                 int32_t deflate_level, int64_t chunk_bytes, int32_t nthreads, uint64_t* addr) {
    return guard([&] {
        if (!w) fail(MSLRIO_ERR_ARG, "null writer");
        uint64_t a = w->write(name, dtype, rank, dims, data, matlab_class, matlab_int_decode, matlab_empty,
                              deflate_level, chunk_bytes, nthreads);
        if (addr) *addr = a;
    });
}

int mslrio_finish(mslrio_writer* w) {
    if (!w) return MSLRIO_OK;
    int rc = guard([&] { w->finish(); });
    if (::close(w->fd) != 0 && rc == MSLRIO_OK) {
        g_err = "close failed";
        rc = MSLRIO_ERR_IO;
    }
    delete w;
    return rc;
}

int mslrio_abort(mslrio_writer* w) {
    if (!w) return MSLRIO_OK;
    ::close(w->fd);
    unlink(w->path.c_str());
    delete w;
    return MSLRIO_OK;
}

const char* mslrio_last_error(void) { return g_err.c_str(); }

}  // extern "C"
