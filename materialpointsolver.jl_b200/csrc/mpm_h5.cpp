// mpm_h5.cpp -- snapshot files in the HDF5 format, written without libhdf5.
//
// submit_work! (src/solver.jl:54-111) writes, through HDF5.jl, one group
// "group<i>" per snapshot holding the particle fields as datasets, then a few
// root-level datasets (FILE_NUM, grid_coords, mp_coords0, nid, vbc_*).  This
// writer produces the same tree: groups of contiguous, uncompressed datasets
// of IEEE little-endian floats or two's-complement integers.
//
// File structure (HDF5 file format specification, "version 0" objects, the
// form libhdf5 writes with its default, earliest-format settings):
//   * superblock version 0 at address 0 (8-byte offsets and lengths), whose
//     root symbol-table entry caches the root group's B-tree and heap;
//   * every object header is version 1 (16-byte prefix, 8-byte aligned
//     messages);
//   * a group is an object header with one symbol-table message that points
//     at a version-1 B-tree (node type 0, a single leaf-level node) whose
//     children are symbol-table nodes ("SNOD") listing the members in name
//     order, and at a local heap ("HEAP") holding the member names;
//   * a dataset is an object header with a dataspace (version 1), a datatype
//     (version 1, class 0 fixed-point or 1 floating-point) and a data-layout
//     message (version 3, contiguous), the raw data stored before it.
// Datasets are written when they arrive; groups, being small, are written
// when the file is closed, and the superblock last of all, so the file only
// becomes readable once mpm_h5_close() returned.
//
// Dimensions are given slowest-varying first (the HDF5 order).  HDF5.jl
// writes a Julia (column-major) np x k matrix as the dataspace (k, np), so the
// column-major buffer of such a matrix is passed with dims = {k, np}.
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/mpm_b200.h"

namespace mpm_detail {
void set_global_error(const std::string &m);
}

namespace {

constexpr uint64_t UNDEF = ~0ull;          // the undefined address
constexpr uint64_t HEAP_FREE_NULL = 1;     // "no free block" in a local heap header
constexpr int INTERNAL_K = 16;             // B-tree node: up to 2K children
constexpr uint64_t SUPERBLOCK_BYTES = 96;

struct Buf {
    std::vector<uint8_t> b;
    void u8(uint32_t v) { b.push_back((uint8_t)v); }
    void u16(uint32_t v) { for (int i = 0; i < 2; ++i) b.push_back((uint8_t)(v >> (8 * i))); }
    void u32(uint32_t v) { for (int i = 0; i < 4; ++i) b.push_back((uint8_t)(v >> (8 * i))); }
    void u64(uint64_t v) { for (int i = 0; i < 8; ++i) b.push_back((uint8_t)(v >> (8 * i))); }
    void raw(const void *p, size_t n) { b.insert(b.end(), (const uint8_t *)p, (const uint8_t *)p + n); }
    void zeros(size_t n) { b.insert(b.end(), n, 0); }
    void pad8() { while (b.size() % 8) b.push_back(0); }
    size_t size() const { return b.size(); }
};

// One header message: type, size of the (8-byte padded) body, flags 0.
void message(Buf &oh, uint32_t type, const Buf &body) {
    Buf p = body;
    p.pad8();
    oh.u16(type);
    oh.u16((uint32_t)p.size());
    oh.u8(0);
    oh.zeros(3);
    oh.raw(p.b.data(), p.size());
}

// Version-1 object header around the given message bytes.
Buf object_header(uint32_t nmsg, const Buf &msgs) {
    Buf oh;
    oh.u8(1);            // version
    oh.u8(0);            // reserved
    oh.u16(nmsg);
    oh.u32(1);           // reference count
    oh.u32((uint32_t)msgs.size());
    oh.zeros(4);         // pad the prefix to 16 bytes
    oh.raw(msgs.b.data(), msgs.size());
    return oh;
}

struct Obj {
    bool group = true;
    uint64_t header = UNDEF;             // object header address
    std::map<std::string, Obj> kids;     // byte-wise name order = the order the B-tree needs
};

}  // namespace

struct mpm_h5 {
    FILE *f = nullptr;
    uint64_t eof = SUPERBLOCK_BYTES;
    Obj root;
    std::mutex mu;
    std::string path;
};

namespace {

bool put(mpm_h5 *h, uint64_t addr, const void *p, size_t n) {
    if (fseeko(h->f, (off_t)addr, SEEK_SET) != 0) return false;
    return n == 0 || fwrite(p, 1, n, h->f) == n;
}

// Appends at the end of the file (8-byte aligned); returns the address.
uint64_t append(mpm_h5 *h, const void *p, size_t n, bool *ok) {
    uint64_t a = (h->eof + 7) & ~7ull;
    if (a != h->eof) {
        static const uint8_t z[8] = {0};
        *ok = *ok && put(h, h->eof, z, a - h->eof);
    }
    *ok = *ok && put(h, a, p, n);
    h->eof = a + n;
    return a;
}

size_t elem_size(int32_t type) {
    switch (type) {
    case MPM_T_F64: case MPM_T_I64: return 8;
    case MPM_T_F32: case MPM_T_I32: return 4;
    default: return 0;
    }
}

Buf datatype_body(int32_t type) {
    Buf t;
    if (type == MPM_T_F64 || type == MPM_T_F32) {
        const bool d = type == MPM_T_F64;
        t.u8(0x11);                      // version 1, class 1 (floating point)
        t.u8(0x20);                      // little-endian, zero padding, implied mantissa msb
        t.u8(d ? 63 : 31);               // sign bit position
        t.u8(0);
        t.u32(d ? 8 : 4);                // size in bytes
        t.u16(0);                        // bit offset
        t.u16(d ? 64 : 32);              // precision
        t.u8(d ? 52 : 23);               // exponent location
        t.u8(d ? 11 : 8);                // exponent size
        t.u8(0);                         // mantissa location
        t.u8(d ? 52 : 23);               // mantissa size
        t.u32(d ? 1023 : 127);           // exponent bias
    } else {
        t.u8(0x10);                      // version 1, class 0 (fixed point)
        t.u8(0x08);                      // little-endian, signed
        t.u8(0);
        t.u8(0);
        t.u32((uint32_t)elem_size(type));
        t.u16(0);                        // bit offset
        t.u16((uint32_t)(8 * elem_size(type)));
    }
    return t;
}

// Finds (creating groups on the way) the parent group of `path` and the leaf name.
Obj *parent_of(mpm_h5 *h, const std::string &path, std::string *leaf) {
    Obj *g = &h->root;
    size_t s = 0;
    while (true) {
        size_t e = path.find('/', s);
        if (e == std::string::npos) {
            *leaf = path.substr(s);
            return g;
        }
        std::string part = path.substr(s, e - s);
        if (part.empty()) return nullptr;
        Obj &k = g->kids[part];
        if (!k.group) return nullptr;   // a dataset of that name exists
        g = &k;
        s = e + 1;
    }
}

// Writes the heap, symbol-table nodes, B-tree and object header of `g`
// (children first).  leaf_k: the file's group leaf-node K.
bool write_group(mpm_h5 *h, Obj &g, int leaf_k) {
    bool ok = true;
    for (auto &kv : g.kids)
        if (kv.second.group && !write_group(h, kv.second, leaf_k)) return false;
    // local heap: offset 0 holds the empty string (the B-tree's left-most key)
    Buf heap;
    heap.zeros(8);
    std::vector<uint64_t> name_off;
    for (auto &kv : g.kids) {
        name_off.push_back(heap.size());
        heap.raw(kv.first.data(), kv.first.size());
        heap.u8(0);
        heap.pad8();
    }
    Buf hh;
    hh.raw("HEAP", 4);
    hh.u8(0);
    hh.zeros(3);
    hh.u64(heap.size());
    hh.u64(HEAP_FREE_NULL);
    const uint64_t heap_hdr = (h->eof + 7) & ~7ull;
    hh.u64(heap_hdr + 32);               // data segment follows the 32-byte header
    hh.raw(heap.b.data(), heap.size());
    if (append(h, hh.b.data(), hh.size(), &ok) != heap_hdr) return false;
    // symbol-table nodes of up to 2*leaf_k entries each
    const size_t cap = 2 * (size_t)leaf_k, n = g.kids.size();
    const size_t nsnod = (n + cap - 1) / cap;
    if (nsnod > 2 * (size_t)INTERNAL_K) return false;
    std::vector<uint64_t> snod_addr, snod_key;
    auto it = g.kids.begin();
    for (size_t s = 0; s < nsnod; ++s) {
        const size_t cnt = std::min(cap, n - s * cap);
        Buf sn;
        sn.raw("SNOD", 4);
        sn.u8(1);
        sn.u8(0);
        sn.u16((uint32_t)cnt);
        for (size_t j = 0; j < cnt; ++j, ++it) {
            const size_t idx = s * cap + j;
            sn.u64(name_off[idx]);
            sn.u64(it->second.header);
            sn.u32(0);                   // no cached scratch data
            sn.u32(0);
            sn.zeros(16);
            if (j + 1 == cnt) snod_key.push_back(name_off[idx]);
        }
        sn.zeros((cap - cnt) * 40);
        snod_addr.push_back(append(h, sn.b.data(), sn.size(), &ok));
    }
    // one leaf-level B-tree node: key0 = "" < child0 <= key1 < child1 <= key2 ...
    Buf bt;
    bt.raw("TREE", 4);
    bt.u8(0);                            // group node
    bt.u8(0);                            // leaf level
    bt.u16((uint32_t)nsnod);
    bt.u64(UNDEF);
    bt.u64(UNDEF);
    bt.u64(0);
    for (size_t s = 0; s < nsnod; ++s) {
        bt.u64(snod_addr[s]);
        bt.u64(snod_key[s]);
    }
    bt.zeros((2 * INTERNAL_K - nsnod) * 16);
    const uint64_t btree = append(h, bt.b.data(), bt.size(), &ok);
    Buf stab;
    stab.u64(btree);
    stab.u64(heap_hdr);
    Buf msgs;
    message(msgs, 0x0011, stab);
    Buf oh = object_header(1, msgs);
    g.header = append(h, oh.b.data(), oh.size(), &ok);
    // the root's B-tree and heap are cached in the superblock's root entry
    if (&g == &h->root) {
        Buf sb;
        sb.raw("\x89HDF\r\n\x1a\n", 8);
        sb.u8(0);                        // superblock version
        sb.u8(0);                        // free-space storage version
        sb.u8(0);                        // root group symbol table entry version
        sb.u8(0);
        sb.u8(0);                        // shared header message format version
        sb.u8(8);                        // size of offsets
        sb.u8(8);                        // size of lengths
        sb.u8(0);
        sb.u16((uint32_t)leaf_k);
        sb.u16(INTERNAL_K);
        sb.u32(0);                       // file consistency flags
        sb.u64(0);                       // base address
        sb.u64(UNDEF);                   // free-space info
        sb.u64(h->eof);                  // end of file
        sb.u64(UNDEF);                   // driver information block
        sb.u64(0);                       // root entry: link name offset
        sb.u64(g.header);
        sb.u32(1);                       // cache type 1: scratch = B-tree, heap
        sb.u32(0);
        sb.u64(btree);
        sb.u64(heap_hdr);
        ok = ok && sb.size() == SUPERBLOCK_BYTES && put(h, 0, sb.b.data(), sb.size());
    }
    return ok;
}

size_t max_members(const Obj &g) {
    size_t m = g.kids.size();
    for (auto &kv : g.kids)
        if (kv.second.group) m = std::max(m, max_members(kv.second));
    return m;
}

int h5_fail(const std::string &m) {
    mpm_detail::set_global_error(m);
    return MPM_E_ARG;
}

}  // namespace

extern "C" {

int mpm_h5_create(const char *path, mpm_h5 **out) {
    if (!path || !out) return h5_fail("mpm_h5_create: null argument");
    *out = nullptr;
    std::unique_ptr<mpm_h5> h(new (std::nothrow) mpm_h5);
    if (!h) return h5_fail("mpm_h5_create: out of host memory");
    h->f = std::fopen(path, "wb+");
    if (!h->f) return h5_fail(std::string("mpm_h5_create: cannot create ") + path);
    static const uint8_t z[SUPERBLOCK_BYTES] = {0};
    if (!put(h.get(), 0, z, sizeof(z))) {
        std::fclose(h->f);
        return h5_fail(std::string("mpm_h5_create: cannot write ") + path);
    }
    h->path = path;
    *out = h.release();
    return MPM_OK;
}

int mpm_h5_write(mpm_h5 *h, const char *name, int32_t type, int32_t rank, const int64_t *dims,
                 const void *data) {
    if (!h || !name) return h5_fail("mpm_h5_write: null argument");
    const size_t es = elem_size(type);
    if (!es) return h5_fail("mpm_h5_write: unknown element type");
    if (rank < 0 || rank > 8 || (rank > 0 && !dims)) return h5_fail("mpm_h5_write: bad rank");
    uint64_t n = 1;
    for (int r = 0; r < rank; ++r) {
        if (dims[r] < 0) return h5_fail("mpm_h5_write: negative dimension");
        n *= (uint64_t)dims[r];
    }
    if (n && !data) return h5_fail("mpm_h5_write: null data");
    std::lock_guard<std::mutex> lk(h->mu);
    std::string leaf;
    Obj *parent = parent_of(h, name, &leaf);
    if (!parent || leaf.empty()) return h5_fail(std::string("mpm_h5_write: bad dataset path ") + name);
    if (parent->kids.count(leaf)) return h5_fail(std::string("mpm_h5_write: ") + name + " exists");
    bool ok = true;
    const uint64_t bytes = n * es;
    const uint64_t addr = bytes ? append(h, data, bytes, &ok) : UNDEF;
    Buf space;
    space.u8(1);                         // version
    space.u8((uint32_t)rank);
    space.u8(0);                         // no maximum dimensions
    space.zeros(5);
    for (int r = 0; r < rank; ++r) space.u64((uint64_t)dims[r]);
    Buf layout;
    layout.u8(3);                        // version
    layout.u8(1);                        // contiguous
    layout.u64(addr);
    layout.u64(bytes);
    Buf msgs;
    message(msgs, 0x0001, space);
    message(msgs, 0x0003, datatype_body(type));
    message(msgs, 0x0008, layout);
    Buf oh = object_header(3, msgs);
    Obj d;
    d.group = false;
    d.header = append(h, oh.b.data(), oh.size(), &ok);
    if (!ok) return h5_fail("mpm_h5_write: write to " + h->path + " failed");
    parent->kids.emplace(leaf, std::move(d));
    return MPM_OK;
}

int mpm_h5_close(mpm_h5 *h) {
    if (!h) return MPM_OK;
    int rc = MPM_OK;
    {
        std::lock_guard<std::mutex> lk(h->mu);
        const size_t m = max_members(h->root);
        const int leaf_k = (int)std::max<size_t>(4, (m + 4 * INTERNAL_K - 1) / (4 * INTERNAL_K));
        if (leaf_k > 32767) rc = h5_fail("mpm_h5_close: too many members in one group");
        else if (!write_group(h, h->root, leaf_k) || std::fflush(h->f) != 0)
            rc = h5_fail("mpm_h5_close: write to " + h->path + " failed");
        if (std::fclose(h->f) != 0 && rc == MPM_OK) rc = h5_fail("mpm_h5_close: close failed");
    }
    delete h;
    return rc;
}

}  // extern "C"
