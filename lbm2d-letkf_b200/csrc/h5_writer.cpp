// h5_writer.cpp -- a minimal HDF5 writer for the LETKF matrix dumps: one file holding
// one contiguous dataset "data" of rank 3, float32 or float64, little-endian.  It
// replaces H5Fcreate + H5LTmake_dataset (cu_matrix.hpp:108-117) without libhdf5.
//
// File structure (HDF5 file format specification, version 0 superblock, the layout
// libhdf5 itself writes by default):
//   0     superblock v0 (offsets and lengths of 8 bytes, group K 4 / 16) whose root
//         symbol-table entry caches the root group's B-tree and local heap
//   96    root group object header v1: one symbol-table message
//   136   local heap "HEAP": names "" at 0 and "data" at 8, one free block at 16
//   256   v1 B-tree "TREE" node (group, leaf, one child): 544 bytes for K = 16
//   800   symbol-table node "SNOD" with the entry "data": 328 bytes for K = 4
//   1128  dataset object header v1: dataspace v1, datatype v1 (IEEE float),
//         fill value v2 (undefined), layout v3 (contiguous)
//   1264  the raw data, dims {d0, d1, d2} in C order over the caller's buffer
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "lbl_internal.h"

namespace lbl {
namespace {

constexpr uint64_t kUndef = ~uint64_t(0);
constexpr uint64_t kHeapFreeNull = 1;  // end of a local-heap free list (offsets are multiples of 8)

struct Buf {
    std::vector<uint8_t> b;
    void u8(uint64_t v) { b.push_back(uint8_t(v)); }
    void u16(uint64_t v) { for (int i = 0; i < 2; i++) b.push_back(uint8_t(v >> (8 * i))); }
    void u32(uint64_t v) { for (int i = 0; i < 4; i++) b.push_back(uint8_t(v >> (8 * i))); }
    void u64(uint64_t v) { for (int i = 0; i < 8; i++) b.push_back(uint8_t(v >> (8 * i))); }
    void bytes(const char* s, size_t n) { b.insert(b.end(), s, s + n); }
    void pad_to(size_t n) { if (b.size() < n) b.resize(n, 0); }
    size_t size() const { return b.size(); }
};

// v1 object header message: type, size, flags, 3 reserved, data padded to 8 bytes
void message(Buf& o, uint16_t type, uint8_t flags, const Buf& data) {
    const size_t n = (data.size() + 7) & ~size_t(7);
    o.u16(type);
    o.u16(n);
    o.u8(flags);
    o.u8(0); o.u8(0); o.u8(0);
    o.b.insert(o.b.end(), data.b.begin(), data.b.end());
    o.pad_to(o.size() + (n - data.size()));
}

}  // namespace

int write_h5_dataset(const std::string& path, const uint64_t dims[3], const void* data, bool is_double,
                     std::string& err) {
    const uint64_t esize = is_double ? 8 : 4;
    const uint64_t nbytes = dims[0] * dims[1] * dims[2] * esize;
    const uint64_t a_root = 96, a_heap = 136, a_heap_data = 168, heap_size = 88, a_tree = 256, a_snod = 800,
                   a_dset = 1128, a_data = 1264;
    const uint64_t eof = a_data + nbytes;
    Buf f;
    // superblock v0
    const char sig[8] = {'\x89', 'H', 'D', 'F', '\r', '\n', '\x1a', '\n'};
    f.bytes(sig, 8);
    f.u8(0); f.u8(0); f.u8(0); f.u8(0);  // superblock, free space, root entry, reserved
    f.u8(0); f.u8(8); f.u8(8); f.u8(0);  // shared header version, sizeof offsets, sizeof lengths, reserved
    f.u16(4); f.u16(16);                 // group leaf node K, group internal node K
    f.u32(0);                            // file consistency flags
    f.u64(0); f.u64(kUndef); f.u64(eof); f.u64(kUndef);  // base, free space, end of file, driver info
    f.u64(0); f.u64(a_root); f.u32(1); f.u32(0); f.u64(a_tree); f.u64(a_heap);  // root symbol-table entry
    // root group object header v1: the symbol-table message (B-tree, heap)
    {
        Buf msgs, st;
        st.u64(a_tree);
        st.u64(a_heap);
        message(msgs, 0x0011, 0, st);
        f.u8(1); f.u8(0); f.u16(1); f.u32(1); f.u32(msgs.size()); f.u32(0);
        f.b.insert(f.b.end(), msgs.b.begin(), msgs.b.end());
    }
    // local heap and its data segment
    f.pad_to(a_heap);
    f.bytes("HEAP", 4); f.u8(0); f.u8(0); f.u8(0); f.u8(0);
    f.u64(heap_size); f.u64(16); f.u64(a_heap_data);
    f.pad_to(a_heap_data);
    f.pad_to(a_heap_data + 8);                 // offset 0: ""
    f.bytes("data\0\0\0\0", 8);                // offset 8: "data"
    f.u64(kHeapFreeNull); f.u64(heap_size - 16);  // offset 16: free block (next, size)
    f.pad_to(a_heap_data + heap_size);
    // v1 B-tree node for the group: keys are heap offsets, one child (the SNOD)
    f.pad_to(a_tree);
    f.bytes("TREE", 4); f.u8(0); f.u8(0); f.u16(1); f.u64(kUndef); f.u64(kUndef);
    f.u64(0); f.u64(a_snod); f.u64(8);
    f.pad_to(a_tree + 24 + 2 * 16 * 8 + (2 * 16 + 1) * 8);
    // symbol-table node with the entry "data"
    f.pad_to(a_snod);
    f.bytes("SNOD", 4); f.u8(1); f.u8(0); f.u16(1);
    f.u64(8); f.u64(a_dset); f.u32(0); f.u32(0); f.u64(0); f.u64(0);
    f.pad_to(a_snod + 8 + 2 * 4 * 40);
    // dataset object header v1
    f.pad_to(a_dset);
    {
        Buf msgs, space, type, fill, layout;
        space.u8(1); space.u8(3); space.u8(0); space.u8(0); space.u32(0);
        for (int d = 0; d < 3; d++) space.u64(dims[d]);
        message(msgs, 0x0001, 0, space);
        type.u8(0x11);                                   // version 1, class 1 (floating point)
        type.u8(0x20); type.u8(is_double ? 63 : 31); type.u8(0);  // LE, implied-msb mantissa, sign bit
        type.u32(esize);
        type.u16(0); type.u16(esize * 8);                // bit offset, precision
        type.u8(is_double ? 52 : 23); type.u8(is_double ? 11 : 8);  // exponent location, size
        type.u8(0); type.u8(is_double ? 52 : 23);        // mantissa location, size
        type.u32(is_double ? 1023 : 127);                // exponent bias
        message(msgs, 0x0003, 1, type);
        fill.u8(2); fill.u8(2); fill.u8(2); fill.u8(0);  // version 2, late allocation, fill if set, undefined
        message(msgs, 0x0005, 1, fill);
        layout.u8(3); layout.u8(1); layout.u64(a_data); layout.u64(nbytes);  // version 3, contiguous
        message(msgs, 0x0008, 0, layout);
        f.u8(1); f.u8(0); f.u16(4); f.u32(1); f.u32(msgs.size()); f.u32(0);
        f.b.insert(f.b.end(), msgs.b.begin(), msgs.b.end());
    }
    if (f.size() != a_data) {
        err = "internal HDF5 layout error";
        return LBL_ERR_IO;
    }
    std::FILE* fp = std::fopen(path.c_str(), "wb");
    if (!fp) {
        err = "could not open file: " + path;
        return LBL_ERR_IO;
    }
    bool ok = std::fwrite(f.b.data(), 1, f.size(), fp) == f.size();
    ok = ok && (nbytes == 0 || std::fwrite(data, 1, nbytes, fp) == nbytes);
    ok = (std::fclose(fp) == 0) && ok;
    if (!ok) {
        err = "could not write h5 data: " + path;
        return LBL_ERR_IO;
    }
    return LBL_OK;
}

}  // namespace lbl
