// h5_writer.cpp — HDF5 file of 1-D datasets in the root group (h5_writer.h).
//
// Layout of the file (every address absolute, base address 0, 8-byte offsets
// and lengths, all structures on 8-byte boundaries):
//   superblock version 0 (root symbol-table entry caching the B-tree and heap)
//   root group object header (version 1): one Symbol Table message
//   local heap: header, then the data segment with "" at offset 0 and every
//     dataset name, NUL-terminated and padded to 8 bytes; empty free list
//   one version-1 B-tree leaf node of group type over the symbol-table nodes
//   symbol-table nodes (up to 2 * kLeafK entries each, names in byte order)
//   one object header per dataset: Dataspace, Datatype, Fill Value, Layout
//   the raw data of each dataset, contiguous
#include "h5_writer.h"

#include <algorithm>
#include <cstdio>
#include <cstring>

namespace cupf_host {

namespace {

constexpr uint64_t kUndef = ~0ull;
constexpr int kLeafK = 16;  // symbol-table node capacity = 2 * kLeafK entries
constexpr int kNodeK = 16;  // group B-tree node capacity = 2 * kNodeK children
constexpr size_t kSuperblock = 96;
constexpr size_t kHeapHeader = 32;
constexpr size_t kBtreeNode = 8 + 2 * 8 + (2 * kNodeK + 1) * 8 + 2 * kNodeK * 8;
constexpr size_t kEntry = 40;  // symbol-table entry
constexpr size_t kSnod = 8 + 2 * kLeafK * kEntry;
constexpr size_t kFreeNull = 1;  // terminator of a local heap's free list

size_t pad8(size_t n) { return (n + 7) & ~size_t(7); }

struct Buf {
  std::string s;
  void u8(uint8_t v) { s.push_back((char)v); }
  void u16(uint16_t v) { for (int i = 0; i < 2; ++i) u8((uint8_t)(v >> (8 * i))); }
  void u32(uint32_t v) { for (int i = 0; i < 4; ++i) u8((uint8_t)(v >> (8 * i))); }
  void u64(uint64_t v) { for (int i = 0; i < 8; ++i) u8((uint8_t)(v >> (8 * i))); }
  void bytes(const void* p, size_t n) { s.append(static_cast<const char*>(p), n); }
  void zeros(size_t n) { s.append(n, '\0'); }
  void pad_to(size_t n) { if (s.size() < n) zeros(n - s.size()); }
};

// header message of a version-1 object header: type, size of the (8-byte
// padded) data, flags, 3 reserved bytes, data
void message(Buf& b, uint16_t type, const Buf& data) {
  const size_t n = pad8(data.s.size());
  b.u16(type);
  b.u16((uint16_t)n);
  b.u8(0);
  b.zeros(3);
  b.bytes(data.s.data(), data.s.size());
  b.zeros(n - data.s.size());
}

// version-1 object header prefix: version, reserved, message count, reference
// count, size of the message data, then 4 bytes so messages start 8-aligned
void object_header(Buf& b, uint16_t nmsgs, const Buf& msgs) {
  b.u8(1);
  b.u8(0);
  b.u16(nmsgs);
  b.u32(1);
  b.u32((uint32_t)msgs.s.size());
  b.zeros(4);
  b.bytes(msgs.s.data(), msgs.s.size());
}

Buf datatype(char kind, size_t elem) {
  Buf d;
  if (kind == 'i') {
    d.u8(0x10);  // version 1, class 0 (fixed point)
    d.u8(0x08);  // little endian, signed
    d.u8(0);
    d.u8(0);
    d.u32((uint32_t)elem);
    d.u16(0);                     // bit offset
    d.u16((uint16_t)(8 * elem));  // bit precision
  } else {
    const bool dbl = elem == 8;
    d.u8(0x11);  // version 1, class 1 (floating point)
    d.u8(0x20);  // little endian, no padding, implied leading mantissa bit
    d.u8(dbl ? 63 : 31);  // sign bit position
    d.u8(0);
    d.u32((uint32_t)elem);
    d.u16(0);                        // bit offset
    d.u16((uint16_t)(8 * elem));     // bit precision
    d.u8(dbl ? 52 : 23);             // exponent location
    d.u8(dbl ? 11 : 8);              // exponent size
    d.u8(0);                         // mantissa location
    d.u8(dbl ? 52 : 23);             // mantissa size
    d.u32(dbl ? 1023u : 127u);       // exponent bias
  }
  return d;
}

}  // namespace

void H5Writer::add_raw(const std::string& name, char kind, const void* data, size_t count,
                       size_t elem) {
  Entry e;
  e.name = name;
  e.kind = kind;
  e.elem = elem;
  e.count = count;
  e.data.assign(static_cast<const char*>(data), count * elem);
  mEntries.push_back(std::move(e));
}

void H5Writer::add(const std::string& name, const std::vector<float>& v) {
  add_raw(name, 'f', v.data(), v.size(), sizeof(float));
}

void H5Writer::add(const std::string& name, const std::vector<int>& v) {
  add_raw(name, 'i', v.data(), v.size(), sizeof(int));
}

void H5Writer::add(const std::string& name, const std::vector<double>& v) {
  add_raw(name, 'f', v.data(), v.size(), sizeof(double));
}

std::string H5Writer::bytes() const {
  // names in byte order (the order of the symbol-table nodes and B-tree keys);
  // a repeated name keeps the last array added under it
  std::vector<const Entry*> ents;
  for (const Entry& e : mEntries) {
    auto it = std::find_if(ents.begin(), ents.end(),
                           [&](const Entry* x) { return x->name == e.name; });
    if (it != ents.end()) *it = &e;
    else ents.push_back(&e);
  }
  std::sort(ents.begin(), ents.end(), [](const Entry* a, const Entry* b) {
    return std::strcmp(a->name.c_str(), b->name.c_str()) < 0;
  });
  const size_t n = ents.size();
  const size_t nsnod = std::max<size_t>(1, (n + 2 * kLeafK - 1) / (2 * kLeafK));
  if (nsnod > 2 * kNodeK) return std::string();

  // local heap data: "" at 0, then the names
  Buf heap;
  heap.zeros(8);
  std::vector<uint64_t> name_off(n);
  for (size_t i = 0; i < n; ++i) {
    name_off[i] = heap.s.size();
    heap.bytes(ents[i]->name.c_str(), ents[i]->name.size() + 1);
    heap.pad_to(pad8(heap.s.size()));
  }

  // addresses
  const uint64_t a_root = kSuperblock;
  const uint64_t a_heap = a_root + 16 + 8 + 16;
  const uint64_t a_heapdata = a_heap + kHeapHeader;
  const uint64_t a_btree = a_heapdata + heap.s.size();
  const uint64_t a_snod = a_btree + kBtreeNode;
  uint64_t p = a_snod + nsnod * kSnod;
  std::vector<Buf> headers(n);
  std::vector<uint64_t> a_hdr(n), a_data(n);
  for (size_t i = 0; i < n; ++i) {
    const Entry& e = *ents[i];
    a_hdr[i] = p;
    Buf msgs;
    Buf ds;  // Dataspace version 1: rank 1, no maximum dimensions
    ds.u8(1);
    ds.u8(1);
    ds.u8(0);
    ds.zeros(5);
    ds.u64(e.count);
    message(msgs, 0x0001, ds);
    message(msgs, 0x0003, datatype(e.kind, e.elem));
    Buf fv;  // Fill Value version 1: late allocation, fill if set, default value
    fv.u8(1);
    fv.u8(2);
    fv.u8(2);
    fv.u8(1);
    fv.u32(0);
    message(msgs, 0x0005, fv);
    Buf lay;  // Data Layout version 3, contiguous: address, size (filled in below)
    lay.u8(3);
    lay.u8(1);
    lay.u64(0);
    lay.u64(e.data.size());
    message(msgs, 0x0008, lay);
    object_header(headers[i], 4, msgs);
    p += headers[i].s.size();
  }
  for (size_t i = 0; i < n; ++i) {
    a_data[i] = p;
    p = pad8(p + ents[i]->data.size());
  }
  const uint64_t eof = p;

  Buf f;
  // superblock version 0
  f.bytes("\x89HDF\r\n\x1a\n", 8);
  f.u8(0);  // superblock version
  f.u8(0);  // free-space storage version
  f.u8(0);  // root group symbol table entry version
  f.u8(0);
  f.u8(0);  // shared header message format version
  f.u8(8);  // size of offsets
  f.u8(8);  // size of lengths
  f.u8(0);
  f.u16(kLeafK);
  f.u16(kNodeK);
  f.u32(0);  // file consistency flags
  f.u64(0);  // base address
  f.u64(kUndef);  // free-space info
  f.u64(eof);
  f.u64(kUndef);  // driver information block
  // root group symbol table entry: cache type 1 holds the B-tree and heap addresses
  f.u64(0);
  f.u64(a_root);
  f.u32(1);
  f.u32(0);
  f.u64(a_btree);
  f.u64(a_heap);
  // root group object header: Symbol Table message
  {
    Buf st;
    st.u64(a_btree);
    st.u64(a_heap);
    Buf msgs;
    message(msgs, 0x0011, st);
    object_header(f, 1, msgs);
  }
  // local heap
  f.bytes("HEAP", 4);
  f.u8(0);
  f.zeros(3);
  f.u64(heap.s.size());
  f.u64(kFreeNull);
  f.u64(a_heapdata);
  f.bytes(heap.s.data(), heap.s.size());
  // B-tree leaf (node type 0 = group): key i = name offset below child i's
  // names ("" first), key i+1 = the last name of child i
  {
    const size_t start = f.s.size();
    f.bytes("TREE", 4);
    f.u8(0);
    f.u8(0);
    f.u16((uint16_t)nsnod);
    f.u64(kUndef);
    f.u64(kUndef);
    f.u64(0);
    for (size_t c = 0; c < nsnod; ++c) {
      const size_t last = std::min(n, (c + 1) * 2 * kLeafK);
      f.u64(a_snod + c * kSnod);
      f.u64(n ? name_off[last - 1] : 0);
    }
    f.pad_to(start + kBtreeNode);
  }
  // symbol-table nodes
  for (size_t c = 0; c < nsnod; ++c) {
    const size_t start = f.s.size();
    const size_t b0 = c * 2 * kLeafK, b1 = std::min(n, b0 + 2 * kLeafK);
    f.bytes("SNOD", 4);
    f.u8(1);
    f.u8(0);
    f.u16((uint16_t)(b1 - b0));
    for (size_t i = b0; i < b1; ++i) {
      f.u64(name_off[i]);
      f.u64(a_hdr[i]);
      f.u32(0);  // nothing cached
      f.u32(0);
      f.zeros(16);
    }
    f.pad_to(start + kSnod);
  }
  // dataset object headers, with the data addresses patched into the layout
  for (size_t i = 0; i < n; ++i) {
    std::string& h = headers[i].s;
    // the layout message is the header's last: its 18 data bytes (version,
    // class, address, size) padded to 24 end the header
    const size_t lay_data = h.size() - 24;
    uint64_t a = a_data[i];
    for (int k = 0; k < 8; ++k) h[lay_data + 2 + k] = (char)(a >> (8 * k));
    f.bytes(h.data(), h.size());
  }
  for (size_t i = 0; i < n; ++i) {
    f.pad_to(a_data[i]);
    f.bytes(ents[i]->data.data(), ents[i]->data.size());
  }
  f.pad_to(eof);
  return f.s;
}

bool H5Writer::write(const std::string& path) const {
  const std::string b = bytes();
  if (b.empty()) return false;
  FILE* fp = std::fopen(path.c_str(), "wb");
  if (!fp) return false;
  const bool ok = std::fwrite(b.data(), 1, b.size(), fp) == b.size();
  return std::fclose(fp) == 0 && ok;
}

}  // namespace cupf_host
