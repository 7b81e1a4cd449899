// hdf5_catalog.cpp — write_catalog_hdf5 (ext/HDF5Ext.jl:47-104) without
// libhdf5: the catalogue's columns as one-dimensional little-endian Float32
// datasets in the root group of an HDF5 file, written byte by byte in the
// file format's original layout (superblock version 0, a root group held
// by a version 1 B-tree, a local heap of names and one symbol table node,
// version 1 object headers, contiguous storage).  Any HDF5 reader opens it.
//
// Columns (the reference's): x, y, z, ra, dec, redshift, chi, M200m, RTHL,
// vx, vy, vz, and for 33-field records also vx2, vy2, vz2, overdensity,
// e_v, p_v, Rf, zform.  chi = |x| (Mpc/h, from the origin), redshift =
// chi_to_z on build_chi_to_z(cosmo; z_max) (Cosmology.jl:333-358),
// M200m = 4/3 pi 2.775e11 Om h^2 RTHL^3, (ra, dec) = _rect_to_radec(x, y, z).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "ppb_ctx.h"

namespace ppb {
namespace {

constexpr uint64_t kUndef = ~0ull;
constexpr int kLeafK = 16;       // symbol table node: up to 2 kLeafK entries (one node holds every column)
constexpr int kInternalK = 16;   // group B-tree node: up to 2 kInternalK children

struct Buf {
  std::vector<uint8_t> b;
  size_t size() const { return b.size(); }
  void u8(uint8_t v) { b.push_back(v); }
  void u16(uint16_t v) { for (int i = 0; i < 2; i++) b.push_back((uint8_t)(v >> (8 * i))); }
  void u32(uint32_t v) { for (int i = 0; i < 4; i++) b.push_back((uint8_t)(v >> (8 * i))); }
  void u64(uint64_t v) { for (int i = 0; i < 8; i++) b.push_back((uint8_t)(v >> (8 * i))); }
  void bytes(const void* p, size_t n) { b.insert(b.end(), (const uint8_t*)p, (const uint8_t*)p + n); }
  void pad8() { while (b.size() % 8) b.push_back(0); }
  void zeros(size_t n) { b.insert(b.end(), n, 0); }
  void put64(size_t at, uint64_t v) { for (int i = 0; i < 8; i++) b[at + i] = (uint8_t)(v >> (8 * i)); }
};

// one object header message of a version 1 object header: type, size,
// flags, then the body padded to 8 bytes
void message(Buf& o, uint16_t type, uint8_t flags, const Buf& body) {
  Buf p = body;
  p.pad8();
  o.u16(type);
  o.u16((uint16_t)p.size());
  o.u8(flags);
  o.zeros(3);
  o.bytes(p.b.data(), p.size());
}

// version 1 object header: prefix (version, reserved, message count,
// reference count, size of the messages, alignment padding), messages
void object_header(Buf& out, const std::vector<Buf>& msgs) {
  size_t sz = 0;
  for (const Buf& m : msgs) sz += m.size();
  out.u8(1);
  out.u8(0);
  out.u16((uint16_t)msgs.size());
  out.u32(1);
  out.u32((uint32_t)sz);
  out.zeros(4);
  for (const Buf& m : msgs) out.bytes(m.b.data(), m.size());
}

struct Column {
  std::string name;
  std::vector<float> v;
};

void write_file(const std::string& path, std::vector<Column>& cols, int64_t n) {
  std::sort(cols.begin(), cols.end(), [](const Column& a, const Column& b) { return a.name < b.name; });
  const size_t ncol = cols.size();
  PPB_REQUIRE(ncol <= 2 * kLeafK, "too many datasets for one symbol table node");
  // local heap of names: "" at offset 0, then each name, 8-byte aligned,
  // then one free block (next free block "1": the end of the free list;
  // its size), as the format's own writer leaves the heap
  Buf heap;
  heap.zeros(8);
  std::vector<uint64_t> name_off(ncol);
  for (size_t c = 0; c < ncol; c++) {
    name_off[c] = heap.size();
    heap.bytes(cols[c].name.data(), cols[c].name.size());
    heap.u8(0);
    heap.pad8();
  }
  const uint64_t free_off = heap.size();
  heap.u64(1);
  heap.u64(16);
  // addresses (the root group's object header holds the symbol table
  // message and a null message: 16 + 24 + 16 bytes)
  const uint64_t a_root = 96, a_heap = a_root + 16 + 24 + 16, a_heapdata = a_heap + 32;
  const uint64_t a_btree = a_heapdata + heap.size();
  const uint64_t btree_size = 24 + (2 * kInternalK + 1) * 8 + 2 * kInternalK * 8;
  const uint64_t a_snod = a_btree + btree_size;
  const uint64_t snod_size = 8 + 2 * kLeafK * 40;
  uint64_t at = a_snod + (ncol ? snod_size : 0);
  // datasets: object header, then the data (8-byte aligned)
  std::vector<Buf> dsets(ncol);
  std::vector<uint64_t> a_obj(ncol);
  const uint64_t nbytes = (uint64_t)n * 4;
  for (size_t c = 0; c < ncol; c++) {
    Buf space, type, fill, layout;
    space.u8(1);            // dataspace version 1
    space.u8(1);            // rank
    space.u8(0);            // no maximum dimensions
    space.zeros(5);
    space.u64((uint64_t)n);
    type.u8(0x11);          // version 1, floating point
    type.u8(0x20);          // little endian, implied mantissa MSB
    type.u8(31);            // sign bit position
    type.u8(0);
    type.u32(4);            // size in bytes
    type.u16(0);            // bit offset
    type.u16(32);           // precision
    type.u8(23);            // exponent location
    type.u8(8);             // exponent size
    type.u8(0);             // mantissa location
    type.u8(23);            // mantissa size
    type.u32(127);          // exponent bias
    fill.u8(2);             // fill value message version 2
    fill.u8(1);             // space allocated early
    fill.u8(2);             // fill value never written
    fill.u8(0);             // no fill value defined
    const uint64_t hdr_size = 16 + (8 + 16) + (8 + 24) + (8 + 8) + (8 + 24);
    a_obj[c] = at;
    const uint64_t a_data = at + hdr_size;
    layout.u8(3);           // layout message version 3
    layout.u8(1);           // contiguous
    layout.u64(n > 0 ? a_data : kUndef);
    layout.u64(nbytes);
    std::vector<Buf> msgs(4);
    message(msgs[0], 0x0001, 0, space);
    message(msgs[1], 0x0003, 1, type);
    message(msgs[2], 0x0005, 1, fill);
    message(msgs[3], 0x0008, 0, layout);
    object_header(dsets[c], msgs);
    PPB_REQUIRE(dsets[c].size() == hdr_size, "object header size");
    dsets[c].bytes(cols[c].v.data(), nbytes);
    dsets[c].pad8();
    at += dsets[c].size();
  }
  const uint64_t eof = at;

  Buf f;
  // superblock version 0
  const uint8_t sig[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};
  f.bytes(sig, 8);
  f.u8(0); f.u8(0); f.u8(0); f.u8(0); f.u8(0);
  f.u8(8);                  // size of offsets
  f.u8(8);                  // size of lengths
  f.u8(0);
  f.u16(kLeafK);
  f.u16(kInternalK);
  f.u32(0);                 // consistency flags
  f.u64(0);                 // base address
  f.u64(kUndef);            // free-space info
  f.u64(eof);
  f.u64(kUndef);            // driver information block
  // root group symbol table entry: cache type 1 keeps the B-tree and heap
  f.u64(0);
  f.u64(a_root);
  f.u32(1);
  f.u32(0);
  f.u64(a_btree);
  f.u64(a_heap);
  PPB_REQUIRE(f.size() == a_root, "superblock size");
  // root group object header: the symbol table message
  {
    Buf st, nil;
    st.u64(a_btree);
    st.u64(a_heap);
    nil.zeros(8);
    std::vector<Buf> msgs(2);
    message(msgs[0], 0x0011, 0, st);
    message(msgs[1], 0x0000, 0, nil);
    object_header(f, msgs);
  }
  PPB_REQUIRE(f.size() == a_heap, "root object header size");
  // local heap
  f.bytes("HEAP", 4);
  f.u8(0);
  f.zeros(3);
  f.u64(heap.size());
  f.u64(free_off);          // head of the free list
  f.u64(a_heapdata);
  f.bytes(heap.b.data(), heap.size());
  // group B-tree node (leaf level: children are symbol table nodes)
  PPB_REQUIRE(f.size() == a_btree, "heap size");
  f.bytes("TREE", 4);
  f.u8(0);                  // group node
  f.u8(0);                  // level 0
  f.u16(ncol ? 1 : 0);      // entries used
  f.u64(kUndef);
  f.u64(kUndef);
  {
    const size_t keys_at = f.size();
    f.zeros((2 * kInternalK + 1) * 8 + 2 * kInternalK * 8);
    if (ncol) {
      f.put64(keys_at, 0);                       // key 0: the empty name
      f.put64(keys_at + 8, a_snod);              // child 0
      f.put64(keys_at + 16, name_off[ncol - 1]); // key 1: the last name of the child
    }
  }
  if (ncol) {
    PPB_REQUIRE(f.size() == a_snod, "B-tree node size");
    f.bytes("SNOD", 4);
    f.u8(1);
    f.u8(0);
    f.u16((uint16_t)ncol);
    for (size_t c = 0; c < 2 * kLeafK; c++) {
      if (c < ncol) {
        f.u64(name_off[c]);
        f.u64(a_obj[c]);
        f.u32(0);           // no cached data
        f.u32(0);
        f.zeros(16);
      } else {
        f.zeros(40);
      }
    }
  }
  for (size_t c = 0; c < ncol; c++) {
    PPB_REQUIRE(f.size() == a_obj[c], "dataset address");
    f.bytes(dsets[c].b.data(), dsets[c].size());
  }
  PPB_REQUIRE(f.size() == eof, "end of file");
  FILE* fp = std::fopen(path.c_str(), "wb");
  PPB_REQUIRE(fp != nullptr, "cannot open " + path + " for writing");
  const size_t w = std::fwrite(f.b.data(), 1, f.size(), fp);
  std::fclose(fp);
  PPB_REQUIRE(w == f.size(), "short write to " + path);
}

}  // namespace

// the reference's columns from 11- or 33-field records
void write_catalog_hdf5_host(const std::string& path, const float* rec, int64_t n, int nf, double Om, double OL,
                             double h, double z_max) {
  PPB_REQUIRE(nf == 11 || nf == 33, "nfields must be 11 or 33");
  PPB_REQUIRE(n >= 0, "negative record count");
  std::vector<Column> cols;
  if (n > 0) {
    const std::vector<double> chis = make_chi_table(Om, OL, h, z_max, 2000);
    const double rho_m = 2.775e11 * Om * h * h;
    auto field = [&](int f) {
      std::vector<float> v((size_t)n);
      for (int64_t i = 0; i < n; i++) v[i] = rec[i * nf + f];
      return v;
    };
    std::vector<float> ra((size_t)n), dec((size_t)n), red((size_t)n), chi((size_t)n), mass((size_t)n);
    for (int64_t i = 0; i < n; i++) {
      const double x = rec[i * nf], y = rec[i * nf + 1], z = rec[i * nf + 2];
      const double r = std::sqrt(x * x + y * y + z * z);
      chi[i] = (float)r;
      red[i] = (float)chi_to_z_host(chis, z_max, (double)chi[i]);
      const double R = rec[i * nf + 6];
      mass[i] = (float)(4.0 / 3.0 * 3.141592653589793 * rho_m * (R * R * R));
      // _rect_to_radec (ext/HDF5Ext.jl:18-26) on the Float32 positions
      if (r == 0.0) {
        ra[i] = 0.f;
        dec[i] = 0.f;
      } else {
        dec[i] = (float)std::asin(std::min(1.0, std::max(-1.0, z / r)));
        ra[i] = (float)std::atan2(y, x);
      }
    }
    cols.push_back({"x", field(0)});
    cols.push_back({"y", field(1)});
    cols.push_back({"z", field(2)});
    cols.push_back({"ra", std::move(ra)});
    cols.push_back({"dec", std::move(dec)});
    cols.push_back({"redshift", std::move(red)});
    cols.push_back({"chi", std::move(chi)});
    cols.push_back({"M200m", std::move(mass)});
    cols.push_back({"RTHL", field(6)});
    cols.push_back({"vx", field(3)});
    cols.push_back({"vy", field(4)});
    cols.push_back({"vz", field(5)});
    if (nf == 33) {
      cols.push_back({"vx2", field(7)});
      cols.push_back({"vy2", field(8)});
      cols.push_back({"vz2", field(9)});
      cols.push_back({"overdensity", field(10)});
      cols.push_back({"e_v", field(11)});
      cols.push_back({"p_v", field(12)});
      cols.push_back({"Rf", field(27)});
      cols.push_back({"zform", field(20)});
    }
  }
  write_file(path, cols, n);
}

}  // namespace ppb
