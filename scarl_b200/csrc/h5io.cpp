// h5io.cpp -- classic-format HDF5 writer and reader (see h5io.h).  Layout of
// a written file, all little-endian, 8-byte offsets and lengths:
//
//   superblock v0 (96 B) | root object header | local heap (header + data)
//   | v1 B-tree group node (K = 16: 544 B) | symbol table nodes (leaf K = 4:
//   328 B each) | dataset object headers | raw data of each dataset
//
// Structures and field orders follow the HDF5 File Format Specification
// (superblock version 0, object header version 1, messages: dataspace v1,
// datatype v1, fill value v1, layout v3 contiguous, attribute v1, symbol
// table).  The heap keeps a trailing free block whose "next" field is 1, the
// value the HDF5 library reads as the end of the free list.
#include "h5io.h"

#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <map>

namespace scarl {
namespace h5 {

namespace {

constexpr uint64_t kUndef = ~(uint64_t)0;
constexpr int kLeafK = 4;       // symbol table node: up to 2K entries
constexpr int kInternalK = 16;  // group B-tree node: up to 2K children
constexpr size_t kTreeBytes = 24 + (2 * kInternalK) * 8 + (2 * kInternalK + 1) * 8;  // 544
constexpr size_t kSnodBytes = 8 + (2 * kLeafK) * 40;                                  // 328

struct Buf {
  std::vector<uint8_t> b;
  void u8(uint32_t v) { b.push_back((uint8_t)v); }
  void u16(uint32_t v) { for (int i = 0; i < 2; ++i) b.push_back((uint8_t)(v >> (8 * i))); }
  void u32(uint32_t v) { for (int i = 0; i < 4; ++i) b.push_back((uint8_t)(v >> (8 * i))); }
  void u64(uint64_t v) { for (int i = 0; i < 8; ++i) b.push_back((uint8_t)(v >> (8 * i))); }
  void bytes(const void* p, size_t n) { b.insert(b.end(), (const uint8_t*)p, (const uint8_t*)p + n); }
  void pad8() { while (b.size() % 8) b.push_back(0); }
  void zeros(size_t n) { b.insert(b.end(), n, 0); }
  size_t size() const { return b.size(); }
};

size_t up8(size_t n) { return (n + 7) / 8 * 8; }

std::vector<uint8_t> enc_dtype(Kind k, int strsize) {
  Buf o;
  switch (k) {
    case F64:
      o.u8(0x11); o.u8(0x20); o.u8(63); o.u8(0); o.u32(8);
      o.u16(0); o.u16(64); o.u8(52); o.u8(11); o.u8(0); o.u8(52); o.u32(1023);
      break;
    case F32:
      o.u8(0x11); o.u8(0x20); o.u8(31); o.u8(0); o.u32(4);
      o.u16(0); o.u16(32); o.u8(23); o.u8(8); o.u8(0); o.u8(23); o.u32(127);
      break;
    case I32:
      o.u8(0x10); o.u8(0x08); o.u8(0); o.u8(0); o.u32(4);
      o.u16(0); o.u16(32);
      break;
    case STR:  // space padded, ASCII (Fortran strings)
      o.u8(0x13); o.u8(0x02); o.u8(0); o.u8(0); o.u32((uint32_t)strsize);
      break;
  }
  return o.b;
}

std::vector<uint8_t> enc_space(const std::vector<uint64_t>& dims) {
  Buf o;
  o.u8(1); o.u8((uint32_t)dims.size()); o.u8(0); o.u8(0); o.u32(0);
  for (uint64_t d : dims) o.u64(d);
  return o.b;
}

void message(Buf& oh, uint32_t type, const std::vector<uint8_t>& data, uint32_t flags) {
  oh.u16(type);
  oh.u16((uint32_t)up8(data.size()));
  oh.u8(flags);
  oh.u8(0); oh.u8(0); oh.u8(0);
  oh.bytes(data.data(), data.size());
  oh.pad8();
}

std::vector<uint8_t> enc_attr(const Attr& a) {
  const std::vector<uint8_t> dt = enc_dtype(a.kind, a.strsize);
  const std::vector<uint8_t> ds = enc_space(a.dims);
  Buf o;
  o.u8(1); o.u8(0);
  o.u16((uint32_t)a.name.size() + 1);
  o.u16((uint32_t)dt.size());
  o.u16((uint32_t)ds.size());
  o.bytes(a.name.c_str(), a.name.size() + 1);
  o.pad8();
  o.bytes(dt.data(), dt.size());
  o.pad8();
  o.bytes(ds.data(), ds.size());
  o.pad8();
  o.bytes(a.data.data(), a.data.size());
  return o.b;
}

// Object header v1: prefix (16 B) + messages; total size of messages >= 32
// (a NIL message fills up, as the library does).
std::vector<uint8_t> object_header(const std::vector<std::pair<uint32_t, std::vector<uint8_t>>>& msgs,
                                   const std::vector<uint32_t>& flags) {
  Buf body;
  int n = 0;
  for (size_t i = 0; i < msgs.size(); ++i, ++n) message(body, msgs[i].first, msgs[i].second, flags[i]);
  if (body.size() < 32) {
    const size_t fill = 32 - body.size() - 8;
    message(body, 0, std::vector<uint8_t>(fill, 0), 0);
    ++n;
  }
  Buf o;
  o.u8(1); o.u8(0); o.u16((uint32_t)n); o.u32(1); o.u32((uint32_t)body.size()); o.u32(0);
  o.bytes(body.b.data(), body.size());
  return o.b;
}

std::vector<uint8_t> dataset_header(const Dataset& d, uint64_t addr) {
  std::vector<std::pair<uint32_t, std::vector<uint8_t>>> m;
  std::vector<uint32_t> fl;
  // fill value v1: allocation late, write if set, defined with size 0
  m.push_back({0x5, {1, 2, 2, 1, 0, 0, 0, 0}});
  fl.push_back(1);
  m.push_back({0x3, enc_dtype(d.kind, d.strsize)});
  fl.push_back(1);
  m.push_back({0x1, enc_space(d.dims)});
  fl.push_back(0);
  Buf lay;
  lay.u8(3); lay.u8(1); lay.u64(addr); lay.u64(d.nbytes);
  m.push_back({0x8, lay.b});
  fl.push_back(1);
  for (const Attr& a : d.attrs) {
    m.push_back({0xC, enc_attr(a)});
    fl.push_back(0);
  }
  return object_header(m, fl);
}

}  // namespace

int elem_size(Kind k, int strsize) {
  return k == F64 ? 8 : (k == STR ? strsize : 4);
}

Attr attr_f64(const std::string& n, const double* v, int count, bool scalar) {
  Attr a;
  a.name = n;
  a.kind = F64;
  if (!scalar) a.dims = {(uint64_t)count};
  a.data.resize((size_t)count * 8);
  memcpy(a.data.data(), v, (size_t)count * 8);
  return a;
}

Attr attr_i32(const std::string& n, const int* v, int count, bool scalar) {
  Attr a;
  a.name = n;
  a.kind = I32;
  if (!scalar) a.dims = {(uint64_t)count};
  a.data.resize((size_t)count * 4);
  memcpy(a.data.data(), v, (size_t)count * 4);
  return a;
}

Attr attr_str(const std::string& n, const std::string& v) {
  Attr a;
  a.name = n;
  a.kind = STR;
  a.strsize = (int)std::max<size_t>(1, v.size());
  a.data.assign(v.begin(), v.end());
  if (a.data.empty()) a.data.push_back(' ');
  return a;
}

int write_file(const std::string& path, const std::vector<Attr>& root,
               const std::vector<Dataset>& dsets_in, std::string* err) {
  std::vector<const Dataset*> ds;
  for (const Dataset& d : dsets_in) ds.push_back(&d);
  std::sort(ds.begin(), ds.end(), [](const Dataset* a, const Dataset* b) {
    return strcmp(a->name.c_str(), b->name.c_str()) < 0;
  });
  for (size_t i = 1; i < ds.size(); ++i)
    if (ds[i]->name == ds[i - 1]->name) {
      *err = "duplicate dataset name " + ds[i]->name;
      return 1;
    }
  const size_t nsnod = (ds.size() + 2 * kLeafK - 1) / (2 * kLeafK);
  if (nsnod > 2 * kInternalK) {
    *err = "too many datasets for one group node";
    return 1;
  }
  // local heap data: "" at 0, then the names, then one free block
  Buf heap;
  heap.zeros(8);
  std::vector<uint64_t> name_off;
  for (const Dataset* d : ds) {
    name_off.push_back(heap.size());
    heap.bytes(d->name.c_str(), d->name.size() + 1);
    heap.pad8();
  }
  const uint64_t free_off = heap.size();
  const uint64_t heap_size = heap.size() + 16 + 8 * 8;
  heap.u64(1);  // next free block: none
  heap.u64(heap_size - free_off);
  heap.zeros(heap_size - heap.size());
  // addresses
  const uint64_t a_root = 96;
  std::vector<std::pair<uint32_t, std::vector<uint8_t>>> rm;
  std::vector<uint32_t> rf;
  rm.push_back({0x11, std::vector<uint8_t>(16, 0)});
  rf.push_back(1);
  for (const Attr& a : root) {
    rm.push_back({0xC, enc_attr(a)});
    rf.push_back(0);
  }
  const size_t root_size = object_header(rm, rf).size();
  const uint64_t a_heap = a_root + up8(root_size);
  const uint64_t a_heapdata = a_heap + 32;
  const uint64_t a_tree = a_heapdata + heap.size();
  const uint64_t a_snod = a_tree + kTreeBytes;
  uint64_t a = a_snod + nsnod * kSnodBytes;
  std::vector<uint64_t> a_oh(ds.size()), oh_size(ds.size());
  for (size_t i = 0; i < ds.size(); ++i) {
    a_oh[i] = a;
    oh_size[i] = dataset_header(*ds[i], 0).size();
    a += up8(oh_size[i]);
  }
  std::vector<uint64_t> a_data(ds.size());
  for (size_t i = 0; i < ds.size(); ++i) {
    a_data[i] = a;
    a += up8(ds[i]->nbytes);
  }
  const uint64_t eof = a;
  // serialise the metadata
  Buf f;
  const uint8_t sig[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};
  f.bytes(sig, 8);
  f.u8(0); f.u8(0); f.u8(0); f.u8(0); f.u8(0); f.u8(8); f.u8(8); f.u8(0);
  f.u16(kLeafK); f.u16(kInternalK); f.u32(0);
  f.u64(0); f.u64(kUndef); f.u64(eof); f.u64(kUndef);
  f.u64(0); f.u64(a_root); f.u32(1); f.u32(0); f.u64(a_tree); f.u64(a_heap);
  {
    Buf st;
    st.u64(a_tree);
    st.u64(a_heap);
    rm[0].second = st.b;
    std::vector<uint8_t> oh = object_header(rm, rf);
    f.bytes(oh.data(), oh.size());
    f.pad8();
  }
  f.bytes("HEAP", 4); f.u8(0); f.u8(0); f.u8(0); f.u8(0);
  f.u64(heap.size()); f.u64(free_off); f.u64(a_heapdata);
  f.bytes(heap.b.data(), heap.size());
  {
    const size_t t0 = f.size();
    f.bytes("TREE", 4); f.u8(0); f.u8(0); f.u16((uint32_t)nsnod); f.u64(kUndef); f.u64(kUndef);
    f.u64(0);
    for (size_t c = 0; c < nsnod; ++c) {
      f.u64(a_snod + c * kSnodBytes);
      const size_t last = std::min(ds.size(), (c + 1) * 2 * kLeafK) - 1;
      f.u64(name_off[last]);
    }
    f.zeros(kTreeBytes - (f.size() - t0));
  }
  for (size_t c = 0; c < nsnod; ++c) {
    const size_t s0 = f.size();
    const size_t lo = c * 2 * kLeafK, hi = std::min(ds.size(), lo + 2 * kLeafK);
    f.bytes("SNOD", 4); f.u8(1); f.u8(0); f.u16((uint32_t)(hi - lo));
    for (size_t i = lo; i < hi; ++i) {
      f.u64(name_off[i]); f.u64(a_oh[i]); f.u32(0); f.u32(0); f.zeros(16);
    }
    f.zeros(kSnodBytes - (f.size() - s0));
  }
  for (size_t i = 0; i < ds.size(); ++i) {
    std::vector<uint8_t> oh = dataset_header(*ds[i], a_data[i]);
    f.bytes(oh.data(), oh.size());
    f.pad8();
  }
  FILE* fp = fopen(path.c_str(), "wb");
  if (!fp) {
    *err = "cannot create " + path;
    return 6;
  }
  bool ok = fwrite(f.b.data(), 1, f.size(), fp) == f.size();
  for (size_t i = 0; ok && i < ds.size(); ++i) {
    ok = ds[i]->write ? ds[i]->write(fp) : ds[i]->nbytes == 0;
    const size_t pad = up8(ds[i]->nbytes) - ds[i]->nbytes;
    static const uint8_t z[8] = {0};
    if (ok && pad) ok = fwrite(z, 1, pad, fp) == pad;
  }
  if (ok) ok = (uint64_t)ftell(fp) == eof || ftello(fp) == (off_t)eof;
  if (fclose(fp) != 0) ok = false;
  if (!ok) {
    *err = "write error on " + path;
    return 6;
  }
  return 0;
}

// ===========================================================================
// Reader
// ===========================================================================
namespace {

struct In {
  FILE* fp = nullptr;
  uint64_t base = 0;
  std::string* err;
  bool at(uint64_t rel, void* dst, size_t n) {
    if (fseeko(fp, (off_t)(base + rel), SEEK_SET) != 0) return false;
    return fread(dst, 1, n, fp) == n;
  }
  bool abs(uint64_t a, void* dst, size_t n) {
    if (fseeko(fp, (off_t)a, SEEK_SET) != 0) return false;
    return fread(dst, 1, n, fp) == n;
  }
};

uint64_t le(const uint8_t* p, int n) {
  uint64_t v = 0;
  for (int i = n - 1; i >= 0; --i) v = (v << 8) | p[i];
  return v;
}

bool parse_dtype(const uint8_t* p, size_t n, Kind* k, int* size) {
  if (n < 8) return false;
  const int cls = p[0] & 0x0f;
  const int sz = (int)le(p + 4, 4);
  if (cls == 1) {
    if (p[1] & 1) return false;  // big-endian
    if (sz == 8) *k = F64;
    else if (sz == 4) *k = F32;
    else return false;
  } else if (cls == 0) {
    if (p[1] & 1) return false;
    if (sz != 4 && sz != 8 && sz != 2 && sz != 1) return false;
    *k = I32;
  } else if (cls == 3) {
    *k = STR;
  } else {
    return false;
  }
  *size = sz;
  return true;
}

bool parse_space(const uint8_t* p, size_t n, std::vector<uint64_t>* dims) {
  if (n < 4) return false;
  const int ver = p[0], rank = p[1];
  dims->clear();
  size_t off;
  if (ver == 1) off = 8;
  else if (ver == 2) off = 4;
  else return false;
  if (ver == 2 && p[3] == 2) return true;  // null dataspace
  for (int i = 0; i < rank; ++i) {
    if (off + 8 > n) return false;
    dims->push_back(le(p + off, 8));
    off += 8;
  }
  return true;
}

bool parse_attr(const uint8_t* p, size_t n, Attr* a) {
  if (n < 8) return false;
  const int ver = p[0];
  const size_t nl = le(p + 2, 2), dl = le(p + 4, 2), sl = le(p + 6, 2);
  size_t off = ver == 3 ? 9 : 8;
  auto adv = [&](size_t len) { return ver == 1 ? up8(len) : len; };
  if (off + adv(nl) + adv(dl) + adv(sl) > n) return false;
  a->name.assign((const char*)p + off, nl ? nl - 1 : 0);
  off += adv(nl);
  int sz = 0;
  if (!parse_dtype(p + off, dl, &a->kind, &sz)) return false;
  off += adv(dl);
  if (!parse_space(p + off, sl, &a->dims)) return false;
  off += adv(sl);
  uint64_t cnt = 1;
  for (uint64_t d : a->dims) cnt *= d;
  if (a->kind == STR) a->strsize = sz;
  const uint64_t bytes = cnt * (uint64_t)sz;
  if (off + bytes > n) return false;
  if (a->kind == I32 && sz != 4) {  // widen/narrow other integer sizes to int32
    std::vector<uint8_t> d(cnt * 4);
    for (uint64_t i = 0; i < cnt; ++i) {
      int64_t v = (int64_t)le(p + off + i * sz, sz);
      if (sz < 8 && (v >> (8 * sz - 1)) & 1) v -= (int64_t)1 << (8 * sz);
      const int32_t w = (int32_t)v;
      memcpy(d.data() + i * 4, &w, 4);
    }
    a->data = d;
  } else {
    a->data.assign(p + off, p + off + bytes);
  }
  return true;
}

// Messages of a version 1 object header, continuation blocks included.
bool header_messages(In& in, uint64_t addr, std::vector<std::pair<int, std::vector<uint8_t>>>* out) {
  uint8_t pre[16];
  if (!in.at(addr, pre, 16)) return false;
  if (pre[0] != 1) {
    *in.err = "object header version " + std::to_string(pre[0]) + " is not supported";
    return false;
  }
  const int nmsg = (int)le(pre + 2, 2);
  std::vector<std::pair<uint64_t, uint64_t>> chunks = {{addr + 16, le(pre + 8, 4)}};
  int seen = 0;
  for (size_t c = 0; c < chunks.size() && seen < nmsg; ++c) {
    std::vector<uint8_t> buf(chunks[c].second);
    if (!in.at(chunks[c].first, buf.data(), buf.size())) return false;
    size_t off = 0;
    while (off + 8 <= buf.size() && seen < nmsg) {
      const int type = (int)le(&buf[off], 2);
      const size_t sz = le(&buf[off + 2], 2);
      if (off + 8 + sz > buf.size()) return false;
      std::vector<uint8_t> data(buf.begin() + off + 8, buf.begin() + off + 8 + sz);
      if (type == 0x10 && sz >= 16) chunks.push_back({le(&data[0], 8), le(&data[8], 8)});
      else out->push_back({type, data});
      off += 8 + sz;
      ++seen;
    }
  }
  return true;
}

bool read_object(In& in, uint64_t addr, RObject* o) {
  std::vector<std::pair<int, std::vector<uint8_t>>> msgs;
  if (!header_messages(in, addr, &msgs)) return false;
  bool has_type = false, has_space = false, has_layout = false;
  for (auto& m : msgs) {
    const std::vector<uint8_t>& d = m.second;
    if (m.first == 0x1) {
      has_space = parse_space(d.data(), d.size(), &o->dims);
    } else if (m.first == 0x3) {
      has_type = parse_dtype(d.data(), d.size(), &o->kind, &o->elsize);
    } else if (m.first == 0x8 && !d.empty()) {
      const int ver = d[0];
      if (ver == 3 && d.size() >= 18 && d[1] == 1) {
        o->data_addr = in.base + le(&d[2], 8);
        o->nbytes = le(&d[10], 8);
        has_layout = true;
      } else if ((ver == 1 || ver == 2) && d.size() >= 16 && d[2] == 1) {
        const int nd = d[1];
        o->data_addr = in.base + le(&d[8], 8);
        uint64_t n = 1;
        for (int i = 0; i < nd && 16 + 4 * (size_t)i + 4 <= d.size(); ++i) n *= le(&d[16 + 4 * i], 4);
        o->nbytes = n;
        has_layout = true;
      } else {
        *in.err = "only contiguous dataset layouts are supported";
        return false;
      }
    } else if (m.first == 0xC) {
      Attr a;
      if (parse_attr(d.data(), d.size(), &a)) o->attrs.push_back(a);
    }
  }
  o->is_dataset = has_type && has_space && has_layout;
  return true;
}

bool walk_tree(In& in, uint64_t addr, uint64_t heap_data, uint64_t heap_size,
               std::vector<std::pair<std::string, uint64_t>>* entries, int depth) {
  if (depth > 16) return false;
  uint8_t h[24];
  if (!in.at(addr, h, 24) || memcmp(h, "TREE", 4) != 0 || h[4] != 0) return false;
  const int level = h[5];
  const int used = (int)le(h + 6, 2);
  std::vector<uint8_t> body((size_t)used * 16 + 8);
  if (!in.at(addr + 24, body.data(), body.size())) return false;
  for (int i = 0; i < used; ++i) {
    const uint64_t child = le(&body[8 + 16 * (size_t)i], 8);
    if (level > 0) {
      if (!walk_tree(in, child, heap_data, heap_size, entries, depth + 1)) return false;
      continue;
    }
    uint8_t sh[8];
    if (!in.at(child, sh, 8) || memcmp(sh, "SNOD", 4) != 0) return false;
    const int n = (int)le(sh + 6, 2);
    std::vector<uint8_t> es((size_t)n * 40);
    if (!in.at(child + 8, es.data(), es.size())) return false;
    for (int e = 0; e < n; ++e) {
      const uint64_t noff = le(&es[40 * (size_t)e], 8);
      const uint64_t oh = le(&es[40 * (size_t)e + 8], 8);
      if (noff >= heap_size) return false;
      std::string name;
      char c;
      uint64_t p = noff;
      while (p < heap_size && in.at(heap_data + p, &c, 1) && c) {
        name.push_back(c);
        ++p;
      }
      entries->push_back({name, oh});
    }
  }
  return true;
}

}  // namespace

int read_file(const std::string& path, RObject* root, std::vector<RObject>* dsets,
              std::string* err) {
  In in;
  in.err = err;
  in.fp = fopen(path.c_str(), "rb");
  if (!in.fp) {
    *err = "cannot open " + path;
    return 6;
  }
  struct Closer {
    FILE* f;
    ~Closer() { fclose(f); }
  } closer{in.fp};
  const uint8_t sig[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};
  uint64_t sb = kUndef;
  for (uint64_t off = 0; off <= (1ull << 20); off = off ? off * 2 : 512) {
    uint8_t s[8];
    if (!in.abs(off, s, 8)) break;
    if (memcmp(s, sig, 8) == 0) {
      sb = off;
      break;
    }
  }
  if (sb == kUndef) {
    *err = "no HDF5 superblock in " + path;
    return 1;
  }
  uint8_t s[128];
  if (!in.abs(sb, s, 8 + 16)) return (*err = "truncated superblock", 1);
  const int ver = s[8];
  if (ver > 1) return (*err = "superblock version " + std::to_string(ver) + " is not supported", 5);
  if (s[13] != 8 || s[14] != 8) return (*err = "only 8-byte offsets and lengths are supported", 5);
  const size_t head = ver == 0 ? 24 : 28;
  if (!in.abs(sb, s, head + 32 + 40)) return (*err = "truncated superblock", 1);
  in.base = le(s + head, 8);
  const uint8_t* ent = s + head + 32;
  const uint64_t root_oh = le(ent + 8, 8);
  std::vector<std::pair<int, std::vector<uint8_t>>> msgs;
  if (!header_messages(in, root_oh, &msgs)) return 1;
  uint64_t tree = kUndef, heap = kUndef;
  root->name = "";
  for (auto& m : msgs) {
    if (m.first == 0x11 && m.second.size() >= 16) {
      tree = le(&m.second[0], 8);
      heap = le(&m.second[8], 8);
    } else if (m.first == 0xC) {
      Attr a;
      if (parse_attr(m.second.data(), m.second.size(), &a)) root->attrs.push_back(a);
    }
  }
  if (tree == kUndef) return (*err = "root group has no symbol table (new-style groups are not supported)", 5);
  uint8_t hh[32];
  if (!in.at(heap, hh, 32) || memcmp(hh, "HEAP", 4) != 0) return (*err = "bad local heap", 1);
  const uint64_t hsize = le(hh + 8, 8), hdata = le(hh + 24, 8);
  std::vector<std::pair<std::string, uint64_t>> entries;
  if (!walk_tree(in, tree, hdata, hsize, &entries, 0)) {
    if (err->empty()) *err = "bad group B-tree";
    return 1;
  }
  for (auto& e : entries) {
    RObject o;
    o.name = e.first;
    if (!read_object(in, e.second, &o)) {
      if (err->empty()) *err = "bad object header for " + e.first;
      return 1;
    }
    dsets->push_back(o);
  }
  return 0;
}

int read_values(const std::string& path, const RObject& d, double* out64, float* out32,
                std::string* err) {
  if (!d.is_dataset || d.kind == STR) return (*err = d.name + " is not a numeric dataset", 1);
  uint64_t cnt = 1;
  for (uint64_t v : d.dims) cnt *= v;
  if (cnt * (uint64_t)d.elsize != d.nbytes) return (*err = "dataset size mismatch", 1);
  FILE* fp = fopen(path.c_str(), "rb");
  if (!fp) return (*err = "cannot open " + path, 6);
  const uint64_t chunk = 1 << 20;
  std::vector<uint8_t> buf;
  bool ok = fseeko(fp, (off_t)d.data_addr, SEEK_SET) == 0;
  for (uint64_t i = 0; ok && i < cnt; i += chunk) {
    const uint64_t n = std::min(chunk, cnt - i);
    buf.resize(n * d.elsize);
    ok = fread(buf.data(), 1, buf.size(), fp) == buf.size();
    for (uint64_t j = 0; ok && j < n; ++j) {
      double v;
      const uint8_t* p = &buf[j * d.elsize];
      if (d.kind == F64) {
        memcpy(&v, p, 8);
      } else if (d.kind == F32) {
        float f;
        memcpy(&f, p, 4);
        v = f;
      } else {
        int64_t x = (int64_t)le(p, d.elsize);
        if (d.elsize < 8 && (x >> (8 * d.elsize - 1)) & 1) x -= (int64_t)1 << (8 * d.elsize);
        v = (double)x;
      }
      if (out64) out64[i + j] = v;
      if (out32) out32[i + j] = (float)v;
    }
  }
  fclose(fp);
  if (!ok) return (*err = "read error on " + path, 6);
  return 0;
}


int append_root_attrs(const std::string& path, const std::vector<Attr>& attrs, std::string* err) {
  FILE* fp = fopen(path.c_str(), "r+b");
  if (!fp) return (*err = "cannot open " + path + " for update", 6);
  struct Closer {
    FILE* f;
    ~Closer() { if (f) fclose(f); }
  } closer{fp};
  In in;
  in.fp = fp;
  in.err = err;
  const uint8_t sig[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};
  uint64_t sb = kUndef;
  for (uint64_t off = 0; off <= (1ull << 20); off = off ? off * 2 : 512) {
    uint8_t s8[8];
    if (!in.abs(off, s8, 8)) break;
    if (memcmp(s8, sig, 8) == 0) {
      sb = off;
      break;
    }
  }
  if (sb == kUndef) return (*err = "no HDF5 superblock in " + path, 1);
  uint8_t s[128];
  if (!in.abs(sb, s, 24)) return (*err = "truncated superblock", 1);
  const int ver = s[8];
  if (ver > 1 || s[13] != 8 || s[14] != 8) return (*err = "unsupported superblock", 5);
  const size_t head = ver == 0 ? 24 : 28;
  if (!in.abs(sb, s, head + 72)) return (*err = "truncated superblock", 1);
  in.base = le(s + head, 8);
  const uint64_t root_oh = le(s + head + 40, 8);
  // the root header's messages with their flags
  uint8_t pre[16];
  if (!in.at(root_oh, pre, 16) || pre[0] != 1) return (*err = "unsupported root object header", 5);
  const int nmsg = (int)le(pre + 2, 2);
  std::vector<std::pair<uint64_t, uint64_t>> chunks = {{root_oh + 16, le(pre + 8, 4)}};
  std::vector<std::pair<uint32_t, std::vector<uint8_t>>> msgs;
  std::vector<uint32_t> flags;
  int seen = 0;
  for (size_t c = 0; c < chunks.size() && seen < nmsg; ++c) {
    std::vector<uint8_t> buf(chunks[c].second);
    if (!in.at(chunks[c].first, buf.data(), buf.size())) return (*err = "truncated object header", 1);
    size_t off = 0;
    while (off + 8 <= buf.size() && seen < nmsg) {
      const uint32_t type = (uint32_t)le(&buf[off], 2);
      const size_t sz = le(&buf[off + 2], 2);
      if (off + 8 + sz > buf.size()) return (*err = "bad object header", 1);
      std::vector<uint8_t> data(buf.begin() + off + 8, buf.begin() + off + 8 + sz);
      ++seen;
      off += 8 + sz;
      if (type == 0x10) {
        chunks.push_back({le(&data[0], 8), le(&data[8], 8)});
        continue;
      }
      if (type == 0x0) continue;
      if (type == 0xC) {
        Attr old;
        bool replaced = false;
        if (parse_attr(data.data(), data.size(), &old))
          for (const Attr& a : attrs) replaced = replaced || a.name == old.name;
        if (replaced) continue;
      }
      msgs.push_back({type, data});
      flags.push_back(buf[off - 8 - sz + 4]);
    }
  }
  for (const Attr& a : attrs) {
    msgs.push_back({0xC, enc_attr(a)});
    flags.push_back(0);
  }
  const std::vector<uint8_t> oh = object_header(msgs, flags);
  if (fseeko(fp, 0, SEEK_END) != 0) return (*err = "seek error", 6);
  uint64_t end = (uint64_t)ftello(fp);
  static const uint8_t z[8] = {0};
  const size_t pad = (size_t)(up8(end) - end);
  if (pad && fwrite(z, 1, pad, fp) != pad) return (*err = "write error", 6);
  end += pad;
  if (fwrite(oh.data(), 1, oh.size(), fp) != oh.size()) return (*err = "write error", 6);
  const uint64_t new_oh = end - in.base;
  const uint64_t eof = end + up8(oh.size()) - in.base;
  const size_t tail = up8(oh.size()) - oh.size();
  if (tail && fwrite(z, 1, tail, fp) != tail) return (*err = "write error", 6);
  uint8_t w[8];
  for (int i = 0; i < 8; ++i) w[i] = (uint8_t)(new_oh >> (8 * i));
  if (fseeko(fp, (off_t)(sb + head + 40), SEEK_SET) != 0 || fwrite(w, 1, 8, fp) != 8)
    return (*err = "write error", 6);
  for (int i = 0; i < 8; ++i) w[i] = (uint8_t)(eof >> (8 * i));
  if (fseeko(fp, (off_t)(sb + head + 16), SEEK_SET) != 0 || fwrite(w, 1, 8, fp) != 8)
    return (*err = "write error", 6);
  if (fclose(fp) != 0) {
    closer.f = nullptr;
    return (*err = "write error", 6);
  }
  closer.f = nullptr;
  return 0;
}


int overwrite_dataset(const std::string& path, const std::string& name, const void* data,
                      uint64_t nbytes, std::string* err) {
  RObject root;
  std::vector<RObject> ds;
  const int rc = read_file(path, &root, &ds, err);
  if (rc) return rc;
  for (const RObject& d : ds) {
    if (d.name != name) continue;
    if (!d.is_dataset || d.nbytes != nbytes) return (*err = "size mismatch for dataset " + name, 1);
    FILE* fp = fopen(path.c_str(), "r+b");
    if (!fp) return (*err = "cannot open " + path + " for update", 6);
    bool ok = fseeko(fp, (off_t)d.data_addr, SEEK_SET) == 0 && fwrite(data, 1, nbytes, fp) == nbytes;
    ok = (fclose(fp) == 0) && ok;
    return ok ? 0 : (*err = "write error on " + path, 6);
  }
  return (*err = "no dataset " + name, 1);
}

}  // namespace h5
}  // namespace scarl
