// On-disk formats of the flat index path (host code only):
//  * NumPy .npy float32 matrices (the reference's NpyReader / write_npy_f32_matrix,
//    include/vectorcache/datasets/npy.hpp:33-66): C-order (rows, cols) '<f4'.
//  * VCEX exact-top-k files (tools/query-bench.cpp:180-340): "VCEX", u32
//    version 1, u64 n_queries, k, index_n, seed, three u32-length-prefixed
//    strings (source label, split, query split), then n_queries * k u64 ids.
// All integers little-endian.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

#include "tq_abi.h"

namespace vcb {
namespace {

struct NpyHeader {
  size_t rows = 0, cols = 0, data_offset = 0;
};

NpyHeader parse_npy(std::ifstream& in, const char* path) {
  char magic[6];
  in.read(magic, 6);
  if (!in || std::memcmp(magic, "\x93NUMPY", 6) != 0) fail(TQ_ERR_INVALID_ARGUMENT, std::string(path) + ": not a .npy file");
  unsigned char ver[2];
  in.read(reinterpret_cast<char*>(ver), 2);
  uint32_t hlen = 0;
  size_t pre = 10;
  if (ver[0] == 1) {
    unsigned char b[2];
    in.read(reinterpret_cast<char*>(b), 2);
    hlen = b[0] | (b[1] << 8);
  } else if (ver[0] == 2 || ver[0] == 3) {
    unsigned char b[4];
    in.read(reinterpret_cast<char*>(b), 4);
    hlen = b[0] | (b[1] << 8) | (b[2] << 16) | (static_cast<uint32_t>(b[3]) << 24);
    pre = 12;
  } else {
    fail(TQ_ERR_INVALID_ARGUMENT, std::string(path) + ": unsupported .npy version");
  }
  std::string h(hlen, '\0');
  in.read(h.data(), hlen);
  if (!in) fail(TQ_ERR_INVALID_ARGUMENT, std::string(path) + ": truncated .npy header");
  auto field = [&](const char* key) -> std::string {
    const size_t k = h.find(key);
    if (k == std::string::npos) fail(TQ_ERR_INVALID_ARGUMENT, std::string(path) + ": .npy header lacks " + key);
    size_t v = h.find(':', k) + 1;
    while (v < h.size() && h[v] == ' ') ++v;
    return h.substr(v);
  };
  const std::string descr = field("'descr'");
  if (descr.rfind("'<f4'", 0) != 0) fail(TQ_ERR_INVALID_ARGUMENT, std::string(path) + ": .npy dtype must be float32 ('<f4')");
  if (field("'fortran_order'").rfind("False", 0) != 0) {
    fail(TQ_ERR_INVALID_ARGUMENT, std::string(path) + ": .npy must be C-ordered");
  }
  const std::string shape = field("'shape'");
  const size_t open = shape.find('('), close = shape.find(')');
  if (open == std::string::npos || close == std::string::npos) fail(TQ_ERR_INVALID_ARGUMENT, "bad .npy shape");
  std::vector<size_t> dims;
  std::string cur;
  for (size_t i = open + 1; i < close; ++i) {
    const char c = shape[i];
    if (c >= '0' && c <= '9') {
      cur.push_back(c);
    } else if (!cur.empty()) {
      dims.push_back(std::stoull(cur));
      cur.clear();
    }
  }
  if (!cur.empty()) dims.push_back(std::stoull(cur));
  if (dims.size() != 2) fail(TQ_ERR_INVALID_ARGUMENT, std::string(path) + ": .npy matrix must be 2-D (rows, cols)");
  NpyHeader out;
  out.rows = dims[0];
  out.cols = dims[1];
  out.data_offset = pre + hlen;
  return out;
}

void put_u32(std::ostream& o, uint32_t v) {
  unsigned char b[4] = {static_cast<unsigned char>(v), static_cast<unsigned char>(v >> 8),
                        static_cast<unsigned char>(v >> 16), static_cast<unsigned char>(v >> 24)};
  o.write(reinterpret_cast<const char*>(b), 4);
}

void put_u64(std::ostream& o, uint64_t v) {
  put_u32(o, static_cast<uint32_t>(v));
  put_u32(o, static_cast<uint32_t>(v >> 32));
}

uint32_t get_u32(std::istream& in) {
  unsigned char b[4] = {0, 0, 0, 0};
  in.read(reinterpret_cast<char*>(b), 4);
  if (!in) fail(TQ_ERR_INVALID_ARGUMENT, "truncated file");
  return b[0] | (b[1] << 8) | (b[2] << 16) | (static_cast<uint32_t>(b[3]) << 24);
}

uint64_t get_u64(std::istream& in) {
  const uint64_t lo = get_u32(in);
  return lo | (static_cast<uint64_t>(get_u32(in)) << 32);
}

std::string get_str(std::istream& in) {
  const uint32_t n = get_u32(in);
  std::string s(n, '\0');
  if (n) in.read(s.data(), n);
  if (!in) fail(TQ_ERR_INVALID_ARGUMENT, "truncated string");
  return s;
}

void put_str(std::ostream& o, const char* s) {
  const std::string v = s ? s : "";
  put_u32(o, static_cast<uint32_t>(v.size()));
  o.write(v.data(), static_cast<std::streamsize>(v.size()));
}

struct VcexHeader {
  uint64_t nq = 0, k = 0, index_n = 0, seed = 0;
  std::string label, split, query_split;
};

VcexHeader read_vcex_header(std::ifstream& in, const char* path) {
  char magic[4];
  in.read(magic, 4);
  if (!in || std::memcmp(magic, "VCEX", 4) != 0) fail(TQ_ERR_INVALID_ARGUMENT, std::string(path) + ": not a VCEX file");
  if (get_u32(in) != 1) fail(TQ_ERR_INVALID_ARGUMENT, std::string(path) + ": unsupported VCEX version");
  VcexHeader h;
  h.nq = get_u64(in);
  h.k = get_u64(in);
  h.index_n = get_u64(in);
  h.seed = get_u64(in);
  h.label = get_str(in);
  h.split = get_str(in);
  h.query_split = get_str(in);
  return h;
}

}  // namespace
}  // namespace vcb

extern "C" {

int tq_npy_f32_info(const char* path, size_t* rows, size_t* cols) {
  return vcb::guarded([&] {
    vcb::require(path && rows && cols, TQ_ERR_INVALID_ARGUMENT, "null argument");
    std::ifstream in(path, std::ios::binary);
    vcb::require(static_cast<bool>(in), TQ_ERR_INVALID_ARGUMENT, "cannot open .npy file");
    const vcb::NpyHeader h = vcb::parse_npy(in, path);
    *rows = h.rows;
    *cols = h.cols;
  });
}

int tq_npy_f32_read(const char* path, size_t row0, size_t nrows, float* out) {
  return vcb::guarded([&] {
    vcb::require(path && out, TQ_ERR_INVALID_ARGUMENT, "null argument");
    std::ifstream in(path, std::ios::binary);
    vcb::require(static_cast<bool>(in), TQ_ERR_INVALID_ARGUMENT, "cannot open .npy file");
    const vcb::NpyHeader h = vcb::parse_npy(in, path);
    vcb::require(row0 + nrows <= h.rows, TQ_ERR_INVALID_ARGUMENT, "row range outside the .npy matrix");
    in.seekg(static_cast<std::streamoff>(h.data_offset + row0 * h.cols * 4));
    in.read(reinterpret_cast<char*>(out), static_cast<std::streamsize>(nrows * h.cols * 4));
    vcb::require(static_cast<bool>(in), TQ_ERR_INVALID_ARGUMENT, "truncated .npy data");
  });
}

int tq_npy_f32_write(const char* path, size_t rows, size_t cols, const float* data) {
  return vcb::guarded([&] {
    vcb::require(path && (data || rows * cols == 0), TQ_ERR_INVALID_ARGUMENT, "null argument");
    std::string dict = "{'descr': '<f4', 'fortran_order': False, 'shape': (" + std::to_string(rows) + ", " +
                       std::to_string(cols) + "), }";
    // Pad so the data starts on a 64-byte boundary; the header ends with '\n'.
    const size_t total = ((10 + dict.size() + 1 + 63) / 64) * 64;
    dict.append(total - 10 - dict.size() - 1, ' ');
    dict.push_back('\n');
    std::ofstream o(path, std::ios::binary | std::ios::trunc);
    vcb::require(static_cast<bool>(o), TQ_ERR_INVALID_ARGUMENT, "cannot create .npy file");
    o.write("\x93NUMPY\x01\x00", 8);
    const uint16_t hl = static_cast<uint16_t>(dict.size());
    const unsigned char b[2] = {static_cast<unsigned char>(hl), static_cast<unsigned char>(hl >> 8)};
    o.write(reinterpret_cast<const char*>(b), 2);
    o.write(dict.data(), static_cast<std::streamsize>(dict.size()));
    o.write(reinterpret_cast<const char*>(data), static_cast<std::streamsize>(rows * cols * 4));
    vcb::require(static_cast<bool>(o), TQ_ERR_INVALID_ARGUMENT, "write failed");
  });
}

int tq_vcex_write(const char* path, const uint64_t* ids, size_t nq, size_t k, uint64_t index_n, uint64_t seed,
                  const char* source_label, const char* split, const char* query_split) {
  return vcb::guarded([&] {
    vcb::require(path && (ids || nq * k == 0), TQ_ERR_INVALID_ARGUMENT, "null argument");
    const std::string tmp = std::string(path) + ".tmp";
    {
      std::ofstream o(tmp, std::ios::binary | std::ios::trunc);
      vcb::require(static_cast<bool>(o), TQ_ERR_INVALID_ARGUMENT, "cannot create VCEX file");
      o.write("VCEX", 4);
      vcb::put_u32(o, 1);
      vcb::put_u64(o, nq);
      vcb::put_u64(o, k);
      vcb::put_u64(o, index_n);
      vcb::put_u64(o, seed);
      vcb::put_str(o, source_label);
      vcb::put_str(o, split);
      vcb::put_str(o, query_split);
      for (size_t i = 0; i < nq * k; ++i) vcb::put_u64(o, ids[i]);
      vcb::require(static_cast<bool>(o), TQ_ERR_INVALID_ARGUMENT, "write failed");
    }
    vcb::require(std::rename(tmp.c_str(), path) == 0, TQ_ERR_INVALID_ARGUMENT, "rename failed");
  });
}

int tq_vcex_read_header(const char* path, size_t* nq, size_t* k, uint64_t* index_n, uint64_t* seed) {
  return vcb::guarded([&] {
    vcb::require(path != nullptr, TQ_ERR_INVALID_ARGUMENT, "null path");
    std::ifstream in(path, std::ios::binary);
    vcb::require(static_cast<bool>(in), TQ_ERR_INVALID_ARGUMENT, "cannot open VCEX file");
    const vcb::VcexHeader h = vcb::read_vcex_header(in, path);
    if (nq) *nq = h.nq;
    if (k) *k = h.k;
    if (index_n) *index_n = h.index_n;
    if (seed) *seed = h.seed;
  });
}

int tq_vcex_read_ids(const char* path, uint64_t* ids) {
  return vcb::guarded([&] {
    vcb::require(path && ids, TQ_ERR_INVALID_ARGUMENT, "null argument");
    std::ifstream in(path, std::ios::binary);
    vcb::require(static_cast<bool>(in), TQ_ERR_INVALID_ARGUMENT, "cannot open VCEX file");
    const vcb::VcexHeader h = vcb::read_vcex_header(in, path);
    for (uint64_t i = 0; i < h.nq * h.k; ++i) ids[i] = vcb::get_u64(in);
  });
}

}  // extern "C"
