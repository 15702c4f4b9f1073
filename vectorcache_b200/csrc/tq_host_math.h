// Host-side setup math for the flat TurboQuant index: rotation tables,
// Lloyd-Max codebook and the TQ+ anchor quantiles. Everything here runs once
// per index (or once per (bits, dim) pair, memoized) and is uploaded to HBM.
#pragma once

#include <cstddef>
#include <cstdint>
#include <vector>

namespace vcb {

constexpr std::size_t kMaxDim = 16384;

// dim must be a positive multiple of 8 and <= kMaxDim (rotation.cpp:140-145).
bool dim_supported(std::size_t dim);
bool bits_supported(std::size_t bits);
// Byte groups per vector: 8 / bits codes share one byte (pack.cpp:207-212).
inline std::size_t byte_groups(std::size_t bits, std::size_t dim) { return dim / (8 / bits); }
// Walsh-Hadamard block: the lowest set bit of dim (rotation.cpp:22).
inline std::size_t wht_block(std::size_t dim) { return dim & (~dim + 1); }

struct RotationTables {
  std::vector<float> signs;          // +-1 per output coordinate
  std::vector<std::uint32_t> perm;   // source coordinate per output coordinate
};

// One round of ChaCha8-driven signs and Fisher-Yates permutation
// (rotation.cpp:139-160).
RotationTables make_rotation(std::size_t dim);

struct Codebook {
  std::vector<float> boundaries;  // 2^bits - 1, f32 midpoints of the centroids
  std::vector<float> centroids;   // 2^bits, increasing
};

// Lloyd-Max codebook on Beta((dim-1)/2, (dim-1)/2) mapped to [-1, 1]
// (codebook.cpp:135-226). Memoized and thread-safe.
const Codebook& codebook(std::size_t bits, std::size_t dim);

// A table that turns the code of a value (the count of codebook boundaries
// strictly below it, encode.cpp:126-140) into one fused multiply-add, one
// table read and one compare. The device computes, for c clamped to
// [lo, hi], t = fmaf(c, a, k) in [2^23, 2^24) and the cell j = bits(t) -
// bits(2^23 + 2^22): a monotone function of c, so every cell is an interval.
// The host evaluates that same rounding exactly for every boundary and keeps
// at most one boundary per cell; then code(c) = base[j] + (c > inner[j]),
// exactly the count for every float c (NaN: 0).
struct CodeGrid {
  static constexpr int kCells = 64;
  float lo = 0.f, hi = 0.f, a = 0.f, k = 0.f;
  std::uint32_t base[kCells] = {};  // boundaries in earlier cells
  float inner[kCells] = {};         // the boundary inside the cell, or +inf
};
// False when no grid separates the boundaries (callers keep the binary search).
bool make_code_grid(const std::vector<float>& boundaries, CodeGrid* out);

// Regularized incomplete beta I_t(a, a) (encode.cpp:95-112).
double beta_cdf_aa(double a, double t);

// Order-statistic ranks of the TQ+ fit for an n-row sample: the lo/hi sorted
// positions per dimension and the centroid span they map to
// (encode.cpp:233-261).
struct TqplusAnchor {
  std::size_t lo_idx = 0;
  std::size_t hi_idx = 0;
  float qc_lo = 0.f;    // -max|centroid|
  float qc_span = 0.f;  // 2 * max|centroid|
};
TqplusAnchor tqplus_anchor(std::size_t n, std::size_t bits, std::size_t dim);

}  // namespace vcb
