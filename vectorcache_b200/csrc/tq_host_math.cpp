// Host-side setup math: ChaCha8 rotation tables, Lloyd-Max Beta codebook and
// the TQ+ anchor quantile ranks.
//
// The reference builds this code with -O3 -mavx2 -mfma -ffp-contract=fast
// (CMakeLists.txt:62-66), which fuses a multiply into the add that consumes it
// whenever the product has no other use. The codebook's f32 centroids and the
// TQ+ ranks must come out bit-identical, so this file is compiled with
// -ffp-contract=off and spells each of those fusions out with std::fma.
#include "tq_host_math.h"

#include <array>
#include <cmath>
#include <cstring>
#include <limits>
#include <map>
#include <mutex>
#include <utility>

namespace vcb {
namespace {

// ---------------------------------------------------------------------------
// ChaCha8 (chacha8.cpp:34-85): RFC 7539 state layout, 32-byte key, 64-bit
// block counter in words 12..13, zero nonce, four double rounds.
class ChaCha8 {
 public:
  explicit ChaCha8(const std::array<std::uint8_t, 32>& key) {
    state_[0] = 0x61707865u;
    state_[1] = 0x3320646eu;
    state_[2] = 0x79622d32u;
    state_[3] = 0x6b206574u;
    for (int w = 0; w < 8; ++w) {
      std::uint32_t v = 0;
      for (int b = 3; b >= 0; --b) v = (v << 8) | key[static_cast<std::size_t>(4 * w + b)];
      state_[static_cast<std::size_t>(4 + w)] = v;
    }
  }

  std::uint32_t next32() {
    if (used_ == 16) generate();
    return block_[used_++];
  }

  std::uint64_t next64() {
    const std::uint64_t lo = next32();
    return lo | (static_cast<std::uint64_t>(next32()) << 32);
  }

 private:
  static std::uint32_t rotl(std::uint32_t v, int s) { return (v << s) | (v >> (32 - s)); }
  static void qr(std::uint32_t* x, int a, int b, int c, int d) {
    x[a] += x[b]; x[d] = rotl(x[d] ^ x[a], 16);
    x[c] += x[d]; x[b] = rotl(x[b] ^ x[c], 12);
    x[a] += x[b]; x[d] = rotl(x[d] ^ x[a], 8);
    x[c] += x[d]; x[b] = rotl(x[b] ^ x[c], 7);
  }

  void generate() {
    std::array<std::uint32_t, 16> x = state_;
    for (int round = 0; round < 4; ++round) {
      qr(x.data(), 0, 4, 8, 12);
      qr(x.data(), 1, 5, 9, 13);
      qr(x.data(), 2, 6, 10, 14);
      qr(x.data(), 3, 7, 11, 15);
      qr(x.data(), 0, 5, 10, 15);
      qr(x.data(), 1, 6, 11, 12);
      qr(x.data(), 2, 7, 8, 13);
      qr(x.data(), 3, 4, 9, 14);
    }
    for (std::size_t i = 0; i < 16; ++i) block_[i] = x[i] + state_[i];
    if (++state_[12] == 0) ++state_[13];
    used_ = 0;
  }

  std::array<std::uint32_t, 16> state_{};
  std::array<std::uint32_t, 16> block_{};
  std::size_t used_ = 16;
};

// Rotation seed bytes (rotation.cpp:18-20).
constexpr std::array<std::uint8_t, 32> kSeed = {164, 143, 161, 123, 88,  50,  61,  10,
                                                234, 184, 161, 204, 105, 1,   20,  184,
                                                43,  140, 200, 117, 24,  180, 247, 84,
                                                141, 68,  110, 161, 228, 223, 32,  242};

// ---------------------------------------------------------------------------
// Special functions in double.
constexpr double kPi = 3.14159265358979323846;

// Lanczos approximation of log Gamma with g = 7 and the usual nine-term
// coefficient table (codebook.cpp:14-31).
double log_gamma(double z) {
  constexpr double kLanczos[9] = {0.99999999999980993,  676.5203681218851,
                                  -1259.1392167224028,  771.32342877765313,
                                  -176.61502916214059,  12.507343278686905,
                                  -0.13857109526572012, 9.984369654078861e-6,
                                  1.5056327351493116e-7};
  if (z < 0.5) return std::log(kPi) - std::log(std::sin(kPi * z)) - log_gamma(1.0 - z);
  z -= 1.0;
  double series = kLanczos[0];
  for (int i = 1; i < 9; ++i) series += kLanczos[i] / (z + static_cast<double>(i));
  const double t = z + 7.5;
  static const double half_log_2pi = 0.5 * std::log(2.0 * kPi);
  return std::fma(z + 0.5, std::log(t), half_log_2pi) - t + std::log(series);
}

// Lentz continued fraction of the incomplete beta (codebook.cpp:33-79).
double beta_continued_fraction(double a, double b, double x) {
  constexpr double kTiny = 1e-30;
  const double sum_ab = a + b, a_plus = a + 1.0, a_minus = a - 1.0;
  auto guard = [](double v) { return std::fabs(v) < kTiny ? kTiny : v; };
  double c = 1.0;
  double d = 1.0 / guard(1.0 - sum_ab * x / a_plus);
  double h = d;
  for (int m = 1; m <= 200; ++m) {
    const double md = static_cast<double>(m);
    const double two_m = 2.0 * md;
    const double even = md * (b - md) * x / ((a_minus + two_m) * (a + two_m));
    d = 1.0 / guard(std::fma(even, d, 1.0));
    c = guard(1.0 + even / c);
    h *= d * c;
    const double odd = -(a + md) * (sum_ab + md) * x / ((a + two_m) * (a_plus + two_m));
    d = 1.0 / guard(std::fma(odd, d, 1.0));
    c = guard(1.0 + odd / c);
    const double step = d * c;
    h *= step;
    if (std::fabs(step - 1.0) < 3e-14) break;
  }
  return h;
}

double incomplete_beta(double a, double b, double x) {
  if (x <= 0.0) return 0.0;
  if (x >= 1.0) return 1.0;
  const double log_beta = log_gamma(a) + log_gamma(b) - log_gamma(a + b);
  const double front = std::exp(std::fma(std::log(x), a, std::log(1.0 - x) * b) - log_beta);
  if (x < (a + 1.0) / (a + b + 2.0)) return front / a * beta_continued_fraction(a, b, x);
  return std::fma(-(front / b), beta_continued_fraction(b, a, 1.0 - x), 1.0);
}

// Density of Beta(a, a) on (0, 1).
double beta_density(double a, double t) {
  if (t <= 0.0 || t >= 1.0) return 0.0;
  const double log_beta = 2.0 * log_gamma(a) - log_gamma(2.0 * a);
  const double am1 = a - 1.0;
  return std::exp(std::fma(am1, std::log(t), am1 * std::log(1.0 - t)) - log_beta);
}

// First moment x * f(x) of the coordinate law x = 2 * Beta(a, a) - 1.
struct FirstMoment {
  double a;
  double operator()(double x) const { return x * beta_density(a, (x + 1.0) / 2.0) / 2.0; }
};

// Adaptive Simpson with Richardson correction, tolerance halved per level and
// a depth limit (codebook.cpp:112-133).
double simpson_refine(const FirstMoment& f, double lo, double hi, double f_lo, double f_hi,
                      double f_mid, double whole, double tol, int depth) {
  const double mid = (lo + hi) / 2.0;
  const double f_q1 = f((lo + mid) / 2.0);
  const double f_q3 = f((mid + hi) / 2.0);
  const double left = (mid - lo) / 6.0 * (f_lo + 4.0 * f_q1 + f_mid);
  const double right = (hi - mid) / 6.0 * (f_mid + 4.0 * f_q3 + f_hi);
  const double sum = left + right;
  if (depth == 0 || std::fabs(sum - whole) < 15.0 * tol) return sum + (sum - whole) / 15.0;
  return simpson_refine(f, lo, mid, f_lo, f_mid, f_q1, left, tol / 2.0, depth - 1) +
         simpson_refine(f, mid, hi, f_mid, f_hi, f_q3, right, tol / 2.0, depth - 1);
}

double integrate_first_moment(double a, double lo, double hi) {
  const FirstMoment f{a};
  const double mid = (lo + hi) / 2.0;
  const double f_lo = f(lo), f_hi = f(hi), f_mid = f(mid);
  const double whole = (hi - lo) / 6.0 * (f_lo + 4.0 * f_mid + f_hi);
  return simpson_refine(f, lo, hi, f_lo, f_hi, f_mid, whole, 1e-14, 50);
}

Codebook lloyd_max(std::size_t bits, std::size_t dim) {
  const double a = (static_cast<double>(dim) - 1.0) / 2.0;
  const std::size_t levels = std::size_t{1} << bits;
  const double sd = std::sqrt(2.0 * a / ((2.0 * a + 1.0) * 4.0 * a));
  const double spread = 3.0 * sd;
  std::vector<double> c(levels), next(levels), edges(levels + 1);
  for (std::size_t i = 0; i < levels; ++i) {
    c[i] = -spread + 2.0 * spread * static_cast<double>(i) / static_cast<double>(levels - 1);
  }
  for (int iter = 0; iter < 200; ++iter) {
    edges.front() = -1.0;
    edges.back() = 1.0;
    for (std::size_t i = 0; i + 1 < levels; ++i) edges[i + 1] = (c[i] + c[i + 1]) / 2.0;
    for (std::size_t i = 0; i < levels; ++i) {
      const double mass = incomplete_beta(a, a, (edges[i + 1] + 1.0) / 2.0) -
                          incomplete_beta(a, a, (edges[i] + 1.0) / 2.0);
      next[i] = mass < 1e-15 ? c[i] : integrate_first_moment(a, edges[i], edges[i + 1]) / mass;
    }
    double largest_move = 0.0;
    for (std::size_t i = 0; i < levels; ++i) {
      largest_move = std::max(largest_move, std::fabs(c[i] - next[i]));
    }
    c.swap(next);
    if (largest_move < 1e-12) break;
  }
  Codebook out;
  out.centroids.resize(levels);
  for (std::size_t i = 0; i < levels; ++i) out.centroids[i] = static_cast<float>(c[i]);
  out.boundaries.resize(levels - 1);
  for (std::size_t i = 0; i + 1 < levels; ++i) {
    out.boundaries[i] = (out.centroids[i] + out.centroids[i + 1]) * 0.5f;
  }
  return out;
}

}  // namespace

bool dim_supported(std::size_t dim) { return dim > 0 && dim % 8 == 0 && dim <= kMaxDim; }
bool bits_supported(std::size_t bits) { return bits >= 2 && bits <= 4; }

RotationTables make_rotation(std::size_t dim) {
  RotationTables t;
  ChaCha8 rng(kSeed);
  t.signs.resize(dim);
  for (auto& s : t.signs) s = (rng.next32() & 1u) ? -1.f : 1.f;
  t.perm.resize(dim);
  for (std::size_t i = 0; i < dim; ++i) t.perm[i] = static_cast<std::uint32_t>(i);
  for (std::size_t i = dim; i-- > 1;) {
    const std::size_t j = static_cast<std::size_t>(rng.next64() % (static_cast<std::uint64_t>(i) + 1));
    std::swap(t.perm[i], t.perm[j]);
  }
  return t;
}

const Codebook& codebook(std::size_t bits, std::size_t dim) {
  static std::mutex mu;
  static std::map<std::pair<std::size_t, std::size_t>, Codebook> memo;
  {
    std::lock_guard<std::mutex> lock(mu);
    auto it = memo.find({bits, dim});
    if (it != memo.end()) return it->second;
  }
  Codebook cb = lloyd_max(bits, dim);
  std::lock_guard<std::mutex> lock(mu);
  return memo.emplace(std::make_pair(bits, dim), std::move(cb)).first->second;
}

double beta_cdf_aa(double a, double t) { return incomplete_beta(a, a, t); }

TqplusAnchor tqplus_anchor(std::size_t n, std::size_t bits, std::size_t dim) {
  const Codebook& cb = codebook(bits, dim);
  float c_outer = 0.f;
  for (float c : cb.centroids) c_outer = std::max(c_outer, std::fabs(c));
  const double a = (static_cast<double>(dim) - 1.0) / 2.0;
  const double p_hi = incomplete_beta(a, a, (static_cast<double>(c_outer) + 1.0) / 2.0);
  const double p_lo = 1.0 - p_hi;
  TqplusAnchor out;
  out.lo_idx = static_cast<std::size_t>(static_cast<double>(n) * p_lo);
  out.hi_idx = static_cast<std::size_t>(static_cast<double>(n) * p_hi);
  out.hi_idx = std::min(out.hi_idx, n - 1);
  out.hi_idx = std::max(out.hi_idx, out.lo_idx + 1);
  out.qc_lo = -c_outer;
  out.qc_span = c_outer - (-c_outer);
  return out;
}

namespace {

// Cell of c as the device computes it: t = fmaf(c, a, k) rounded once to
// float; returns false when the exact value of c * a + k lies too close to a
// float rounding tie for the long-double evaluation to decide it.
bool grid_cell(float c, float a, float k, int* cell) {
  const long double exact = static_cast<long double>(c) * static_cast<long double>(a) + static_cast<long double>(k);
  // t in [2^23, 2^24): one float ulp is 1, so the rounding point is the
  // nearest integer; stay away from .5 by far more than the long double error.
  const long double frac = exact - std::floor(exact);
  if (std::fabs(frac - 0.5L) < 1e-6L) return false;
  const float t = static_cast<float>(exact);
  if (!(t >= 8388608.f && t < 16777216.f)) return false;
  std::uint32_t bits;
  std::memcpy(&bits, &t, 4);
  *cell = static_cast<int>(bits) - 0x4B400000;
  return true;
}

}  // namespace

bool make_code_grid(const std::vector<float>& b, CodeGrid* out) {
  if (b.empty()) return false;
  const float first = b.front(), last = b.back();
  const float span = last - first;
  if (!(span > 0.f)) return false;
  CodeGrid g;
  g.lo = first - span / 8.f;
  g.hi = last + span / 8.f;
  for (int attempt = 0; attempt < 64; ++attempt) {
    // About kCells - 4 cells across [lo, hi], cell(lo) near 1; the slope
    // changes a little between attempts to move every value off a rounding
    // tie (k is an integer: floats near 2^23 have unit spacing).
    g.a = static_cast<float>((CodeGrid::kCells - 4.0 - 0.013 * attempt) / (static_cast<double>(g.hi) - g.lo));
    g.k = static_cast<float>(std::floor(12582912.0 + 1.25 - static_cast<double>(g.lo) * g.a));
    int c_lo = 0, c_hi = 0;
    if (!grid_cell(g.lo, g.a, g.k, &c_lo) || !grid_cell(g.hi, g.a, g.k, &c_hi)) continue;
    if (c_lo < 0 || c_hi > CodeGrid::kCells - 1) continue;
    bool ok = true;
    int prev = -1;
    std::vector<int> cells(b.size());
    for (std::size_t i = 0; i < b.size() && ok; ++i) {
      ok = grid_cell(b[i], g.a, g.k, &cells[i]) && cells[i] > prev && cells[i] >= c_lo && cells[i] <= c_hi;
      prev = cells[i];
    }
    if (!ok) continue;
    const float inf = std::numeric_limits<float>::infinity();
    std::size_t next = 0;
    for (int j = 0; j < CodeGrid::kCells; ++j) {
      g.base[j] = static_cast<std::uint32_t>(next);
      g.inner[j] = inf;
      if (next < b.size() && cells[next] == j) {
        g.inner[j] = b[next];
        ++next;
      }
    }
    *out = g;
    return true;
  }
  return false;
}

}  // namespace vcb
