// Host-side data model of a scan (see scan.h).
#include "scan.h"

#include <algorithm>
#include <cfenv>
#include <cmath>

namespace ptyb {

namespace {

// Round half to even under the default rounding mode (Rust `f64::round_ties_even`).
double round_half_even(double v) { return std::nearbyint(v); }

// Rust `f64::rem_euclid(1.0)`.
double rem_euclid1(double v) {
  const double r = std::fmod(v, 1.0);
  return r < 0.0 ? r + 1.0 : r;
}

uint64_t mix(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

}  // namespace

// base/positions.rs:289-315.
std::vector<double> pynx_axis(const std::vector<double>& v, double px) {
  const size_t n = v.size();
  if (n == 0) return {};
  double s = 0.0;
  for (double a : v) s += a;
  const double mean = s / (double)n;
  std::vector<double> pos(n), frac(n);
  for (size_t i = 0; i < n; ++i) pos[i] = v[i] - mean;
  for (size_t i = 0; i < n; ++i) frac[i] = rem_euclid1(pos[i] / px);
  bool near = true;
  for (double d : frac) near = near && std::fabs(std::min(d, 1.0 - d)) < 0.1;
  if (near)
    for (size_t i = 0; i < n; ++i) frac[i] = rem_euclid1(pos[i] + 0.5) - 0.5;
  double fs = 0.0;
  for (double d : frac) fs += d;
  const double fmean = fs / (double)n;
  bool close = true;
  for (double d : frac) close = close && std::fabs(d - fmean) <= 0.02 + 1e-5 * std::fabs(fmean);
  if (close)
    for (size_t i = 0; i < n; ++i) pos[i] = round_half_even((pos[i] - fmean * px) / px) * px;
  return pos;
}

// base/addr.rs:123-127.
int64_t view_corner(int64_t obj, int64_t frame, double shift) {
  if (obj < frame) return -1;
  const int64_t span = obj - frame;
  const double c = round_half_even((double)(span / 2) + shift);
  if (!(c >= 0.0 && c <= (double)span)) return -1;
  return (int64_t)c;
}

// base/addr.rs:35-81 (corners only: every mode of a frame shares them).
bool corners_of(const std::vector<double>& y, const std::vector<double>& x, const double pixel[2],
                int ny, int nx, int nyo, int nxo, std::vector<int32_t>* out, std::string* err) {
  if (nyo < ny || nxo < nx) {
    *err = "object smaller than frame";
    return false;
  }
  out->resize(2 * y.size());
  for (size_t f = 0; f < y.size(); ++f) {
    const double dy = y[f] / pixel[0], dx = x[f] / pixel[1];
    const int64_t oy = view_corner(nyo, ny, dy), ox = view_corner(nxo, nx, dx);
    if (oy < 0 || ox < 0) {
      *err = "frame " + std::to_string(f) + " at (" + std::to_string(dy) + ", " +
             std::to_string(dx) + ") object pixels leaves the object";
      return false;
    }
    (*out)[2 * f] = (int32_t)oy;
    (*out)[2 * f + 1] = (int32_t)ox;
  }
  return true;
}

// engine/batch.rs:18-38.
void random_batches(int nframe, int size, uint64_t seed, uint64_t epoch, std::vector<int32_t>* order,
                    std::vector<int32_t>* sizes) {
  uint64_t state = seed ^ mix(epoch);
  order->resize(nframe);
  for (int i = 0; i < nframe; ++i) (*order)[i] = i;
  for (int i = nframe - 1; i >= 1; --i) {
    state += 0x9e3779b97f4a7c15ull;
    const unsigned __int128 r = (unsigned __int128)mix(state) * (unsigned __int128)(i + 1);
    const int j = (int)(r >> 64);
    std::swap((*order)[i], (*order)[j]);
  }
  sizes->clear();
  for (int s = 0; s < nframe; s += size) {
    const int e = std::min(nframe, s + size);
    std::sort(order->begin() + s, order->begin() + e);
    sizes->push_back(e - s);
  }
}

}  // namespace ptyb
