// Seeded synthetic tile generators for the benchmark workloads.
//
// Counter-based randomness (splitmix64 keyed by seed) so that every tile is
// reproducible from (master seed, workload, tile index) alone.
#include <algorithm>
#include <cmath>
#include <cstdint>

#include "j2k_encode.h"

namespace sgn {
namespace synth {

struct Rng {
  uint64_t s;
  explicit Rng(uint64_t seed) : s(seed) {}
  uint64_t next() {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
  double uniform() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
  double normal() {
    double u1 = uniform(), u2 = uniform();
    if (u1 < 1e-300) u1 = 1e-300;
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
  }
  // Poisson sample: inversion for small means, PTRS (Hormann 1993) otherwise.
  uint32_t poisson(double mean) {
    if (mean < 30.0) {
      double L = std::exp(-mean), p = 1.0;
      uint32_t k = 0;
      do {
        ++k;
        p *= uniform();
      } while (p > L);
      return k - 1;
    }
    double slam = std::sqrt(mean), loglam = std::log(mean);
    double b = 0.931 + 2.53 * slam, a = -0.059 + 0.02483 * b;
    double invalpha = 1.1239 + 1.1328 / (b - 3.4), vr = 0.9277 - 3.6224 / (b - 2);
    for (;;) {
      double U = uniform() - 0.5, V = uniform();
      double us = 0.5 - std::fabs(U);
      double k = std::floor((2 * a / us + b) * U + mean + 0.43);
      if (us >= 0.07 && V <= vr) return (uint32_t)k;
      if (k < 0 || (us < 0.013 && V > us)) continue;
      if (std::log(V) + std::log(invalpha) - std::log(a / (us * us) + b) <= -mean + k * loglam - std::lgamma(k + 1))
        return (uint32_t)k;
    }
  }
};

static inline uint8_t clamp_u8(double v) {
  double r = std::nearbyint(v);
  return (uint8_t)std::min(255.0, std::max(0.0, r));
}

// H&E-like RGB8 field: two stain colours (200,120,180) and (90,60,150) blended
// over a (240,238,242) background by a sum of six low-frequency sinusoids
// (periods side/8 .. side/1, random phase and orientation), plus N(0, sigma^2)
// noise per channel.
void he_tile(uint64_t seed, uint32_t w, uint32_t h, double sigma, uint8_t* out) {
  Rng r(seed);
  const double side = (double)std::max(w, h);
  double fx[6], fy[6], ph[6], amp[6];
  for (int k = 0; k < 6; ++k) {
    double period = side / (1.0 + 7.0 * r.uniform());
    double th = 6.283185307179586 * r.uniform();
    fx[k] = std::cos(th) / period * 6.283185307179586;
    fy[k] = std::sin(th) / period * 6.283185307179586;
    ph[k] = 6.283185307179586 * r.uniform();
    amp[k] = 0.5 + 0.5 * r.uniform();
  }
  const double bg[3] = {240, 238, 242}, ca[3] = {200, 120, 180}, cb[3] = {90, 60, 150};
  for (uint32_t y = 0; y < h; ++y)
    for (uint32_t x = 0; x < w; ++x) {
      double sa = 0, sb = 0;
      for (int k = 0; k < 3; ++k) sa += amp[k] * std::sin(fx[k] * x + fy[k] * y + ph[k]);
      for (int k = 3; k < 6; ++k) sb += amp[k] * std::sin(fx[k] * x + fy[k] * y + ph[k]);
      double a = std::min(1.0, std::max(0.0, sa / 1.5)), b = std::min(1.0, std::max(0.0, sb / 1.5));
      if (a + b > 1.0) {
        double s = a + b;
        a /= s;
        b /= s;
      }
      uint8_t* o = out + ((size_t)y * w + x) * 3;
      for (int c = 0; c < 3; ++c) {
        double v = bg[c] + a * (ca[c] - bg[c]) + b * (cb[c] - bg[c]);
        if (sigma > 0) v += sigma * r.normal();
        o[c] = clamp_u8(v);
      }
    }
}

// Near-blank RGB8 background: every sample uniform in 240 +/- 2.
void blank_tile(uint64_t seed, uint32_t w, uint32_t h, uint8_t* out) {
  Rng r(seed);
  for (size_t i = 0; i < (size_t)w * h * 3; ++i) out[i] = (uint8_t)(238 + (r.next() % 5));
}

// Fluorescence-like u16 gray (little-endian): Poisson counts around a mean of
// 50 plus eight Gaussian blobs (sigma 64..256 px) scaled to peak near 4000.
void fluor_tile(uint64_t seed, uint32_t w, uint32_t h, uint8_t* out_le16) {
  Rng r(seed);
  double cx[8], cy[8], s2[8], amp[8];
  for (int k = 0; k < 8; ++k) {
    cx[k] = r.uniform() * w;
    cy[k] = r.uniform() * h;
    double s = 64.0 + 192.0 * r.uniform();
    s2[k] = 2.0 * s * s;
    amp[k] = 3950.0 * (0.25 + 0.75 * r.uniform());
  }
  for (uint32_t y = 0; y < h; ++y)
    for (uint32_t x = 0; x < w; ++x) {
      double m = 0;
      for (int k = 0; k < 8; ++k) {
        double dx = x - cx[k], dy = y - cy[k];
        m += amp[k] * std::exp(-(dx * dx + dy * dy) / s2[k]);
      }
      m = 50.0 + std::min(m, 3950.0);
      uint32_t v = std::min<uint32_t>(r.poisson(m), 65535);
      out_le16[((size_t)y * w + x) * 2] = (uint8_t)(v & 0xFF);
      out_le16[((size_t)y * w + x) * 2 + 1] = (uint8_t)(v >> 8);
    }
}

}  // namespace synth
}  // namespace sgn
