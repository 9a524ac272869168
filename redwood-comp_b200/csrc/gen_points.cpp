// Seeded synthetic point clouds (host side), see rw_tree_generate_points in
// include/rw_tree.h.  Input generation is not part of the timed pipeline.
#include <algorithm>
#include <cmath>
#include <random>
#include <thread>
#include <vector>

#include "rw_tree.h"

namespace {

// splitmix64 finaliser (Steele, Lea, Flood 2014), used as a counter-based
// generator: value(seed, i, lane) = mix(seed_mix + 16 i + lane).
inline uint64_t mix(uint64_t x) {
  x += 0x9e3779b97f4a7c15ull;
  x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
  x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
  return x ^ (x >> 31);
}

inline uint64_t draw(uint64_t seed_mix, uint64_t i, uint64_t lane) {
  return mix(seed_mix + 16 * i + lane);
}

// uniform in [0, 1) with 24 significant bits (exact in float)
inline float unit24(uint64_t h) { return float(h >> 40) * (1.0f / 16777216.0f); }

// uniform in (0, 1) in double, for Box-Muller
inline double unit53(uint64_t h) { return (double(h >> 11) + 0.5) * (1.0 / 9007199254740992.0); }

template <typename F>
void parallel_for(uint64_t n, F&& body) {
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  const uint64_t chunks = std::min<uint64_t>(hw, std::max<uint64_t>(1, n / 65536));
  if (chunks <= 1) {
    body(0, n);
    return;
  }
  std::vector<std::thread> th;
  th.reserve(chunks);
  for (uint64_t c = 0; c < chunks; ++c) {
    const uint64_t lo = n * c / chunks, hi = n * (c + 1) / chunks;
    th.emplace_back([&body, lo, hi] { body(lo, hi); });
  }
  for (auto& t : th) t.join();
}

}  // namespace

extern "C" int rw_tree_generate_points(float* out, uint64_t n, int32_t kind,
                                       uint64_t seed, float min_coord, float range,
                                       int32_t n_components, float sigma_lo,
                                       float sigma_hi) {
  if (!out || !(range > 0.0f)) return RW_ERR_ARG;
  const float hi_edge = std::nextafter(min_coord + range, min_coord);
  auto clampf = [&](float v) { return std::min(std::max(v, min_coord), hi_edge); };

  if (kind == RW_GEN_APPDATA) {
    // AppData (app_data.hpp:32-39): one mt19937 stream, draws in the order a
    // g++ build of glm::vec4(dis(gen), dis(gen), dis(gen), 1.0f) makes them.
    std::mt19937 gen(static_cast<std::mt19937::result_type>(seed));
    std::uniform_real_distribution<float> dis(min_coord, min_coord + range);
    for (uint64_t i = 0; i < n; ++i) {
      const float z = dis(gen);
      const float y = dis(gen);
      const float x = dis(gen);
      out[4 * i + 0] = x;
      out[4 * i + 1] = y;
      out[4 * i + 2] = z;
      out[4 * i + 3] = 1.0f;
    }
    return RW_OK;
  }

  const uint64_t sm = mix(seed ^ 0x5bd1e9955bd1e995ull);
  if (kind == RW_GEN_UNIFORM) {
    parallel_for(n, [&](uint64_t lo, uint64_t hi) {
      for (uint64_t i = lo; i < hi; ++i) {
        for (int a = 0; a < 3; ++a)
          out[4 * i + a] = clampf(min_coord + range * unit24(draw(sm, i, a)));
        out[4 * i + 3] = 1.0f;
      }
    });
    return RW_OK;
  }

  if (kind == RW_GEN_GAUSSIAN_MIXTURE) {
    if (n_components < 1 || !(sigma_lo > 0.0f) || sigma_hi < sigma_lo) return RW_ERR_ARG;
    const uint64_t cm = mix(sm ^ 0xc2b2ae3d27d4eb4full);
    std::vector<float> centre(3 * size_t(n_components)), sigma(n_components);
    for (int k = 0; k < n_components; ++k) {
      for (int a = 0; a < 3; ++a)
        centre[3 * k + a] = min_coord + range * unit24(draw(cm, uint64_t(k), a));
      sigma[k] = sigma_lo + (sigma_hi - sigma_lo) * unit24(draw(cm, uint64_t(k), 3));
    }
    const double two_pi = 6.283185307179586476925286766559;
    parallel_for(n, [&](uint64_t lo, uint64_t hi) {
      for (uint64_t i = lo; i < hi; ++i) {
        const int k = int(draw(sm, i, 0) % uint64_t(n_components));
        // two Box-Muller pairs -> three standard normals
        const double r0 = std::sqrt(-2.0 * std::log(unit53(draw(sm, i, 1))));
        const double t0 = two_pi * unit53(draw(sm, i, 2));
        const double r1 = std::sqrt(-2.0 * std::log(unit53(draw(sm, i, 3))));
        const double t1 = two_pi * unit53(draw(sm, i, 4));
        const double g[3] = {r0 * std::cos(t0), r0 * std::sin(t0), r1 * std::cos(t1)};
        for (int a = 0; a < 3; ++a)
          out[4 * i + a] =
              clampf(float(double(centre[3 * k + a]) + double(sigma[k]) * g[a]));
        out[4 * i + 3] = 1.0f;
      }
    });
    return RW_OK;
  }
  return RW_ERR_ARG;
}
