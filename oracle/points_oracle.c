/* Test infrastructure, not product code.
 *
 * CPU restatement of the library's seeded point generators
 * (rw_tree_generate_points, RW_GEN_UNIFORM and RW_GEN_GAUSSIAN_MIXTURE), so
 * that the reference arm of the benchmark and the CPU tests can build the
 * same clouds without loading the product library.  The reference's own
 * generator (AppData's mt19937 stream, apps/tree/app_data.hpp:32-39) comes
 * from the reference itself in _ref/ (ref_default_points).
 *
 * Counter-based draws: value(seed, i, lane) = splitmix64(seed_mix + 16 i +
 * lane), the splitmix64 finaliser of Steele, Lea and Flood (2014).  Uniform
 * coordinates take the top 24 bits of a draw (exact in float); the mixture
 * picks a component by draw % k and three standard normals from two
 * Box-Muller pairs in double precision.  Coordinates are clamped into
 * [min, nextafterf(min + range, min)].  Compiled without contraction or fast
 * math so that every float and double operation rounds as written.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>

#include "tree_oracle.h"

static uint64_t mix64(uint64_t x) {
  x += 0x9e3779b97f4a7c15ull;
  x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
  x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
  return x ^ (x >> 31);
}

static uint64_t draw(uint64_t seed_mix, uint64_t i, uint64_t lane) {
  return mix64(seed_mix + 16u * i + lane);
}

static float unit24(uint64_t h) { return (float)(h >> 40) * (1.0f / 16777216.0f); }

static double unit53(uint64_t h) {
  return ((double)(h >> 11) + 0.5) * (1.0 / 9007199254740992.0);
}

static float clamp_box(float v, float lo, float hi) {
  const float a = (v < lo) ? lo : v;
  return (hi < a) ? hi : a;
}

int orc_generate_points(float* out, uint64_t n, int kind, uint64_t seed, float min_coord,
                        float range, int n_components, float sigma_lo, float sigma_hi) {
  if (!out || !(range > 0.0f)) return ORC_ERR_ARG;
  const float hi_edge = nextafterf(min_coord + range, min_coord);
  const uint64_t sm = mix64(seed ^ 0x5bd1e9955bd1e995ull);
  if (kind == ORC_GEN_UNIFORM) {
    for (uint64_t i = 0; i < n; ++i) {
      for (int a = 0; a < 3; ++a)
        out[4 * i + a] =
            clamp_box(min_coord + range * unit24(draw(sm, i, (uint64_t)a)), min_coord, hi_edge);
      out[4 * i + 3] = 1.0f;
    }
    return ORC_OK;
  }
  if (kind != ORC_GEN_GAUSSIAN_MIXTURE) return ORC_ERR_ARG;
  if (n_components < 1 || !(sigma_lo > 0.0f) || sigma_hi < sigma_lo) return ORC_ERR_ARG;
  const uint64_t cm = mix64(sm ^ 0xc2b2ae3d27d4eb4full);
  float* centre = (float*)malloc(sizeof(float) * 3u * (size_t)n_components);
  float* sigma = (float*)malloc(sizeof(float) * (size_t)n_components);
  if (!centre || !sigma) {
    free(centre);
    free(sigma);
    return ORC_ERR_ARG;
  }
  for (int k = 0; k < n_components; ++k) {
    for (int a = 0; a < 3; ++a)
      centre[3 * k + a] = min_coord + range * unit24(draw(cm, (uint64_t)k, (uint64_t)a));
    sigma[k] = sigma_lo + (sigma_hi - sigma_lo) * unit24(draw(cm, (uint64_t)k, 3));
  }
  const double two_pi = 6.283185307179586476925286766559;
  for (uint64_t i = 0; i < n; ++i) {
    const int k = (int)(draw(sm, i, 0) % (uint64_t)n_components);
    const double r0 = sqrt(-2.0 * log(unit53(draw(sm, i, 1))));
    const double t0 = two_pi * unit53(draw(sm, i, 2));
    const double r1 = sqrt(-2.0 * log(unit53(draw(sm, i, 3))));
    const double t1 = two_pi * unit53(draw(sm, i, 4));
    const double g[3] = {r0 * cos(t0), r0 * sin(t0), r1 * cos(t1)};
    for (int a = 0; a < 3; ++a)
      out[4 * i + a] = clamp_box(
          (float)((double)centre[3 * k + a] + (double)sigma[k] * g[a]), min_coord, hi_edge);
    out[4 * i + 3] = 1.0f;
  }
  free(centre);
  free(sigma);
  return ORC_OK;
}
