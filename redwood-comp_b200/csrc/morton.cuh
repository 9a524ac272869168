// Morton encode / decode on the device, bit-exact with the reference's CPU
// functions (apps/tree/host/func_morton.hpp:15-80).
//
// Float rules: the quantisation (c - min) / range * scale and the decode
// float(d) / scale * range + min use explicit round-to-nearest intrinsics so
// that no division is approximated and no multiply-add is contracted.
#pragma once

#include <stdint.h>

namespace rwt {

template <typename K>
struct KeyTraits;

// 32-bit keys: 10 bits per axis, 30-bit codes (func_morton.hpp:9,15-39).
template <>
struct KeyTraits<uint32_t> {
  static constexpr int kAxisBits = 10;
  static constexpr int kCodeBits = 30;
  static constexpr int kWordBits = 32;

  // Spread the low 10 bits of v so that bit b lands at bit 3b.
  __device__ __forceinline__ static uint32_t spread(uint32_t v) {
    v &= 0x3ffu;
    v = (v | (v << 16)) & 0x030000ffu;
    v = (v | (v << 8)) & 0x0300f00fu;
    v = (v | (v << 4)) & 0x030c30c3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
  }
  // Inverse of spread: gather bits 0, 3, 6, ... into the low 10 bits.
  __device__ __forceinline__ static uint32_t gather(uint32_t v) {
    v &= 0x09249249u;
    v = (v ^ (v >> 2)) & 0x030c30c3u;
    v = (v ^ (v >> 4)) & 0x0300f00fu;
    v = (v ^ (v >> 8)) & 0x030000ffu;
    v = (v ^ (v >> 16)) & 0x3ffu;
    return v;
  }
  __device__ __forceinline__ static int clz(uint32_t v) { return __clz(v); }
};

// 64-bit keys: 21 bits per axis, 63-bit codes (no reference counterpart).
template <>
struct KeyTraits<uint64_t> {
  static constexpr int kAxisBits = 21;
  static constexpr int kCodeBits = 63;
  static constexpr int kWordBits = 64;

  __device__ __forceinline__ static uint64_t spread(uint64_t v) {
    v &= 0x1fffffull;
    v = (v | (v << 32)) & 0x001f00000000ffffull;
    v = (v | (v << 16)) & 0x001f0000ff0000ffull;
    v = (v | (v << 8)) & 0x100f00f00f00f00full;
    v = (v | (v << 4)) & 0x10c30c30c30c30c3ull;
    v = (v | (v << 2)) & 0x1249249249249249ull;
    return v;
  }
  __device__ __forceinline__ static uint64_t gather(uint64_t v) {
    v &= 0x1249249249249249ull;
    v = (v ^ (v >> 2)) & 0x10c30c30c30c30c3ull;
    v = (v ^ (v >> 4)) & 0x100f00f00f00f00full;
    v = (v ^ (v >> 8)) & 0x001f0000ff0000ffull;
    v = (v ^ (v >> 16)) & 0x001f00000000ffffull;
    v = (v ^ (v >> 32)) & 0x1fffffull;
    return v;
  }
  __device__ __forceinline__ static int clz(uint64_t v) { return __clzll(v); }
};

// (c - min) / range * 2^axis_bits, truncated to unsigned, masked to the axis
// width (func_morton.hpp:27-30).  Coordinates below min are outside the
// reference's defined behaviour (its float->unsigned cast is undefined there).
// With POW2 the caller has checked that range is a power of two (2^k with k
// in [-126, 126]) and passes inv_range = 2^-k: (c - min) / range and
// (c - min) * 2^-k are then both the correctly rounded value of the same real
// number, so the product equals the IEEE quotient bit for bit.
template <typename K, bool POW2 = false>
__device__ __forceinline__ uint32_t quantise(float c, float min_coord, float range,
                                             float inv_range = 0.0f) {
  constexpr float kScale = float(1u << KeyTraits<K>::kAxisBits);
  const float d = __fsub_rn(c, min_coord);
  const float t = POW2 ? __fmul_rn(d, inv_range) : __fdiv_rn(d, range);
  const float q = __fmul_rn(t, kScale);
  return __float2uint_rz(q) & ((1u << KeyTraits<K>::kAxisBits) - 1u);
}

template <typename K, bool POW2 = false>
__device__ __forceinline__ K encode(float x, float y, float z, float min_coord,
                                    float range, float inv_range = 0.0f) {
  using T = KeyTraits<K>;
  const K ix = T::spread(K(quantise<K, POW2>(x, min_coord, range, inv_range)));
  const K iy = T::spread(K(quantise<K, POW2>(y, min_coord, range, inv_range)));
  const K iz = T::spread(K(quantise<K, POW2>(z, min_coord, range, inv_range)));
  return ix | (iy << 1) | (iz << 2);
}

// 2^-k when range = 2^k (k in [-126, 126]), else 0 (host side).
inline float pow2_reciprocal(float range) {
  uint32_t b;
  static_assert(sizeof(b) == sizeof(range), "float is 32 bits");
  __builtin_memcpy(&b, &range, 4);
  const uint32_t ex = (b >> 23) & 0xffu;
  if ((b & 0x807fffffu) != 0 || ex < 1 || ex > 253) return 0.0f;
  const uint32_t r = (254u - ex) << 23;
  float out;
  __builtin_memcpy(&out, &r, 4);
  return out;
}

// morton32_to_xyz (func_morton.hpp:60-80): float(d) / scale * range + min,
// w = 1.
template <typename K>
__device__ __forceinline__ float4 decode(K code, float min_coord, float range) {
  using T = KeyTraits<K>;
  constexpr float kScale = float(1u << T::kAxisBits);
  const float fx = __uint2float_rn(uint32_t(T::gather(code)));
  const float fy = __uint2float_rn(uint32_t(T::gather(code >> 1)));
  const float fz = __uint2float_rn(uint32_t(T::gather(code >> 2)));
  float4 r;
  // kScale is a power of two: dividing by it is multiplying by its exact
  // reciprocal (the same correctly rounded value)
  constexpr float kInv = 1.0f / kScale;
  r.x = __fadd_rn(__fmul_rn(__fmul_rn(fx, kInv), range), min_coord);
  r.y = __fadd_rn(__fmul_rn(__fmul_rn(fy, kInv), range), min_coord);
  r.z = __fadd_rn(__fmul_rn(__fmul_rn(fz, kInv), range), min_coord);
  r.w = 1.0f;
  return r;
}

// delta(a, b) = clz(a ^ b) - 1 over the key word (func_brt.hpp:27-33; kept
// with its -1 although 32-bit codes have two leading zero bits).
template <typename K>
__device__ __forceinline__ int delta(K a, K b) {
  return int(uint8_t(KeyTraits<K>::clz(a ^ b) - 1));
}

}  // namespace rwt
