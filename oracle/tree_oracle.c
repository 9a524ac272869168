/* Test infrastructure, not product code: CPU restatement of the reference tree
 * pipeline used as the parity checker.  See tree_oracle.h for the dataflow.
 * Plain sequential C on purpose: stage 4 and stage 7 are defined by their
 * ascending-index order, which a sequential loop states directly.
 */
#include "tree_oracle.h"

#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------ */
/* key access                                                               */
/* ------------------------------------------------------------------------ */

static inline uint64_t kget(const void* a, int bits, size_t i) {
  return bits == 32 ? (uint64_t)((const uint32_t*)a)[i]
                    : ((const uint64_t*)a)[i];
}

static inline void kset(void* a, int bits, size_t i, uint64_t v) {
  if (bits == 32)
    ((uint32_t*)a)[i] = (uint32_t)v;
  else
    ((uint64_t*)a)[i] = v;
}

/* code width in bits: 30 for 32-bit keys (func_morton.hpp:9), 63 for 64-bit */
static inline int code_bits(int bits) { return bits == 32 ? 30 : 63; }
static inline int axis_bits(int bits) { return bits == 32 ? 10 : 21; }

uint32_t orc_capacity(uint32_t n_input) {
  /* AppData: oct(n_input * k_memory_ratio) with k_memory_ratio = 0.6f
   * (app_data.hpp:13,28): the product is computed in float, then truncated. */
  const float rows = (float)n_input * 0.6f;
  return (uint32_t)rows;
}

uint64_t orc_fnv1a64(const void* data, size_t bytes) {
  const unsigned char* p = (const unsigned char*)data;
  uint64_t h = 0xcbf29ce484222325ull;
  for (size_t i = 0; i < bytes; ++i) {
    h ^= p[i];
    h *= 0x100000001b3ull;
  }
  return h;
}

/* ------------------------------------------------------------------------ */
/* stage 1: Morton encode (func_morton.hpp:15-39)                           */
/* ------------------------------------------------------------------------ */

/* quantise one coordinate: (c - min) / range * bit_scale, IEEE float ops in
 * that order, then truncation to unsigned and the per-axis mask
 * (func_morton.hpp:27-30 and the `& 0x3ff` of :16). */
static inline uint32_t quantise(float c, float min_coord, float range,
                                int abits) {
  const float scale = (float)(1u << abits);
  const float q = (c - min_coord) / range * scale;
  const uint32_t u = (uint32_t)(int64_t)q;
  return u & ((1u << abits) - 1u);
}

/* bit-by-bit interleave: x at bit 3b, y at 3b+1, z at 3b+2.  Written as a
 * loop (not the magic-number spread of func_morton.hpp:15-22) so that the
 * checker and the GPU kernel are independent implementations. */
static inline uint64_t interleave3(uint32_t x, uint32_t y, uint32_t z,
                                   int abits) {
  uint64_t code = 0;
  for (int b = 0; b < abits; ++b) {
    code |= (uint64_t)((x >> b) & 1u) << (3 * b);
    code |= (uint64_t)((y >> b) & 1u) << (3 * b + 1);
    code |= (uint64_t)((z >> b) & 1u) << (3 * b + 2);
  }
  return code;
}

void orc_morton(const float* points, void* keys, uint32_t n, int key_bits,
                float min_coord, float range) {
  const int ab = axis_bits(key_bits);
  for (uint32_t i = 0; i < n; ++i) {
    const float* p = points + 4 * (size_t)i;
    const uint32_t x = quantise(p[0], min_coord, range, ab);
    const uint32_t y = quantise(p[1], min_coord, range, ab);
    const uint32_t z = quantise(p[2], min_coord, range, ab);
    kset(keys, key_bits, i, interleave3(x, y, z, ab));
  }
}

/* decode of a (prefix-shifted) code to a corner (func_morton.hpp:45-80):
 * float(d) / bit_scale * range + min per axis, w = 1. */
static void decode(uint64_t code, int key_bits, float min_coord, float range,
                   float* out4) {
  const int ab = axis_bits(key_bits);
  const float scale = (float)(1u << ab);
  for (int axis = 0; axis < 3; ++axis) {
    uint32_t d = 0;
    for (int b = 0; b < ab; ++b) d |= (uint32_t)((code >> (3 * b + axis)) & 1u) << b;
    const float f = (float)d;
    const float q = f / scale;
    const float s = q * range;
    out4[axis] = s + min_coord;
  }
  out4[3] = 1.0f;
}

int orc_stage1(orc_tree* t) {
  if (!t || t->n_input < 1) return ORC_ERR_ARG;
  orc_morton(t->points, t->keys, t->n_input, t->key_bits, t->min_coord,
             t->range);
  return ORC_OK;
}

/* ------------------------------------------------------------------------ */
/* stage 2: stable LSD radix sort, 8-bit digits (func_sort.cpp:117-171)     */
/* ------------------------------------------------------------------------ */

void orc_sort(void* keys, uint32_t n, int key_bits) {
  if (n < 2) return;
  const size_t esz = key_bits == 32 ? 4 : 8;
  void* tmp = malloc(esz * n);
  void* src = keys;
  void* dst = tmp;
  const int passes = (code_bits(key_bits) + 7) / 8;
  for (int pass = 0; pass < passes; ++pass) {
    const int shift = 8 * pass;
    size_t count[256] = {0};
    for (uint32_t i = 0; i < n; ++i)
      ++count[(kget(src, key_bits, i) >> shift) & 0xff];
    size_t run = 0;
    for (int d = 0; d < 256; ++d) {
      const size_t c = count[d];
      count[d] = run;
      run += c;
    }
    for (uint32_t i = 0; i < n; ++i) {
      const uint64_t k = kget(src, key_bits, i);
      kset(dst, key_bits, count[(k >> shift) & 0xff]++, k);
    }
    void* s = src;
    src = dst;
    dst = s;
  }
  if (src != keys) memcpy(keys, src, esz * n);
  free(tmp);
}

int orc_stage2(orc_tree* t) {
  if (!t || t->n_input < 1) return ORC_ERR_ARG;
  const size_t esz = t->key_bits == 32 ? 4 : 8;
  memcpy(t->keys_alt, t->keys, esz * t->n_input);
  orc_sort(t->keys_alt, t->n_input, t->key_bits);
  return ORC_OK;
}

/* ------------------------------------------------------------------------ */
/* stage 3: unique copy sorted -> keys (host_dispatchers.cpp:183-194)       */
/* ------------------------------------------------------------------------ */

int orc_stage3(orc_tree* t) {
  if (!t || t->n_input < 1) return ORC_ERR_ARG;
  uint32_t u = 0;
  for (uint32_t i = 0; i < t->n_input; ++i) {
    const uint64_t k = kget(t->keys_alt, t->key_bits, i);
    if (i == 0 || k != kget(t->keys_alt, t->key_bits, i - 1))
      kset(t->keys, t->key_bits, u++, k);
  }
  t->n_unique = u;
  t->n_brt_nodes = u - 1;
  return ORC_OK;
}

/* ------------------------------------------------------------------------ */
/* stage 4: Karras radix tree (func_brt.hpp:22-138)                         */
/* ------------------------------------------------------------------------ */

/* delta = clz(a ^ b) - 1 over the key word (func_brt.hpp:27-33), kept with
 * its -1 even though 32-bit codes have two leading zero bits; with
 * ORC_OPT_GEOMETRIC_DELTA, 32-bit keys subtract one more (g_delta_bias). */
static int g_delta_bias = 0;

static inline int delta(uint64_t a, uint64_t b, int key_bits) {
  if (key_bits == 32)
    return (uint8_t)(__builtin_clz((uint32_t)(a ^ b)) - 1 - g_delta_bias);
  return (uint8_t)(__builtin_clzll(a ^ b) - 1);
}

static inline unsigned ceil_div_u(unsigned a, unsigned b) {
  return (a + b - 1) / b;
}

/* func_brt.hpp:35-43 */
static inline int log2_ceil_u(unsigned x) {
  const unsigned lower = 32u - (unsigned)__builtin_clz(x) - 1u;
  return (int)(lower + (((unsigned)(1 << lower)) < x));
}

/* process_radix_tree_i (func_brt.hpp:45-138); n = n_brt_nodes */
static void brt_node(int i, int n, const void* codes, int kb, uint8_t* prefix_n,
                     uint8_t* hl, uint8_t* hr, int32_t* lc, int32_t* parent) {
  const uint64_t ci = kget(codes, kb, (size_t)i);
  int d;
  if (i == 0) {
    d = 1;
  } else {
    const int dr = delta(ci, kget(codes, kb, (size_t)(i + 1)), kb);
    const int dl = delta(ci, kget(codes, kb, (size_t)(i - 1)), kb);
    const int diff = dr - dl;
    d = (diff > 0) - (diff < 0);
  }
  int l = 0;
  if (i == 0) {
    l = n - 1; /* the root's range is [0, n_brt-1] in the reference */
  } else {
    const int dmin = delta(ci, kget(codes, kb, (size_t)(i - d)), kb);
    int lmax = 2;
    while ((long)i + (long)lmax * d >= 0 && i + lmax * d <= n &&
           delta(ci, kget(codes, kb, (size_t)(i + lmax * d)), kb) > dmin)
      lmax *= 2;
    const int lcut = (d == -1) ? i : n - i;
    for (int tt = lmax / 2, div = 2; tt >= 1; div *= 2, tt = lmax / div) {
      if (l + tt <= lcut &&
          delta(ci, kget(codes, kb, (size_t)(i + (l + tt) * d)), kb) > dmin)
        l += tt;
    }
  }
  const int j = i + l * d;
  const int dnode = delta(ci, kget(codes, kb, (size_t)j), kb);
  prefix_n[i] = (uint8_t)dnode;
  int s = 0;
  const int maxdiv = 1 << log2_ceil_u((unsigned)l);
  int div = 2;
  const int scut = (d == -1) ? i - 1 : n - i - 1;
  for (unsigned tt = ceil_div_u((unsigned)l, 2); div <= maxdiv;
       div <<= 1, tt = ceil_div_u((unsigned)l, (unsigned)div)) {
    if ((unsigned)s + tt <= (unsigned)scut) {
      const unsigned idx = (unsigned)i + ((unsigned)s + tt) * (unsigned)d;
      if (delta(ci, kget(codes, kb, idx), kb) > dnode) s += (int)tt;
    }
  }
  const int gamma = i + s * d + (d < 0 ? d : 0);
  lc[i] = gamma;
  const int lo = i < j ? i : j;
  const int hi = i < j ? j : i;
  hl[i] = (uint8_t)(lo == gamma);
  hr[i] = (uint8_t)(hi == gamma + 1);
  if (!hl[i]) parent[gamma] = i;
  if (!hr[i]) parent[gamma + 1] = i;
}

int orc_stage4(orc_tree* t) {
  if (!t) return ORC_ERR_ARG;
  if (t->n_unique < 3) return ORC_ERR_DEGENERATE;
  const int n = (int)t->n_brt_nodes;
  /* a fresh AppData's buffers are zero; nodes nobody names as a child keep 0 */
  memset(t->prefix_n, 0, (size_t)n);
  memset(t->has_leaf_left, 0, (size_t)n);
  memset(t->has_leaf_right, 0, (size_t)n);
  memset(t->left_child, 0, 4 * (size_t)n);
  memset(t->parents, 0, 4 * (size_t)n);
  g_delta_bias = (t->options & ORC_OPT_GEOMETRIC_DELTA) && t->key_bits == 32 ? 1 : 0;
  for (int i = 0; i < n; ++i)
    brt_node(i, n, t->keys, t->key_bits, t->prefix_n, t->has_leaf_left,
             t->has_leaf_right, t->left_child, t->parents);
  g_delta_bias = 0;
  return ORC_OK;
}

/* ------------------------------------------------------------------------ */
/* stage 5: edge count (func_edge.hpp:9-16)                                 */
/* ------------------------------------------------------------------------ */

int orc_stage5(orc_tree* t) {
  if (!t || t->n_unique < 3) return ORC_ERR_DEGENERATE;
  const int n = (int)t->n_brt_nodes;
  for (int i = 0; i < n; ++i)
    t->edge_count[i] =
        t->prefix_n[i] / 3 - t->prefix_n[t->parents[i]] / 3;
  return ORC_OK;
}

/* ------------------------------------------------------------------------ */
/* stage 6: global exclusive scan (cu_dispatcher.cu:672-686, count fixed)   */
/* ------------------------------------------------------------------------ */

int orc_stage6(orc_tree* t) {
  if (!t || t->n_unique < 3) return ORC_ERR_DEGENERATE;
  const int n = (int)t->n_brt_nodes;
  int32_t run = 0;
  for (int i = 0; i < n; ++i) {
    t->edge_offset[i] = run;
    run += t->edge_count[i];
  }
  t->n_octree_nodes = (uint32_t)run;
  return ORC_OK;
}

/* ------------------------------------------------------------------------ */
/* stage 7: octree (func_octree.hpp:9-112, root init 07_octree.cu:188-198)  */
/* ------------------------------------------------------------------------ */

static inline void set_child(orc_tree* t, int node, unsigned which, int value) {
  t->children[8 * (size_t)node + which] = value;
  t->child_node_mask[node] |= 1 << which;
}

int orc_stage7(orc_tree* t) {
  if (!t || t->n_unique < 3) return ORC_ERR_DEGENERATE;
  const uint32_t m = t->n_octree_nodes;
  if ((uint64_t)m + 1 > t->capacity) return ORC_ERR_CAPACITY;
  const int kb = t->key_bits;
  const int B = code_bits(kb);
  const int n = (int)t->n_brt_nodes;
  const size_t rows = (size_t)m + 1;
  memset(t->children, 0, 32 * rows);
  memset(t->child_node_mask, 0, 4 * rows);
  memset(t->child_leaf_mask, 0, 4 * rows);

  const int root_level = t->prefix_n[0] / 3;
  {
    const uint64_t rp = kget(t->keys, kb, 0) >> (B - 3 * root_level);
    decode(rp << (B - 3 * root_level), kb, t->min_coord, t->range, t->corner);
    t->cell_size[0] = t->range;
  }

  for (int i = 1; i < n; ++i) {
    const uint64_t code = kget(t->keys, kb, (size_t)i);
    int oct = t->edge_offset[i];
    const int nn = t->edge_count[i];
    const int li = t->prefix_n[i] / 3;
    for (int j = 0; j < nn - 1; ++j) {
      const int level = li - j;
      const uint64_t pre = code >> (B - 3 * level);
      const unsigned which = (unsigned)(pre & 7u);
      const int par = oct + 1;
      set_child(t, par, which, oct);
      decode(pre << (B - 3 * level), kb, t->min_coord, t->range,
             t->corner + 4 * (size_t)oct);
      t->cell_size[oct] = t->range / (float)(1 << (level - root_level));
      oct = par;
    }
    if (nn > 0) {
      int rp = t->parents[i];
      int counter = 0;
      while (t->edge_count[rp] == 0) {
        rp = t->parents[rp];
        ++counter;
        if (counter > 30) break;
      }
      const int oct_parent = t->edge_offset[rp];
      const int top = li - nn + 1;
      const uint64_t pre = code >> (B - 3 * top);
      const unsigned which = (unsigned)(pre & 7u);
      set_child(t, oct_parent, which, oct);
      decode(pre << (B - 3 * top), kb, t->min_coord, t->range,
             t->corner + 4 * (size_t)oct);
      t->cell_size[oct] = t->range / (float)(1 << (top - root_level));
    }
  }
  if (t->options & ORC_OPT_LINK_LEAVES) return orc_link_leaves(t);
  return ORC_OK;
}

/* process_link_leaf (func_octree.hpp:114-163) for node i: each leaf child of
 * i goes into slot (leaf's code at level prefix_n[i]/3 + 1) & 7 of the bottom
 * octree node of the nearest radix-tree ancestor-or-self that owns octree
 * nodes; set_leaf (func_octree.hpp:18-25) clears that slot's leaf-mask bit.
 * Two definitions where the reference's are not total:
 *   - the walk up the radix tree stops after 31 steps, as the left-leaf walk
 *     of the CUDA restatement does (07_octree.cu:136-147); the CPU version's
 *     walk never ends when it reaches the root with no octree nodes (the
 *     root's parent is itself);
 *   - the level shift B - 3 * level is negative for 32-bit keys when
 *     prefix_n[i] = 30 (possible only with the reference's clz - 1); the
 *     shift count is then taken modulo 32, as the x86 shift instruction a
 *     g++ build of the reference executes does. */
static void link_leaf(orc_tree* t, int i) {
  const int kb = t->key_bits;
  const int B = code_bits(kb);
  const int W = kb == 32 ? 32 : 64;
  for (int side = 0; side < 2; ++side) {
    const uint8_t has = side ? t->has_leaf_right[i] : t->has_leaf_left[i];
    if (!has) continue;
    const int leaf = t->left_child[i] + side;
    const int level = t->prefix_n[i] / 3 + 1;
    const int sh = (B - 3 * level) & (W - 1);
    const uint64_t pre = kget(t->keys, kb, (size_t)leaf) >> sh;
    const unsigned which = (unsigned)(pre & 7u);
    int rt = i, counter = 0;
    while (t->edge_count[rt] == 0) {
      rt = t->parents[rt];
      if (++counter > 30) break;
    }
    const int bottom = t->edge_offset[rt];
    t->children[8 * (size_t)bottom + which] = leaf;
    t->child_leaf_mask[bottom] &= ~(1 << which);
  }
}

int orc_link_leaves(orc_tree* t) {
  if (!t || t->n_unique < 3) return ORC_ERR_DEGENERATE;
  const int n = (int)t->n_brt_nodes;
  for (int i = 0; i < n; ++i) link_leaf(t, i);
  return ORC_OK;
}

int orc_run_all(orc_tree* t) {
  int rc;
  if ((rc = orc_stage1(t))) return rc;
  if ((rc = orc_stage2(t))) return rc;
  if ((rc = orc_stage3(t))) return rc;
  if ((rc = orc_stage4(t))) return rc;
  if ((rc = orc_stage5(t))) return rc;
  if ((rc = orc_stage6(t))) return rc;
  return orc_stage7(t);
}
