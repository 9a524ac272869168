/* Test infrastructure, not product code.
 *
 * CPU restatement of the reference tree pipeline (ucsc-redwood/redwood-comp,
 * apps/tree): Morton encode -> sort -> unique -> Karras binary radix tree ->
 * edge count -> prefix sum -> octree, with the canonical dataflow:
 *   - sort output lands in keys_alt, unique output in keys
 *     (apps/tree/app_data.hpp:139-157);
 *   - stage 6 is a global exclusive scan and n_octree_nodes = off[b-1]+ec[b-1];
 *   - stage 7 runs process_oct_node for i = 1 .. n_brt-1 in ascending order on
 *     zeroed octree rows after the root initialisation of
 *     apps/tree/cuda/07_octree.cu:188-198.
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it,
 * and only as the checker.  Every function cites the reference code it
 * restates.  32-bit keys follow the reference exactly (30-bit codes, 10 bits per
 * axis); 64-bit keys (63-bit codes, 21 bits per axis) are the same functions at
 * the wider width, which the reference does not have.
 */
#ifndef RW_TREE_ORACLE_H
#define RW_TREE_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  ORC_OK = 0,
  ORC_ERR_ARG = 1,        /* bad sizes / pointers */
  ORC_ERR_DEGENERATE = 2, /* fewer than 3 distinct keys: no tree */
  ORC_ERR_CAPACITY = 3    /* n_octree_nodes + 1 > octree capacity */
};

typedef struct orc_tree {
  uint32_t n_input;
  uint32_t capacity; /* octree rows: floor(n_input * 0.6f), app_data.hpp:13,28 */
  int key_bits;      /* 32 or 64 */
  float min_coord;
  float range;
  const float* points; /* [4 n] x y z w */
  void* keys;          /* [n] u32 or u64: Morton after stage 1, unique after 3 */
  void* keys_alt;      /* [n] sorted keys after stage 2 */
  uint8_t* prefix_n;   /* [n] */
  uint8_t* has_leaf_left;
  uint8_t* has_leaf_right;
  int32_t* left_child;
  int32_t* parents;
  int32_t* edge_count;  /* [n] */
  int32_t* edge_offset; /* [n] */
  int32_t* children;    /* [8 capacity] */
  float* corner;        /* [4 capacity] */
  float* cell_size;     /* [capacity] */
  int32_t* child_node_mask;
  int32_t* child_leaf_mask;
  uint32_t n_unique;
  uint32_t n_brt_nodes;
  uint32_t n_octree_nodes;
  int options; /* ORC_OPT_* bits; 0 is the reference's own behaviour */
} orc_tree;

/* Options outside the bit-exact contract with the reference (both change its
 * outputs on purpose):
 *   ORC_OPT_GEOMETRIC_DELTA - delta = clz(a ^ b) - 2 for 32-bit keys, the true
 *     common-prefix length of 30-bit codes (the reference's clz - 1 of
 *     func_brt.hpp:27-33 counts one of the two always-zero top bits).  64-bit
 *     codes are 63 bits wide, so their clz - 1 is already the true length and
 *     the option changes nothing for them.
 *   ORC_OPT_LINK_LEAVES - after stage 7, process_link_leaf
 *     (func_octree.hpp:114-163) for every radix-tree node in ascending order,
 *     the launch the reference leaves commented out (cu_dispatcher.cu:738-749). */
enum { ORC_OPT_GEOMETRIC_DELTA = 1, ORC_OPT_LINK_LEAVES = 2 };

uint32_t orc_capacity(uint32_t n_input);
int orc_stage1(orc_tree* t);
int orc_stage2(orc_tree* t);
int orc_stage3(orc_tree* t);
int orc_stage4(orc_tree* t);
int orc_stage5(orc_tree* t);
int orc_stage6(orc_tree* t);
int orc_stage7(orc_tree* t);
int orc_run_all(orc_tree* t);
/* The leaf links alone (stage 7 calls it under ORC_OPT_LINK_LEAVES). */
int orc_link_leaves(orc_tree* t);

/* Single stages on raw arrays, for tests of one kernel at a time. */
void orc_morton(const float* points, void* keys, uint32_t n, int key_bits,
                float min_coord, float range);
void orc_sort(void* keys, uint32_t n, int key_bits);
uint64_t orc_fnv1a64(const void* data, size_t bytes);

/* Seeded clouds identical to the library's rw_tree_generate_points for its
 * counter-based kinds (points_oracle.c); kind 1 uniform, 2 Gaussian mixture. */
enum { ORC_GEN_UNIFORM = 1, ORC_GEN_GAUSSIAN_MIXTURE = 2 };
int orc_generate_points(float* out, uint64_t n, int kind, uint64_t seed, float min_coord,
                        float range, int n_components, float sigma_lo, float sigma_hi);

#ifdef __cplusplus
}
#endif

#endif
