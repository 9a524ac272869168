// Test infrastructure, not product code: the reference's CUDA tree sources,
// included where they lie (the recipe in oracle/Makefile puts the reference
// checkout on the include path), as one translation unit.  Its dispatcher
// launches kernel templates that only 06_prefix_sum.cu defines and
// instantiates (06_prefix_sum.cuh declares them); compiled as separate units
// here, that launch found no device function on the B200 (stage 6,
// "invalid device function").  In one unit every template kernel is defined
// where it is launched.
#include "cuda/01_morton.cu"
#include "cuda/03_unique.cu"
#include "cuda/04_radix_tree.cu"
#include "cuda/05_edge_count.cu"
#include "cuda/06_prefix_sum.cu"
#include "cuda/07_octree.cu"
#include "cuda/im_storage.cu"
#include "cuda/cu_dispatcher.cu"
