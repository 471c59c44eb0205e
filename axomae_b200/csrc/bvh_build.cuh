/* On-device binned-SAH BVH build (declarations).  See bvh_build.cu. */
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace nb {

struct BvhBuildParams {
  int max_leaf;     /* preferred maximum leaf size (SAH may stop earlier); hard cap 16 */
  int hard_leaf;    /* nodes with more primitives are always split (median when SAH finds no plane) */
  int bins;         /* SAH bins per axis (<= 32) */
  float cost_trav;  /* SAH cost of one inner-node visit relative to one triangle test */
  uint32_t small_task; /* nodes of at most this many primitives are built whole by one CTA (0: default) */
};

struct BvhBuildResult {
  uint32_t n_nodes;
  uint32_t n_leaves;
  int max_depth;
  double ms;
};

/* Builds a binary BVH over n primitive boxes (lo/hi: world-space, float4 with w unused).
 * nodes: room for max(2n, 2) nodes (4 float4 each, layout in device_scene.cuh).
 * order: receives, for every leaf slot, the index (into lo/hi) of the primitive stored there.
 * Returns a CUDA error code (cudaSuccess on success). */
cudaError_t build_bvh(const float4 *lo, const float4 *hi, uint32_t n, const BvhBuildParams &p, float4 *nodes,
                      uint32_t *order, cudaStream_t stream, BvhBuildResult *res);

/* Renumbers the n nodes of a built binary BVH in depth-first preorder (root stays 0, every child
 * after its parent, a subtree contiguous).  Scratch comes from the stream's memory pool. */
cudaError_t reorder_depth_first(float4 *nodes, uint32_t n, cudaStream_t stream);

}  // namespace nb
