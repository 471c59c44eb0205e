/* Compressed 8-wide BVH: layout, decode helpers and the collapse from the binary BVH.
 *
 * Node (80 B, five float4):
 *   w0 = (p.x, p.y, p.z, hdr)           p = node box lower corner; hdr bytes 0..2 = biased exponents
 *                                       e_x, e_y, e_z of the per-axis scale 2^(e - 127), byte 3 =
 *                                       imask (bit s set: slot s holds an inner child)
 *   w1 = (child_base, tri_base, meta[0..3], meta[4..7])
 *                                       inner children are nodes child_base + rank(s) where rank(s) =
 *                                       popc(imask & ((1 << s) - 1)); a leaf slot's meta byte holds
 *                                       its triangle offset (bits 0..4, from tri_base) and count - 1
 *                                       (bits 5..6), so leaves hold 1..4 triangles
 *   w2 = (qlo_x[0..3], qlo_x[4..7], qlo_y[0..3], qlo_y[4..7])
 *   w3 = (qlo_z[..], qhi_x[..])         w4 = (qhi_y[..], qhi_z[..])
 * Child slot s's box is p + q * scale per axis; empty slots have qlo = 255 > qhi = 0.
 *
 * Slot order: bit k of a slot index means "on the positive side of the node centre along axis k"
 * (children are assigned greedily by their centroid direction), so a ray whose direction-sign bits
 * are `oct` meets slots roughly in increasing order of (slot ^ oct).  Inner children and the leaf
 * triangles of a node are each stored contiguously in slot order.
 */
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace nb {

constexpr int kWideStack = 32;
constexpr int kWideLeafMax = 4;

struct WideBuildResult {
  uint32_t n_nodes;
  uint32_t n_tris;
  int depth;
  double ms;
};

/* Collapses a validated binary BVH (nodes2, leaves of <= 4 triangles, tris2 in leaf order) into
 * the wide layout.  wnodes: room for n_nodes2 + 1 wide nodes (80 B each); tris_out: n_tris records. */
cudaError_t build_wide_bvh(const float4 *nodes2, uint32_t n_nodes2, const float4 *tris2, uint32_t n_tris,
                           float4 *wnodes, float4 *tris_out, cudaStream_t stream, WideBuildResult *res);

}  // namespace nb
