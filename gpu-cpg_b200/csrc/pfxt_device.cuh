// Device pieces of the prefix-tree enumeration shared by the closure kernel
// (pfxt.cu) and the persistent query engine (engine.cu).  Both translation
// units are compiled with --use_fast_math like the reference, so
// child_cost_reference evaluates the reference's expression
// (gpucpg/gpucpg.cu:3271-3276) with the reference's device quotient.
#pragma once

#include "device_common.cuh"

namespace cpg {

__device__ __forceinline__ float child_cost_reference(float slack, int dn,
                                                      float wgt, int dv) {
  auto dist_neighbor = (float)dn / kScaleUp;
  auto dist_v = (float)dv / kScaleUp;
  auto new_path_slack = slack + dist_neighbor + wgt - dist_v;
  return new_path_slack;
}

__device__ __forceinline__ float child_cost_ieee(float slack, int dn, float wgt,
                                                 int dv) {
  const float a = __fadd_rn(slack, __fdiv_rn(static_cast<float>(dn), 10000.0f));
  const float b = __fadd_rn(a, wgt);
  return __fsub_rn(b, __fdiv_rn(static_cast<float>(dv), 10000.0f));
}

__device__ __forceinline__ float child_cost(int division, float slack, int dn,
                                            float wgt, int dv) {
  return division == CPG_DIV_IEEE ? child_cost_ieee(slack, dn, wgt, dv)
                                  : child_cost_reference(slack, dn, wgt, dv);
}

__device__ __forceinline__ HeapNode load_node(const HeapNode* h, int i) {
  const int4 r = __ldg(reinterpret_cast<const int4*>(h + i));
  HeapNode n;
  n.vtx = r.x;
  n.left = r.y;
  n.right = r.z;
  n.key = __int_as_float(r.w);
  return n;
}

__device__ __forceinline__ DevSidetrack load_dev(const DevSidetrack* d, int i) {
  const int4 r = __ldg(reinterpret_cast<const int4*>(d + i));
  DevSidetrack s;
  s.head = r.x;
  s.w = __int_as_float(r.y);
  s.dist_head = r.z;
  s.key = __int_as_float(r.w);
  return s;
}

// Candidate (parent path, heap node, index j): fills its cost.  Returns false
// if the candidate does not exist.
__device__ __forceinline__ bool make_candidate(const PfxtGraph& g, int node,
                                               int j, float parent_cost,
                                               float& cost) {
  if (node < 0) return false;
  const HeapNode hn = load_node(g.hnodes, node);
  const int v = hn.vtx;
  if (j >= __ldg(g.dev_cnt + v)) return false;
  const DevSidetrack d = load_dev(g.dev, __ldg(g.adjp + v) + j);
  cost = child_cost(g.division, parent_cost, d.dist_head, d.w, __ldg(g.dist + v));
  return true;
}


}  // namespace cpg
