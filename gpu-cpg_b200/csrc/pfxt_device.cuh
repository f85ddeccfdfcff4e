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
  const int4 a = __ldg(reinterpret_cast<const int4*>(h + i));
  const int4 b = __ldg(reinterpret_cast<const int4*>(h + i) + 1);
  HeapNode n;
  n.vtx = a.x;
  n.left = a.y;
  n.right = a.z;
  n.row = a.w;
  n.head = b.x;
  n.w = __int_as_float(b.y);
  n.dist_head = b.z;
  n.dist_v = b.w;
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

// Candidate (node, 0): the cheapest deviation of the node's vertex, priced
// from the record the node carries.  False if there is no node.
__device__ __forceinline__ bool cand_top(const PfxtGraph& g, int node, float parent_cost,
                                         float& cost) {
  if (node < 0) return false;
  const HeapNode n = load_node(g.hnodes, node);
  cost = child_cost(g.division, parent_cost, n.dist_head, n.w, n.dist_v);
  return true;
}

// Candidate (entry j >= 1 of the sorted row of hn's vertex).  The entry and
// the row's count are requested together (rows are padded, so the entry's
// load stays inside the allocation for any j a search asks); false if j is
// past the count.
__device__ __forceinline__ bool cand_row(const PfxtGraph& g, const HeapNode& hn, int j,
                                         float parent_cost, float& cost) {
  const int cnt = __ldg(g.dev_cnt + hn.vtx);
  const DevSidetrack d = load_dev(g.dev, hn.row + j);
  if (j >= cnt) return false;
  cost = child_cost(g.division, parent_cost, d.dist_head, d.w, hn.dist_v);
  return true;
}

// Head of entry j of the sorted row of hn's vertex: the last edge of the
// path that takes that deviation.
__device__ __forceinline__ int dev_head(const PfxtGraph& g, const HeapNode& hn, int j) {
  return j == 0 ? hn.head : load_dev(g.dev, hn.row + j).head;
}

}  // namespace cpg
