// pf_bvh.cuh -- building-aware likelihood of the 3D filters
// (src/particle_filter/weight_3d.cu, weight_3d_bvh.cu of the reference):
// a bounding-volume hierarchy over a triangle mesh, built on the host, and
// per-particle, per-satellite shadow rays traced through it on the device.
//
// Mesh frame.  The mesh is stored in FP32 in a local East/North/Up frame
// about an FP64 origin (the mean vertex): ray origins (particles) and
// directions (to the satellites) are formed in FP64 and rounded once, so
// the FP32 traversal keeps sub-millimetre precision across a city.
//
// Layout (device):
//   nodes  4 x float4 per inner node, the boxes of its two children:
//          (left bmin, left ref) (left bmax, right ref) (right bmin, -)
//          (right bmax, -), refs bit-cast ints: >= 0 an inner node, < 0 a
//          leaf ~(first triangle << 3 | count - 1).  Node 0 is the root.
//   tris   3 x float4 per triangle: v0, e1 = v1 - v0, e2 = v2 - v0.
// The builder splits by the binned surface-area heuristic down to depth 32
// and at the median centroid below that (leaves of at most kBvhLeaf
// triangles), so the depth stays below 32 + log2(n / kBvhLeaf) + 2 and the
// traversal stack of kBvhStack entries (at most depth + 1 are live) cannot
// overflow for any mesh the 32-bit indices can hold.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

namespace pfb {

constexpr int kBvhLeaf = 4;
constexpr int kBvhStack = 64;  // >= depth + 1: surface-area splits to depth 32, median below

// ---------------------------------------------------------------- host
struct HostBvh {
  std::vector<float> nodes;  // 8 floats per node
  std::vector<float> tris;   // 12 floats per triangle
  int n_nodes = 0;
};

#ifndef PF_BVH_SAH
#define PF_BVH_SAH 1
#endif
constexpr int kSahBins = 16;
constexpr int kBvhSahDepth = 32;  // deeper subtrees split at the median (keeps the depth bounded)

inline float half_area(const float* mn, const float* mx) {
  const float dx = mx[0] - mn[0], dy = mx[1] - mn[1], dz = mx[2] - mn[2];
  return dx * dy + dy * dz + dz * dx;
}

// Binned surface-area split of idx[b, e): the axis and bin boundary with
// the least sum over children of (triangles x box surface).  Reorders
// idx[b, e) around the boundary and returns it in mid; false when every
// centroid falls into one bin (the caller splits at the median).
inline bool sah_split(std::vector<int>& idx, const std::vector<float>& cen, const std::vector<float>& lo,
                      const std::vector<float>& hi, int b, int e, const float* cmn, const float* cmx, int& mid) {
  float best = INFINITY;
  int best_ax = -1, best_k = 0;
  for (int ax = 0; ax < 3; ++ax) {
    const float ext = cmx[ax] - cmn[ax];
    if (!(ext > 0.f)) continue;
    const float scale = kSahBins / ext;
    int cnt[kSahBins] = {0};
    float bmn[kSahBins][3], bmx[kSahBins][3];
    for (int k = 0; k < kSahBins; ++k)
      for (int a = 0; a < 3; ++a) {
        bmn[k][a] = INFINITY;
        bmx[k][a] = -INFINITY;
      }
    for (int q = b; q < e; ++q) {
      const int i = idx[q];
      const int k = std::min(kSahBins - 1, (int)((cen[3 * (size_t)i + ax] - cmn[ax]) * scale));
      ++cnt[k];
      for (int a = 0; a < 3; ++a) {
        bmn[k][a] = std::min(bmn[k][a], lo[3 * (size_t)i + a]);
        bmx[k][a] = std::max(bmx[k][a], hi[3 * (size_t)i + a]);
      }
    }
    // sweep: right-side prefix areas, then left to right
    float rarea[kSahBins];
    int rcnt[kSahBins];
    float rmn[3] = {INFINITY, INFINITY, INFINITY}, rmx[3] = {-INFINITY, -INFINITY, -INFINITY};
    int rc = 0;
    for (int k = kSahBins - 1; k > 0; --k) {
      rc += cnt[k];
      for (int a = 0; a < 3; ++a) {
        rmn[a] = std::min(rmn[a], bmn[k][a]);
        rmx[a] = std::max(rmx[a], bmx[k][a]);
      }
      rcnt[k] = rc;
      rarea[k] = rc ? half_area(rmn, rmx) : 0.f;
    }
    float lmn[3] = {INFINITY, INFINITY, INFINITY}, lmx[3] = {-INFINITY, -INFINITY, -INFINITY};
    int lc = 0;
    for (int k = 0; k < kSahBins - 1; ++k) {
      lc += cnt[k];
      for (int a = 0; a < 3; ++a) {
        lmn[a] = std::min(lmn[a], bmn[k][a]);
        lmx[a] = std::max(lmx[a], bmx[k][a]);
      }
      if (lc == 0 || rcnt[k + 1] == 0) continue;
      const float c = lc * half_area(lmn, lmx) + rcnt[k + 1] * rarea[k + 1];
      if (c < best) {
        best = c;
        best_ax = ax;
        best_k = k;
      }
    }
  }
  if (best_ax < 0) return false;
  const float scale = kSahBins / (cmx[best_ax] - cmn[best_ax]);
  auto it = std::partition(idx.begin() + b, idx.begin() + e, [&](int i) {
    return std::min(kSahBins - 1, (int)((cen[3 * (size_t)i + best_ax] - cmn[best_ax]) * scale)) <= best_k;
  });
  mid = (int)(it - idx.begin());
  return mid > b && mid < e;
}

// tris_m: n x 9 doubles already in the mesh frame.
inline void build_bvh(const std::vector<double>& tris_m, int n, HostBvh& out) {
  std::vector<int> idx(n);
  std::vector<float> cen((size_t)n * 3), lo((size_t)n * 3), hi((size_t)n * 3);
  for (int i = 0; i < n; ++i) {
    idx[i] = i;
    for (int a = 0; a < 3; ++a) {
      const double v0 = tris_m[9 * (size_t)i + a], v1 = tris_m[9 * (size_t)i + 3 + a], v2 = tris_m[9 * (size_t)i + 6 + a];
      const double mn = std::min(v0, std::min(v1, v2)), mx = std::max(v0, std::max(v1, v2));
      // boxes widened by one float ulp each way so the FP32 box holds the triangle
      lo[3 * (size_t)i + a] = std::nextafter((float)mn, -INFINITY);
      hi[3 * (size_t)i + a] = std::nextafter((float)mx, INFINITY);
      cen[3 * (size_t)i + a] = (float)((v0 + v1 + v2) / 3.0);
    }
  }
  struct Item { int node, b, e, depth; };
  std::vector<float>& nodes = out.nodes;
  nodes.clear();
  auto new_node = [&]() {
    nodes.resize(nodes.size() + 8, 0.f);
    return (int)(nodes.size() / 8) - 1;
  };
  std::vector<Item> stack;
  if (n > 0) stack.push_back({new_node(), 0, n, 0});
  while (!stack.empty()) {
    const Item it = stack.back();
    stack.pop_back();
    float bmn[3] = {INFINITY, INFINITY, INFINITY}, bmx[3] = {-INFINITY, -INFINITY, -INFINITY};
    float cmn[3] = {INFINITY, INFINITY, INFINITY}, cmx[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int k = it.b; k < it.e; ++k) {
      const int i = idx[k];
      for (int a = 0; a < 3; ++a) {
        bmn[a] = std::min(bmn[a], lo[3 * (size_t)i + a]);
        bmx[a] = std::max(bmx[a], hi[3 * (size_t)i + a]);
        cmn[a] = std::min(cmn[a], cen[3 * (size_t)i + a]);
        cmx[a] = std::max(cmx[a], cen[3 * (size_t)i + a]);
      }
    }
    float* nd = &nodes[8 * (size_t)it.node];
    for (int a = 0; a < 3; ++a) {
      nd[a] = bmn[a];
      nd[4 + a] = bmx[a];
    }
    int ia, ib;
    if (it.e - it.b <= kBvhLeaf) {
      ia = -(it.b + 1);
      ib = it.e - it.b;
    } else {
      int ax = 0;
      for (int a = 1; a < 3; ++a)
        if (cmx[a] - cmn[a] > cmx[ax] - cmn[ax]) ax = a;
      int mid = (it.b + it.e) / 2;
      bool done = false;
      if (PF_BVH_SAH && it.depth < kBvhSahDepth) done = sah_split(idx, cen, lo, hi, it.b, it.e, cmn, cmx, mid);
      if (!done)
        std::nth_element(idx.begin() + it.b, idx.begin() + mid, idx.begin() + it.e, [&](int p, int q) {
          const float cp = cen[3 * (size_t)p + ax], cq = cen[3 * (size_t)q + ax];
          return cp < cq || (cp == cq && p < q);
        });
      const int l = new_node(), r = new_node();
      nd = &nodes[8 * (size_t)it.node];  // the vector may have moved
      ia = l;
      ib = r;
      stack.push_back({r, mid, it.e, it.depth + 1});
      stack.push_back({l, it.b, mid, it.depth + 1});
    }
    memcpy(&nd[3], &ia, 4);
    memcpy(&nd[7], &ib, 4);
  }
  // Child-box layout: each inner node of the binary tree becomes one node
  // holding its two children's boxes, so a traversal tests both children
  // at the parent, visits the nearer and never pops a missed node.
  const int nb = (int)(nodes.size() / 8);
  auto ia_of = [&](int k) { int v; memcpy(&v, &nodes[8 * (size_t)k + 3], 4); return v; };
  auto ib_of = [&](int k) { int v; memcpy(&v, &nodes[8 * (size_t)k + 7], 4); return v; };
  std::vector<int> inner_id(nb, -1);
  int n_inner = 0;
  for (int k = 0; k < nb; ++k)
    if (ia_of(k) >= 0) inner_id[k] = n_inner++;
  auto child_ref = [&](int k) {
    const int a = ia_of(k);
    return a >= 0 ? inner_id[k] : ~(((-a - 1) << 3) | (ib_of(k) - 1));
  };
  // child k's box and reference into the left (side 0) or right (side 1)
  // slots of a node: boxes at [0..2]/[4..6] and [8..10]/[12..14], references
  // at [3] and [7]
  auto put_child = [&](float* dst, int side, int k) {
    const int ref = child_ref(k);
    for (int a = 0; a < 3; ++a) {
      dst[8 * side + a] = nodes[8 * (size_t)k + a];
      dst[8 * side + 4 + a] = nodes[8 * (size_t)k + 4 + a];
    }
    memcpy(&dst[side == 0 ? 3 : 7], &ref, 4);
  };
  std::vector<float> wide;
  if (nb > 0) {
    wide.assign((size_t)std::max(n_inner, 1) * 16, 0.f);
    if (n_inner == 0) {  // the whole mesh is one leaf: a root with it on the left and, on the right,
      n_inner = 1;       // a point box far outside any ray's reach
      put_child(&wide[0], 0, 0);
      for (int a = 0; a < 3; ++a) wide[8 + a] = wide[12 + a] = 1e30f;
      const int none = ~0;
      memcpy(&wide[7], &none, 4);
    } else {
      for (int k = 0; k < nb; ++k) {
        if (inner_id[k] < 0) continue;
        float* dst = &wide[16 * (size_t)inner_id[k]];
        put_child(dst, 0, ia_of(k));
        put_child(dst, 1, ib_of(k));
      }
    }
  }
  nodes.swap(wide);
  out.n_nodes = nb > 0 ? n_inner : 0;
  out.tris.assign((size_t)n * 12, 0.f);
  for (int k = 0; k < n; ++k) {
    const int i = idx[k];
    const double* t = &tris_m[9 * (size_t)i];
    float* o = &out.tris[12 * (size_t)k];
    for (int a = 0; a < 3; ++a) {
      o[a] = (float)t[a];
      o[4 + a] = (float)(t[3 + a] - t[a]);
      o[8 + a] = (float)(t[6 + a] - t[a]);
    }
  }
}

// -------------------------------------------------------------- device
struct MeshDev {
  const float4* nodes;
  const float4* tris;
  int n_nodes, n_tris;
  double origin[3];
  double rot[9];
};

// Moller-Trumbore: does the segment origin + t dir, t in (1e-6, tmax), hit
// the triangle (v0, e1, e2)?
__device__ __forceinline__ bool tri_hit(const float3 o, const float3 d, const float4 v0, const float4 e1,
                                        const float4 e2, float tmax) {
  const float hx = d.y * e2.z - d.z * e2.y, hy = d.z * e2.x - d.x * e2.z, hz = d.x * e2.y - d.y * e2.x;
  const float a = e1.x * hx + e1.y * hy + e1.z * hz;
  if (fabsf(a) < 1e-12f) return false;
  const float f = 1.0f / a;
  const float sx = o.x - v0.x, sy = o.y - v0.y, sz = o.z - v0.z;
  const float u = f * (sx * hx + sy * hy + sz * hz);
  if (u < 0.f || u > 1.f) return false;
  const float qx = sy * e1.z - sz * e1.y, qy = sz * e1.x - sx * e1.z, qz = sx * e1.y - sy * e1.x;
  const float v = f * (d.x * qx + d.y * qy + d.z * qz);
  if (v < 0.f || u + v > 1.f) return false;
  const float t = f * (e2.x * qx + e2.y * qy + e2.z * qz);
  return t > 1e-6f && t < tmax;
}

__device__ __forceinline__ bool slab(const float4 mn, const float4 mx, const float3 o, const float3 inv, float tmax,
                                     float& tin) {
  float a = (mn.x - o.x) * inv.x, b = (mx.x - o.x) * inv.x;
  float t0 = fmaxf(0.f, fminf(a, b)), t1 = fminf(tmax, fmaxf(a, b));
  a = (mn.y - o.y) * inv.y;
  b = (mx.y - o.y) * inv.y;
  t0 = fmaxf(t0, fminf(a, b));
  t1 = fminf(t1, fmaxf(a, b));
  a = (mn.z - o.z) * inv.z;
  b = (mx.z - o.z) * inv.z;
  t0 = fmaxf(t0, fminf(a, b));
  t1 = fminf(t1, fmaxf(a, b));
  tin = t0;
  return t0 <= t1;
}

// Triangles of leaf reference `ref` (~(start << 3 | count - 1)).
__device__ __forceinline__ bool leaf_hit(const MeshDev& m, int ref, const float3 o, const float3 d, float tmax) {
  const int code = ~ref, s0 = code >> 3, c = (code & 7) + 1;
  if (s0 + c > m.n_tris) return false;  // malformed reference
  for (int k = 0; k < c; ++k) {
    const float4* t = m.tris + 3 * (s0 + k);
    if (tri_hit(o, d, __ldg(t), __ldg(t + 1), __ldg(t + 2), tmax)) return true;
  }
  return false;
}

// Is any triangle between o and o + tmax d (d unit)?  Any-hit traversal of
// the child-box layout: both children tested at the parent, leaves
// intersected at once, the nearer inner child visited first, the other
// stacked.  A full stack (impossible with the builder's depth bound) would
// drop the farther child and could report a blocked ray clear.
__device__ __forceinline__ bool bvh_blocked(const MeshDev& m, const float3 o, const float3 d, float tmax) {
  if (m.n_nodes <= 0) return false;
  const float3 inv = make_float3(1.0f / d.x, 1.0f / d.y, 1.0f / d.z);
  int stack[kBvhStack];
  int sp = 0, node = 0;
  // a tree visits each node at most once: the bound only guards against a
  // malformed mesh description (which would otherwise loop)
  for (int visits = 0; visits <= m.n_nodes; ++visits) {
    if ((unsigned)node >= (unsigned)m.n_nodes) return false;
    const float4* nd = m.nodes + 4 * node;
    const float4 l0 = __ldg(nd), l1 = __ldg(nd + 1), r0 = __ldg(nd + 2), r1 = __ldg(nd + 3);
    float tl, tr;
    bool hl = slab(l0, l1, o, inv, tmax, tl), hr = slab(r0, r1, o, inv, tmax, tr);
    const int cl = __float_as_int(l0.w), cr = __float_as_int(l1.w);
    if (hl && cl < 0) {
      if (leaf_hit(m, cl, o, d, tmax)) return true;
      hl = false;
    }
    if (hr && cr < 0) {
      if (leaf_hit(m, cr, o, d, tmax)) return true;
      hr = false;
    }
    if (hl && hr) {
      const bool lf = tl <= tr;
      if (sp < kBvhStack) stack[sp++] = lf ? cr : cl;
      node = lf ? cl : cr;
    } else if (hl) {
      node = cl;
    } else if (hr) {
      node = cr;
    } else {
      if (sp == 0) return false;
      node = stack[--sp];
    }
  }
  return false;
}

// Mesh-frame origin of an ECEF point (FP64 in, rounded once).
__device__ __forceinline__ float3 mesh_origin(const MeshDev& m, const double p[3]) {
  const double q[3] = {p[0] - m.origin[0], p[1] - m.origin[1], p[2] - m.origin[2]};
  return make_float3((float)(m.rot[0] * q[0] + m.rot[1] * q[1] + m.rot[2] * q[2]),
                     (float)(m.rot[3] * q[0] + m.rot[4] * q[1] + m.rot[5] * q[2]),
                     (float)(m.rot[6] * q[0] + m.rot[7] * q[1] + m.rot[8] * q[2]));
}

// Mesh-frame unit direction of the ECEF vector v of length L (the FP64
// unit vector rounded to FP32, then rotated in FP32: 1e-7 rad).
__device__ __forceinline__ float3 mesh_dir(const MeshDev& m, const double v[3], double L) {
  const double il = 1.0 / L;
  const float ux = (float)(v[0] * il), uy = (float)(v[1] * il), uz = (float)(v[2] * il);
  return make_float3((float)m.rot[0] * ux + (float)m.rot[1] * uy + (float)m.rot[2] * uz,
                     (float)m.rot[3] * ux + (float)m.rot[4] * uy + (float)m.rot[5] * uz,
                     (float)m.rot[6] * ux + (float)m.rot[7] * uy + (float)m.rot[8] * uz);
}

struct Sat3d {
  double sat[3];
  double pr;
  double w;
};
constexpr int kMax3dSats = 64;

struct Weight3dArgs {
  int n_sat;
  int accumulate;
  double inv_s2_los, inv_s2_nlos, nlos_bias, p_blocked, p_clear;
};

__device__ __forceinline__ double mix_loglik(double los, double nlos, double p) {
  if (p <= 0.0) return los;
  if (p >= 1.0) return nlos;
  const double a = log(1.0 - p) + los, b = log(p) + nlos;
  const double mx = a > b ? a : b;
  return mx + log(exp(a - mx) + exp(b - mx));
}

}  // namespace pfb
