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
//   nodes  2 x float4 per node: (bmin, a) (bmax, b) with a, b bit-cast ints;
//          a >= 0: inner node with children a and b; a < 0: leaf holding
//          triangles [-a - 1, -a - 1 + b).
//   tris   3 x float4 per triangle: v0, e1 = v1 - v0, e2 = v2 - v0.
// The builder splits at the median centroid along the widest centroid
// extent (leaves of at most kBvhLeaf triangles), so the depth stays below
// log2(n / kBvhLeaf) + 2 and the traversal stack of kBvhStack entries
// (at most depth + 1 are live) cannot overflow for any mesh the 32-bit
// indices can hold.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

namespace pfb {

constexpr int kBvhLeaf = 4;
constexpr int kBvhStack = 32;  // >= depth + 1 for any 32-bit triangle count

// ---------------------------------------------------------------- host
struct HostBvh {
  std::vector<float> nodes;  // 8 floats per node
  std::vector<float> tris;   // 12 floats per triangle
  int n_nodes = 0;
};

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
  struct Item { int node, b, e; };
  std::vector<float>& nodes = out.nodes;
  nodes.clear();
  auto new_node = [&]() {
    nodes.resize(nodes.size() + 8, 0.f);
    return (int)(nodes.size() / 8) - 1;
  };
  std::vector<Item> stack;
  if (n > 0) stack.push_back({new_node(), 0, n});
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
      const int mid = (it.b + it.e) / 2;
      std::nth_element(idx.begin() + it.b, idx.begin() + mid, idx.begin() + it.e, [&](int p, int q) {
        const float cp = cen[3 * (size_t)p + ax], cq = cen[3 * (size_t)q + ax];
        return cp < cq || (cp == cq && p < q);
      });
      const int l = new_node(), r = new_node();
      nd = &nodes[8 * (size_t)it.node];  // the vector may have moved
      ia = l;
      ib = r;
      stack.push_back({r, mid, it.e});
      stack.push_back({l, it.b, mid});
    }
    memcpy(&nd[3], &ia, 4);
    memcpy(&nd[7], &ib, 4);
  }
  out.n_nodes = (int)(nodes.size() / 8);
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

// Is any triangle between o and o + tmax d (d unit)?  Any-hit traversal,
// left child first; a full stack (impossible with the builder's depth
// bound) would end the walk early and report the ray clear.
__device__ __forceinline__ bool bvh_blocked(const MeshDev& m, const float3 o, const float3 d, float tmax) {
  if (m.n_nodes <= 0) return false;
  const float3 inv = make_float3(1.0f / d.x, 1.0f / d.y, 1.0f / d.z);
  int stack[kBvhStack];
  int sp = 0;
  stack[sp++] = 0;
  while (sp > 0) {
    const int ni = stack[--sp];
    const float4 n0 = __ldg(m.nodes + 2 * ni), n1 = __ldg(m.nodes + 2 * ni + 1);
    float t0 = 0.f, t1 = tmax;
    {
      float a = (n0.x - o.x) * inv.x, b = (n1.x - o.x) * inv.x;
      t0 = fmaxf(t0, fminf(a, b));
      t1 = fminf(t1, fmaxf(a, b));
      a = (n0.y - o.y) * inv.y;
      b = (n1.y - o.y) * inv.y;
      t0 = fmaxf(t0, fminf(a, b));
      t1 = fminf(t1, fmaxf(a, b));
      a = (n0.z - o.z) * inv.z;
      b = (n1.z - o.z) * inv.z;
      t0 = fmaxf(t0, fminf(a, b));
      t1 = fminf(t1, fmaxf(a, b));
    }
    if (t0 > t1) continue;
    const int ia = __float_as_int(n0.w), ib = __float_as_int(n1.w);
    if (ia < 0) {
      const int s = -ia - 1;
      for (int k = 0; k < ib; ++k) {
        const float4* t = m.tris + 3 * (s + k);
        if (tri_hit(o, d, __ldg(t), __ldg(t + 1), __ldg(t + 2), tmax)) return true;
      }
    } else if (sp + 2 <= kBvhStack) {
      stack[sp++] = ib;
      stack[sp++] = ia;
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
