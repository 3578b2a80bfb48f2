// pf_city.cuh -- line of sight through a box city (the simulator's cities:
// an n x n grid of cells of side `cell`, at most one axis-aligned box
// building per cell), one ray per thread.  It restates the host DDA of
// gnss_gpu_b200/citysim.py (los_blocked) operation for operation in FP64
// with explicitly rounded multiply / add (no contraction), so the flags are
// the host's bit for bit; the ray directions come from the host.
#pragma once
#include <cuda_runtime.h>
#include <math.h>

namespace pfb {

struct CityDev {
  const unsigned char* occ;  // [n * n], cell (ix, iy) at ix * n + iy
  const double* box;         // [n * n * 4] x0, x1, y0, y1 (local E/N, m)
  const double* height;      // [n * n] m
  int n;
  double cell, hmax;
  int steps;                 // cells a ray may cross before it is declared clear
};

// Is the ray from p toward the unit direction d (d.z > 0) blocked by a
// building?  Walks the cells the ray crosses (ties between an x and a y
// boundary go to y), tests the box of every occupied cell, and stops once
// it is above every roof.
__device__ inline bool city_blocked(const CityDev& c, const double p[3], const double d[3]) {
  const double big = 1e30;
  const double t_end = __ddiv_rn(fmax(__dsub_rn(c.hmax, p[2]), 0.0), d[2]);
  if (!(t_end > 0.0)) return false;
  long long ix = (long long)floor(__ddiv_rn(p[0], c.cell));
  long long iy = (long long)floor(__ddiv_rn(p[1], c.cell));
  const int sx = d[0] > 0.0 ? 1 : -1, sy = d[1] > 0.0 ? 1 : -1;
  const bool fx = fabs(d[0]) > 1e-12, fy = fabs(d[1]) > 1e-12;
  const double inv_dx = fx ? __drcp_rn(d[0]) : big;
  const double inv_dy = fy ? __drcp_rn(d[1]) : big;
  double t_max_x = fx ? __dmul_rn(__dsub_rn(__dmul_rn((double)(ix + (sx > 0)), c.cell), p[0]), inv_dx) : big;
  double t_max_y = fy ? __dmul_rn(__dsub_rn(__dmul_rn((double)(iy + (sy > 0)), c.cell), p[1]), inv_dy) : big;
  const double t_dx = fx ? __dmul_rn(c.cell, fabs(inv_dx)) : big;
  const double t_dy = fy ? __dmul_rn(c.cell, fabs(inv_dy)) : big;
  for (int it = 0; it < c.steps; ++it) {
    if (ix >= 0 && ix < c.n && iy >= 0 && iy < c.n) {
      const long long k = ix * c.n + iy;
      if (c.occ[k]) {
        const double* b = c.box + 4 * k;
        const double h = c.height[k];
        double lo_x, hi_x, lo_y, hi_y;
        if (fx) {
          const double t0 = __dmul_rn(__dsub_rn(b[0], p[0]), inv_dx), t1 = __dmul_rn(__dsub_rn(b[1], p[0]), inv_dx);
          lo_x = fmin(t0, t1);
          hi_x = fmax(t0, t1);
        } else {  // parallel to the x slab: inside it or never
          const bool in = p[0] >= b[0] && p[0] <= b[1];
          lo_x = in ? -big : big;
          hi_x = in ? big : -big;
        }
        if (fy) {
          const double t0 = __dmul_rn(__dsub_rn(b[2], p[1]), inv_dy), t1 = __dmul_rn(__dsub_rn(b[3], p[1]), inv_dy);
          lo_y = fmin(t0, t1);
          hi_y = fmax(t0, t1);
        } else {
          const bool in = p[1] >= b[2] && p[1] <= b[3];
          lo_y = in ? -big : big;
          hi_y = in ? big : -big;
        }
        const double lo_z = __ddiv_rn(__dsub_rn(0.0, p[2]), d[2]), hi_z = __ddiv_rn(__dsub_rn(h, p[2]), d[2]);
        const double t_in = fmax(fmax(lo_x, lo_y), fmax(lo_z, 0.0));
        const double t_out = fmin(fmin(hi_x, hi_y), hi_z);
        if (t_in <= t_out) return true;
      }
    }
    const bool go_x = t_max_x < t_max_y;
    const double t_cur = go_x ? t_max_x : t_max_y;
    if (go_x) {
      ix += sx;
      t_max_x = __dadd_rn(t_max_x, t_dx);
    } else {
      iy += sy;
      t_max_y = __dadd_rn(t_max_y, t_dy);
    }
    if (!(t_cur <= t_end)) return false;
  }
  return false;
}

__global__ void k_city_los(CityDev c, const double* __restrict__ p, const double* __restrict__ d, int n_ray,
                           unsigned char* __restrict__ blocked) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_ray) return;
  const double pp[3] = {p[3 * i], p[3 * i + 1], p[3 * i + 2]};
  const double dd[3] = {d[3 * i], d[3 * i + 1], d[3 * i + 2]};
  blocked[i] = city_blocked(c, pp, dd) ? 1 : 0;
}

}  // namespace pfb
