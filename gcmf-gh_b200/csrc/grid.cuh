// grid.cuh -- uniform-grid MBR candidates: the join's MBR filter as a grid probe.
//
// The reference finds MBR candidates with a sort-sweep on x (GPU_MBR.h:339-539): each
// polygon scans the other layer's x1-sorted starts between its own x endpoints and checks
// y.  On values that accepts (b, o) iff x1b <= x1o < x2b or x1o < x1b <= x2o, with closed
// overlap in y.  Here one layer's valid MBRs are listed in the cells of a uniform grid
// that their boxes cover, and each polygon of the other layer tests the entries of the
// cells its own box covers with that predicate.  Every accepted pair's boxes overlap
// (closed), so the lower-left corner of the overlap lies in both boxes and its cell is
// probed by the polygon and lists the entry; the pair is taken only in that cell, so it
// is found exactly once.  cell_of is monotone in the coordinate, which makes the corner's
// cell one of the probed ones.  The candidates are the sweep's, whatever the grid.
#pragma once
#include <cmath>
#include <cstdint>
#include <cuda_runtime.h>
#include "common.cuh"

namespace gcmfgh {
namespace {

struct GridIndex {
  double x0, y0, cw, ch;
  int gx, gy;
  const int64_t* cellOff;     // ncells + 1 entries
  const int32_t* cellList;    // polygon ids, cell by cell
};

__device__ __forceinline__ int cell_of(double v, double c0, double cs, int g) {
  double t = (v - c0) / cs;
  if (!(t > 0)) return 0;
  if (t >= (double)g) return g - 1;
  return (int)t;
}

// Grid over an extent: cells about the mean MBR size, at most kGridMaxAxis per axis.
constexpr int kGridMaxAxis = 2048;
inline GridIndex grid_over(double x0, double y0, double x1, double y1, double meanW, double meanH) {
  GridIndex G{0, 0, 1, 1, 1, 1, nullptr, nullptr};
  if (!(x1 >= x0) || !(y1 >= y0)) return G;
  const double W = x1 - x0, H = y1 - y0, A = kGridMaxAxis;
  G.gx = (int)std::min(A, std::max(1.0, std::ceil(W / std::max(meanW, W / A))));
  G.gy = (int)std::min(A, std::max(1.0, std::ceil(H / std::max(meanH, H / A))));
  if (!(G.gx >= 1)) G.gx = 1;
  if (!(G.gy >= 1)) G.gy = 1;
  G.x0 = x0; G.y0 = y0;
  G.cw = W > 0 ? W / G.gx : 1.0;
  G.ch = H > 0 ? H / G.gy : 1.0;
  return G;
}

// kMode 0: entries per cell (cnt, atomics); kMode 1: list each valid MBR in its cells
// (list[off[c] + slot], cnt counting again from zero).  Thread per polygon.
template <int kMode>
__global__ void index_kernel(const double* __restrict__ mbr, const uint8_t* __restrict__ valid, int64_t n,
                             GridIndex G, int32_t* __restrict__ cnt, const int64_t* __restrict__ off,
                             int32_t* __restrict__ list) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || !valid[i]) return;
  double4 m = reinterpret_cast<const double4*>(mbr)[i];
  int x0 = cell_of(m.x, G.x0, G.cw, G.gx), x1 = cell_of(m.z, G.x0, G.cw, G.gx);
  int y0 = cell_of(m.y, G.y0, G.ch, G.gy), y1 = cell_of(m.w, G.y0, G.ch, G.gy);
  for (int y = y0; y <= y1; ++y)
    for (int x = x0; x <= x1; ++x) {
      int64_t c = (int64_t)y * G.gx + x;
      int slot = atomicAdd(&cnt[c], 1);
      if (kMode == 1) list[off[c] + slot] = (int32_t)i;
    }
}

// The join's MBR candidate predicate (GPU_MBR.h:339-539):
// x1b <= x1o < x2b or x1o < x1b <= x2o, and closed overlap in y.
__device__ __forceinline__ bool sweep_pair(double4 B, double4 O) {
  bool x = (B.x <= O.x && O.x < B.z) || (O.x < B.x && B.x <= O.z);
  return x && O.y <= B.w && B.y <= O.w;
}

// Warp per probing polygon q (the "base" side of the predicate): the indexed polygons
// listed in the cells of q's MBR that pass the predicate, each taken in the cell of the
// overlap's lower-left corner.  The lanes take the cells (32 at a time, row by row), each
// lane every entry of its cell, so a box spanning thousands of cells is probed in
// parallel.  kMode 0 counts (cnt[q]); kMode 1 writes keys (q << obits | o) from off[q]
// (order within q is the cells' order; the caller sorts).
__device__ __forceinline__ bool grid_hit(const double4& B, const double* __restrict__ rmbr, int32_t o,
                                         const GridIndex& G, int x, int y) {
  const double4 O = reinterpret_cast<const double4*>(rmbr)[o];
  if (!sweep_pair(B, O)) return false;
  const double cx = fmax(B.x, O.x), cy = fmax(B.y, O.y);
  return cell_of(cx, G.x0, G.cw, G.gx) == x && cell_of(cy, G.y0, G.ch, G.gy) == y;
}

template <int kMode>
__global__ void candidate_kernel(const double* __restrict__ qmbr, const uint8_t* __restrict__ qvalid, int64_t nq,
                                 const double* __restrict__ rmbr, GridIndex G, int32_t* __restrict__ cnt,
                                 const int64_t* __restrict__ off, uint64_t* __restrict__ keys, int obits) {
  int64_t w = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (w >= nq) return;
  int64_t c = 0;
  if (qvalid[w]) {
    const double4 B = reinterpret_cast<const double4*>(qmbr)[w];
    const int x0 = cell_of(B.x, G.x0, G.cw, G.gx), x1 = cell_of(B.z, G.x0, G.cw, G.gx);
    const int y0 = cell_of(B.y, G.y0, G.ch, G.gy), y1 = cell_of(B.w, G.y0, G.ch, G.gy);
    const int nx = x1 - x0 + 1;
    const int64_t ncells = (int64_t)nx * (y1 - y0 + 1);
    int64_t pos = (kMode == 1) ? off[w] : 0;
    for (int64_t j0 = 0; j0 < ncells; j0 += 32) {
      const int64_t j = j0 + lane_id();
      int x = 0, y = 0;
      int64_t e0 = 0, e1 = 0;
      if (j < ncells) {
        y = y0 + (int)(j / nx);
        x = x0 + (int)(j - (int64_t)(y - y0) * nx);
        const int64_t cell = (int64_t)y * G.gx + x;
        e0 = G.cellOff[cell];
        e1 = G.cellOff[cell + 1];
      }
      int h = 0;
      for (int64_t e = e0; e < e1; ++e) h += grid_hit(B, rmbr, G.cellList[e], G, x, y) ? 1 : 0;
      if (kMode == 1) {
        int incl = h;                                // this lane's first key: pos + exclusive scan
        for (int d = 1; d < 32; d <<= 1) {
          const int t = __shfl_up_sync(0xffffffffu, incl, d);
          if ((int)lane_id() >= d) incl += t;
        }
        int64_t p = pos + incl - h;
        if (h)
          for (int64_t e = e0; e < e1; ++e) {
            const int32_t o = G.cellList[e];
            if (grid_hit(B, rmbr, o, G, x, y)) keys[p++] = ((uint64_t)w << obits) | (uint64_t)o;
          }
        pos += __shfl_sync(0xffffffffu, incl, 31);
      }
      c += h;
    }
  }
  if (kMode == 0) {
    for (int d = 16; d > 0; d >>= 1) c += __shfl_xor_sync(0xffffffffu, c, d);
    if (lane_id() == 0) cnt[w] = (int32_t)c;
  }
}

// Extent and mean box size of the valid MBRs: per block, (min x1, min y1, max x2, max
// y2, sum of widths, sum of heights, count) into part[7 * blockIdx.x ...]; the host adds
// the blocks' partials in a fixed order.
constexpr int kExtentThreads = 256;
__global__ void __launch_bounds__(kExtentThreads) mbr_extent_kernel(const double* __restrict__ mbr,
                                                                    const uint8_t* __restrict__ valid, int64_t n,
                                                                    double* __restrict__ part) {
  __shared__ double s[7][kExtentThreads / 32];
  double v[7] = {INFINITY, INFINITY, -INFINITY, -INFINITY, 0.0, 0.0, 0.0};
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    if (!valid[i]) continue;
    const double4 m = reinterpret_cast<const double4*>(mbr)[i];
    v[0] = fmin(v[0], m.x); v[1] = fmin(v[1], m.y); v[2] = fmax(v[2], m.z); v[3] = fmax(v[3], m.w);
    v[4] += m.z - m.x; v[5] += m.w - m.y; v[6] += 1.0;
  }
  v[0] = warp_min(v[0]); v[1] = warp_min(v[1]); v[2] = warp_max(v[2]); v[3] = warp_max(v[3]);
  for (int k = 4; k < 7; ++k)
    for (int d = 16; d > 0; d >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], d);
  const int w = threadIdx.x >> 5;
  if (lane_id() == 0)
    for (int k = 0; k < 7; ++k) s[k][w] = v[k];
  __syncthreads();
  if (threadIdx.x == 0) {
    double r[7] = {INFINITY, INFINITY, -INFINITY, -INFINITY, 0.0, 0.0, 0.0};
    for (int j = 0; j < kExtentThreads / 32; ++j) {
      r[0] = fmin(r[0], s[0][j]); r[1] = fmin(r[1], s[1][j]);
      r[2] = fmax(r[2], s[2][j]); r[3] = fmax(r[3], s[3][j]);
      for (int k = 4; k < 7; ++k) r[k] += s[k][j];
    }
    for (int k = 0; k < 7; ++k) part[7 * blockIdx.x + k] = r[k];
  }
}

}  // namespace
}  // namespace gcmfgh
