// common.cuh -- shared device helpers for the join-and-clip kernels (sm_100a).
//
// All geometric arithmetic follows the reference's operation order and is compiled
// with --fmad=false, so every a*b+c is two IEEE-rounded operations, exactly as the
// reference's host code computes it; results are bit-identical to a CPU evaluation.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#define GCMFGH_DEV __device__ __forceinline__

namespace gcmfgh {

constexpr int kWarp = 32;

// ---- error word written by kernels (never __trap): first error wins
enum DevError : int {
  DEV_OK = 0,
  DEV_CAPACITY = 1,      // a per-pair or global buffer bound was exceeded
  DEV_TRACE = 2,         // tracing did not return to its start within its step budget
  DEV_BAD_INPUT = 3,
  DEV_TIMEOUT = 4,       // a bounded spin-wait gave up
};

GCMFGH_DEV void raise_error(int* err, int code) {
  if (err) atomicCAS(err, 0, code);
}

// host-side count of kernel launches issued by the library (gcmfgh_launch_count)
unsigned long long& launch_counter();
inline void note_launch() { ++launch_counter(); }

// ---- geometry (reference arithmetic, see file header)

// twice the signed area of the triangle (P,Q,R): point2D.h:78-80, gppolyclip_mDIV512.cu:16-18
GCMFGH_DEV double area2(double px, double py, double qx, double qy, double rx, double ry) {
  return (qx - px) * (ry - py) - (qy - py) * (rx - px);
}

// Intersection type of edges [P1,P2] x [Q1,Q2] and parameters alpha (on P), beta (on Q):
// gppolyclip_mDIV512.cu:95-169.  Types: 0 none, 1 X, 2 T on Q (P1 on Q), 3 T on P
// (Q1 on P), 4 V, 5 X-overlap, 6 T-overlap on Q, 7 T-overlap on P, 8 V-overlap.
// The collinear branch classifies beta with |alpha|, as the reference does (:157).
GCMFGH_DEV int classify_edges(double p1x, double p1y, double p2x, double p2y,
                              double q1x, double q1y, double q2x, double q2y,
                              double eps, double& alpha, double& beta) {
  double AP1 = area2(p1x, p1y, q1x, q1y, q2x, q2y);
  double AP2 = area2(p2x, p2y, q1x, q1y, q2x, q2y);
  if (fabs(AP1 - AP2) > eps) {
    double AQ1 = area2(q1x, q1y, p1x, p1y, p2x, p2y);
    double AQ2 = area2(q2x, q2y, p1x, p1y, p2x, p2y);
    alpha = AP1 / (AP1 - AP2);
    beta = AQ1 / (AQ1 - AQ2);
    bool a01 = (alpha > eps && alpha < 1.0 - eps);
    bool a0 = !a01 && fabs(alpha) <= eps;
    bool b01 = (beta > eps && beta < 1.0 - eps);
    bool b0 = !b01 && fabs(beta) <= eps;
    if (a01 && b01) return 1;
    if (a0 && b01) return 2;
    if (b0 && a01) return 3;
    if (a0 && b0) return 4;
  } else if (fabs(AP1) < eps) {
    double dPx = p2x - p1x, dPy = p2y - p1y;
    double dQx = q2x - q1x, dQy = q2y - q1y;
    double PQx = q1x - p1x, PQy = q1y - p1y;
    alpha = (PQx * dPx + PQy * dPy) / (dPx * dPx + dPy * dPy);
    beta = -(PQx * dQx + PQy * dQy) / (dQx * dQx + dQy * dQy);
    bool a01 = (alpha > eps && alpha < 1.0 - eps);
    bool a0 = !a01 && fabs(alpha) <= eps;
    bool an = !a01 && !a0;
    bool b01 = (beta > eps && beta < 1.0 - eps);
    bool b0 = !b01 && fabs(alpha) <= eps;
    bool bn = !b01 && !b0;
    if (a01 && b01) return 5;
    if (an && b01) return 6;
    if (bn && a01) return 7;
    if (a0 && b0) return 8;
  }
  return 0;
}

// closed overlap of the two edges' boxes: gppolyclip_mDIV512.cu:345-371
GCMFGH_DEV bool edge_boxes_touch(double p1x, double p1y, double p2x, double p2y,
                                 double q1x, double q1y, double q2x, double q2y) {
  double minPX = fmin(p1x, p2x), maxPX = fmax(p1x, p2x);
  double minPY = fmin(p1y, p2y), maxPY = fmax(p1y, p2y);
  double minQX = fmin(q1x, q2x), maxQX = fmax(q1x, q2x);
  double minQY = fmin(q1y, q2y), maxQY = fmax(q1y, q2y);
  if (minPX > maxQX || maxPX < minQX) return false;
  if (minPY > maxQY || maxPY < minQY) return false;
  return true;
}

// edge box vs a box [x1,y1,x2,y2], closed: gppolyclip_mDIV512.cu:406-413, GPU_Join.h:576-577
GCMFGH_DEV bool edge_touches_box(double ax, double ay, double bx, double by,
                                 double cx1, double cy1, double cx2, double cy2) {
  if ((cx1 > ax && cx1 > bx) || (cx2 < ax && cx2 < bx)) return false;
  if ((cy1 > ay && cy1 > by) || (cy2 < ay && cy2 < by)) return false;
  return true;
}

// double -> u64 whose unsigned order equals the numeric order (NaN-free input)
GCMFGH_DEV uint64_t ordered_key(double v) {
  uint64_t b = (uint64_t)__double_as_longlong(v);
  return (b & 0x8000000000000000ull) ? ~b : (b | 0x8000000000000000ull);
}

// ---- warp helpers
GCMFGH_DEV unsigned lane_id() { return threadIdx.x & 31u; }
GCMFGH_DEV unsigned lanemask_lt() { return (1u << lane_id()) - 1u; }

template <class T>
GCMFGH_DEV T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

template <class T>
GCMFGH_DEV T warp_min(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) { T w = __shfl_xor_sync(0xffffffffu, v, o); v = w < v ? w : v; }
  return v;
}

template <class T>
GCMFGH_DEV T warp_max(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) { T w = __shfl_xor_sync(0xffffffffu, v, o); v = w > v ? w : v; }
  return v;
}

// inclusive warp scan
template <class T>
GCMFGH_DEV T warp_incl_scan(T v) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    T w = __shfl_up_sync(0xffffffffu, v, o);
    if ((int)lane_id() >= o) v += w;
  }
  return v;
}

// largest i in [0,n) with a[i] <= x (a sorted ascending, a[0] <= x)
template <class T>
GCMFGH_DEV int64_t upper_index(const T* a, int64_t n, T x) {
  int64_t lo = 0, hi = n;   // invariant: a[lo] <= x, answer in [lo, hi)
  while (hi - lo > 1) {
    int64_t mid = (lo + hi) >> 1;
    if (a[mid] <= x) lo = mid; else hi = mid;
  }
  return lo;
}

}  // namespace gcmfgh
