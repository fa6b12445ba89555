// common.cuh -- shared device helpers for the join-and-clip kernels (sm_100a).
//
// All geometric arithmetic follows the reference's operation order and is compiled
// with --fmad=false, so every a*b+c is two IEEE-rounded operations, exactly as the
// reference's host code computes it; results are bit-identical to a CPU evaluation.
#pragma once
#include <atomic>
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

// GH vertex labels (IntersectionLabel, polygon.h:21-32), entry/exit flags
// (EntryExitLabel) and relative positions (RelativePositionType, polyclip.h:290-295)
enum : int8_t { L_NONE = 0, L_CROSSING, L_BOUNCING, L_LEFT_ON, L_RIGHT_ON, L_ON_ON, L_ON_LEFT,
                L_ON_RIGHT, L_DELAYED_CROSSING, L_DELAYED_BOUNCING };
enum : int8_t { E_EXIT = 0, E_ENTRY = 1, E_NEITHER = 2 };
enum : int { R_LEFT = 0, R_RIGHT = 1, R_IS_P_M = 2, R_IS_P_P = 3 };

// host-side count of kernel launches issued by the library (gcmfgh_launch_count); contexts
// may launch from several host threads
std::atomic<unsigned long long>& launch_counter();
inline void note_launch() { launch_counter().fetch_add(1, std::memory_order_relaxed); }

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

// Both sides' classification of one edge pair in one pass: the P-side type of
// classify_edges(P1,P2,Q1,Q2) (returned, with alpha and beta) and whether the Q side's
// own call classify_edges(Q1,Q2,P1,P2) finds an intersection (*qhit), the check behind the
// reference's invalid-pair test (gppolyclip_mDIV512.cu:1461).  The Q-side call evaluates
// the same four areas with the same operands (its AP1, AP2 are AQ1, AQ2 here and the other
// way round) and the same two quotients with alpha and beta swapped, so they are computed
// once; only its collinear branch, which is rare, runs separately.  Bit-identical to the
// two calls.
GCMFGH_DEV int classify_edges_both(double p1x, double p1y, double p2x, double p2y,
                                   double q1x, double q1y, double q2x, double q2y,
                                   double eps, double& alpha, double& beta, bool& qhit) {
  const double AP1 = area2(p1x, p1y, q1x, q1y, q2x, q2y);
  const double AP2 = area2(p2x, p2y, q1x, q1y, q2x, q2y);
  const double AQ1 = area2(q1x, q1y, p1x, p1y, p2x, p2y);
  const double AQ2 = area2(q2x, q2y, p1x, p1y, p2x, p2y);
  const bool pCross = fabs(AP1 - AP2) > eps, qCross = fabs(AQ1 - AQ2) > eps;
  double qa = 0.0, qb = 0.0;
  if (pCross || qCross) {
    qa = AP1 / (AP1 - AP2);
    qb = AQ1 / (AQ1 - AQ2);
  }
  auto crossing_type = [eps](double a, double b) {
    const bool a01 = (a > eps && a < 1.0 - eps);
    const bool a0 = !a01 && fabs(a) <= eps;
    const bool b01 = (b > eps && b < 1.0 - eps);
    const bool b0 = !b01 && fabs(b) <= eps;
    if (a01 && b01) return 1;
    if (a0 && b01) return 2;
    if (b0 && a01) return 3;
    if (a0 && b0) return 4;
    return 0;
  };
  int tp = 0;
  if (pCross) {
    alpha = qa;
    beta = qb;
    tp = crossing_type(qa, qb);
  } else if (fabs(AP1) < eps) {
    tp = classify_edges(p1x, p1y, p2x, p2y, q1x, q1y, q2x, q2y, eps, alpha, beta);
  }
  if (qCross) {
    qhit = crossing_type(qb, qa) != 0;
  } else if (fabs(AQ1) < eps) {
    double a2, b2;
    qhit = classify_edges(q1x, q1y, q2x, q2y, p1x, p1y, p2x, p2y, eps, a2, b2) != 0;
  } else {
    qhit = false;
  }
  return tp;
}

// ---- exact-predicate mode
//
// Signs of u.v-type expressions  (a1 - a0) * (b1 - b0) -/+ (c1 - c0) * (d1 - d0)  over
// FP64 inputs, exact for every input (no underflow/overflow assumed).  Method: Shewchuk,
// "Adaptive Precision Floating-Point Arithmetic and Fast Robust Geometric Predicates"
// (1997): a forward error bound decides the sign from the plain FP64 value whenever it
// can (stage A of orient2d, bound (3 + 16 e) e (|left| + |right|), e = 2^-53); otherwise
// every difference is split exactly into two doubles (Two-Diff), every partial product
// into two (Two-Product, formed here with a fused multiply-add), and the sixteen doubles
// are summed into a nonoverlapping expansion (Grow-Expansion), whose largest nonzero
// component carries the sign.

GCMFGH_DEV void two_sum(double a, double b, double& s, double& e) {
  s = a + b;
  double bv = s - a;
  double av = s - bv;
  e = (a - av) + (b - bv);
}

GCMFGH_DEV void two_prod(double a, double b, double& p, double& e) {
  p = a * b;
  e = fma(a, b, -p);
}

GCMFGH_DEV int exact_sign_slow(double a1, double a0, double b1, double b0, double c1, double c0,
                                            double d1, double d0, int sub) {
  double ah, al, bh, bl, ch, cl, dh, dl;
  two_sum(a1, -a0, ah, al);
  two_sum(b1, -b0, bh, bl);
  two_sum(c1, -c0, ch, cl);
  two_sum(d1, -d0, dh, dl);
  const double sgn = sub ? -1.0 : 1.0;
  const double fx[4] = {ah, ah, al, al}, fy[4] = {bh, bl, bh, bl};
  const double gx[4] = {ch, ch, cl, cl}, gy[4] = {dh, dl, dh, dl};
  double h[16];
#pragma unroll
  for (int t = 0; t < 8; ++t) {
    double p, e;
    if (t < 4) two_prod(fx[t], fy[t], p, e);
    else { two_prod(gx[t - 4], gy[t - 4], p, e); p *= sgn; e *= sgn; }
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      double q = u == 0 ? e : p;
      const int n = 2 * t + u;            // components so far (compile-time after unrolling)
#pragma unroll
      for (int i = 0; i < n; ++i) {
        double s, r;
        two_sum(q, h[i], s, r);
        h[i] = r;
        q = s;
      }
      h[n] = q;
    }
  }
  int sg = 0;
#pragma unroll
  for (int i = 0; i < 16; ++i)
    if (h[i] != 0.0) sg = h[i] > 0.0 ? 1 : -1;   // the last nonzero component is the largest
  return sg;
}

// sign of (a1-a0)(b1-b0) - (c1-c0)(d1-d0)  (sub = 1)  or  ... + ...  (sub = 0)
GCMFGH_DEV int exact_sign(double a1, double a0, double b1, double b0, double c1, double c0,
                          double d1, double d0, int sub) {
  const double left = (a1 - a0) * (b1 - b0);
  const double right = (c1 - c0) * (d1 - d0);
  const double r = sub ? right : -right;          // value = left - r
  const double det = left - r;
  if (left > 0.0) { if (r <= 0.0) return 1; }
  else if (left < 0.0) { if (r >= 0.0) return -1; }
  else return (r > 0.0) ? -1 : (r < 0.0 ? 1 : 0);
  const double bound = 3.3306690738754716e-16 * (fabs(left) + fabs(r));   // (3 + 16e) e, e = 2^-53
  if (det >= bound || -det >= bound) return det > 0.0 ? 1 : -1;
  return exact_sign_slow(a1, a0, b1, b0, c1, c0, d1, d0, sub);
}

// exact sign of area2(P, Q, R) = (qx - px)(ry - py) - (qy - py)(rx - px)
GCMFGH_DEV int orient_exact(double px, double py, double qx, double qy, double rx, double ry) {
  return exact_sign(qx, px, ry, py, qy, py, rx, px, 1);
}

GCMFGH_DEV int orient_exact_call(double px, double py, double qx, double qy, double rx, double ry) {
  return orient_exact(px, py, qx, qy, rx, ry);
}

// sign of area2 in the selected mode: the FP64 value's sign, or the exact sign
GCMFGH_DEV int orient_sign(int exact, double px, double py, double qx, double qy, double rx, double ry) {
  if (exact) return orient_exact_call(px, py, qx, qy, rx, ry);
  const double v = area2(px, py, qx, qy, rx, ry);
  return (v > 0.0) - (v < 0.0);
}

// exact sign of (U1 - U0) . (V1 - V0)
GCMFGH_DEV int dot_exact(double u1x, double u1y, double u0x, double u0y, double v1x, double v1y, double v0x,
                         double v0y) {
  return exact_sign(u1x, u0x, v1x, v0x, u1y, u0y, v1y, v0y, 0);
}

// FP64 parameter alpha = A1 / (A1 - A2) of a crossing whose exact signs are known to
// straddle: kept in [0, 1] when rounding of A1, A2 says otherwise.
GCMFGH_DEV double crossing_param(double A1, double A2) {
  double t = A1 / (A1 - A2);
  if (!(t >= 0.0)) t = 0.0;
  if (t > 1.0) t = 1.0;
  return t;
}

// Edge classification with exact predicates (same nine types as classify_edges).
// Non-collinear edges: alpha in (0,1) iff P1, P2 lie strictly on opposite sides of line
// Q; alpha == 0 iff P1 lies on it; likewise beta with Q1, Q2 and line P.  Collinear
// edges: the order of Q1 along P and of P1 along Q from exact dot-product signs;
// "b0" is Q1 == P1, which is what the tolerance rule reduces to without tolerance.
// alpha/beta values are the FP64 expressions of the reference, clamped to [0, 1].
GCMFGH_DEV int classify_exact(double p1x, double p1y, double p2x, double p2y,
                              double q1x, double q1y, double q2x, double q2y,
                              double& alpha, double& beta) {
  const int s1 = orient_exact(p1x, p1y, q1x, q1y, q2x, q2y);
  const int s2 = orient_exact(p2x, p2y, q1x, q1y, q2x, q2y);
  if (s1 != 0 || s2 != 0) {
    if (s1 == s2) return 0;
    const int t1 = orient_exact(q1x, q1y, p1x, p1y, p2x, p2y);
    const int t2 = orient_exact(q2x, q2y, p1x, p1y, p2x, p2y);
    const bool a01 = s1 * s2 < 0, a0 = s1 == 0;
    const bool b01 = t1 * t2 < 0, b0 = t1 == 0;
    if (!((a01 || a0) && (b01 || b0))) return 0;
    const double AP1 = area2(p1x, p1y, q1x, q1y, q2x, q2y), AP2 = area2(p2x, p2y, q1x, q1y, q2x, q2y);
    const double AQ1 = area2(q1x, q1y, p1x, p1y, p2x, p2y), AQ2 = area2(q2x, q2y, p1x, p1y, p2x, p2y);
    alpha = a0 ? 0.0 : crossing_param(AP1, AP2);
    beta = b0 ? 0.0 : crossing_param(AQ1, AQ2);
    if (a01 && b01) return 1;
    if (a0 && b01) return 2;
    if (b0 && a01) return 3;
    return 4;
  }
  const bool same = (p1x == q1x && p1y == q1y);
  const bool a01 = dot_exact(q1x, q1y, p1x, p1y, p2x, p2y, p1x, p1y) > 0 &&
                   dot_exact(p2x, p2y, q1x, q1y, p2x, p2y, p1x, p1y) > 0;
  const bool b01 = dot_exact(p1x, p1y, q1x, q1y, q2x, q2y, q1x, q1y) > 0 &&
                   dot_exact(q2x, q2y, p1x, p1y, q2x, q2y, q1x, q1y) > 0;
  const bool a0 = !a01 && same, an = !a01 && !a0;
  const bool b0 = !b01 && same, bn = !b01 && !b0;
  const int tp = (a01 && b01) ? 5 : (an && b01) ? 6 : (bn && a01) ? 7 : (a0 && b0) ? 8 : 0;
  if (tp) {
    double dPx = p2x - p1x, dPy = p2y - p1y;
    double dQx = q2x - q1x, dQy = q2y - q1y;
    double PQx = q1x - p1x, PQy = q1y - p1y;
    alpha = (PQx * dPx + PQy * dPy) / (dPx * dPx + dPy * dPy);
    beta = -(PQx * dQx + PQy * dQy) / (dQx * dQx + dQy * dQy);
    if (a01) alpha = fmin(fmax(alpha, 0.0), 1.0);
    if (b01) beta = fmin(fmax(beta, 0.0), 1.0);
    if (a0) alpha = 0.0;
    if (b0) beta = 0.0;
  }
  return tp;
}

GCMFGH_DEV int classify_exact_call(double p1x, double p1y, double p2x, double p2y, double q1x,
                                   double q1y, double q2x, double q2y, double* ab) {
  return classify_exact(p1x, p1y, p2x, p2y, q1x, q1y, q2x, q2y, ab[0], ab[1]);
}

GCMFGH_DEV int classify_mode(int exact, double p1x, double p1y, double p2x, double p2y, double q1x,
                             double q1y, double q2x, double q2y, double eps, double& alpha, double& beta) {
  if (exact) {
    double ab[2] = {alpha, beta};
    int t = classify_exact_call(p1x, p1y, p2x, p2y, q1x, q1y, q2x, q2y, ab);
    alpha = ab[0];
    beta = ab[1];
    return t;
  }
  return classify_edges(p1x, p1y, p2x, p2y, q1x, q1y, q2x, q2y, eps, alpha, beta);
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
