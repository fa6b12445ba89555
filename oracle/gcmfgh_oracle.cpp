// gcmfgh_oracle.cpp -- CPU ORACLE. TEST INFRASTRUCTURE ONLY.
//
// A plain, sequential C++ restatement of the reference's join-and-clip path, used by
// tests/, by __graft_entry__.smoke() and by bench.py's CPU-baseline leg as the checker.
// It is never linked into, called by, or shipped with the product library.
//
// Parity pin: the clip half is checked against the reference's own sequential GH code
// compiled from its sources (oracle/_ref/ghclip_ref, see oracle/ref/) on the reference's
// Fig goldens and on seeded random pairs; tests/golden/ holds the fixtures.
//
// What it restates (reference paths are relative to the reference repository root):
//   * MBR per polygon over all stored vertices (SEQ_Overlay.h:316-344; the closing
//     vertex is stored and therefore included).
//   * MBR candidate predicate of the sort-based sweep join (GPU_MBR.h:339-415,
//     420-539 over keys sorted stably by (value, endpoint index)).  Worked out on
//     values, the sweep accepts a (base b, overlay o) pair iff
//       x1o <= x2b && x1b <= x2o && !(x1o == x2b)  and  y1o <= y2b && y1b <= y2o,
//     i.e. closed overlap except where the overlay starts exactly where the base ends.
//   * Common MBR and containment candidates (GPU_Join.h:461-508).
//   * Point-in-polygon crossing parity (GPU_Join.h:882-939, SEQ_Overlay.h:52-61).
//   * Common-MBR edge filter (GPU_Join.h:562-580, 676-699).
//   * Segment-intersection refine (GPU_Join.h:363-446).
//   * Greiner-Hormann clip: GPU intersection phase semantics (gppolyclip_mDIV512.cu:
//     95-169 classification, 345-371 edge-box filter, 382-415 CMBR edge filter,
//     463-547 counts, 1461 invalid check) followed by the CPU phases of
//     GH-CUDA/lib/polyclip.h (computeIntersections :188-268 vertex insertion and
//     linking, step-1 labels :343-397 as computed on the GPU :1171-1223, chains
//     :405-451, special cases :474-541, entry/exit :549-655, split pairs :661-714,
//     crossing candidates :723-734, tracing :743-783, clean-up :791-807) and
//     polygon.h (pointInPoly :427-448, getNonIntersectionPoint/Vertex :480-512).
//
// Arithmetic: every geometric expression is written in the reference's operation
// order; the Makefile builds with -ffp-contract=off so no a*b+c is fused.
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cmath>
#include <vector>
#include <array>
#include <algorithm>
#include <numeric>
#include <thread>
#include <functional>

namespace {

enum Label : int8_t { NONE = 0, CROSSING, BOUNCING, LEFT_ON, RIGHT_ON, ON_ON, ON_LEFT, ON_RIGHT,
                      DELAYED_CROSSING, DELAYED_BOUNCING };
enum EnEx : int8_t { EXIT = 0, ENTRY = 1, NEITHER = 2 };
enum RelPos { LEFT, RIGHT, IS_P_m, IS_P_p };

struct Pt { double x, y; };

inline double A3(double px, double py, double qx, double qy, double rx, double ry) {
  // twice the signed area of (P,Q,R): point2D.h:78-80, gppolyclip_mDIV512.cu:16-18
  return (qx - px) * (ry - py) - (qy - py) * (rx - px);
}

// Intersection type of [P1,P2] x [Q1,Q2] with alpha (on P) and beta (on Q):
// gppolyclip_mDIV512.cu:95-169 (== polyclip.h:60-179), including the reference's use
// of |alpha| when classifying beta in the collinear branch (:157, polyclip.h:156).
int classify(Pt P1, Pt P2, Pt Q1, Pt Q2, double eps, double& alpha, double& beta) {
  double AP1 = A3(P1.x, P1.y, Q1.x, Q1.y, Q2.x, Q2.y);
  double AP2 = A3(P2.x, P2.y, Q1.x, Q1.y, Q2.x, Q2.y);
  if (std::fabs(AP1 - AP2) > eps) {
    double AQ1 = A3(Q1.x, Q1.y, P1.x, P1.y, P2.x, P2.y);
    double AQ2 = A3(Q2.x, Q2.y, P1.x, P1.y, P2.x, P2.y);
    alpha = AP1 / (AP1 - AP2);
    beta = AQ1 / (AQ1 - AQ2);
    bool a0 = false, a01 = false, b0 = false, b01 = false;
    if (alpha > eps && alpha < 1.0 - eps) a01 = true;
    else if (std::fabs(alpha) <= eps) a0 = true;
    if (beta > eps && beta < 1.0 - eps) b01 = true;
    else if (std::fabs(beta) <= eps) b0 = true;
    if (a01 && b01) return 1;
    if (a0 && b01) return 2;
    if (b0 && a01) return 3;
    if (a0 && b0) return 4;
  } else if (std::fabs(AP1) < eps) {
    double dPx = P2.x - P1.x, dPy = P2.y - P1.y;
    double dQx = Q2.x - Q1.x, dQy = Q2.y - Q1.y;
    double PQx = Q1.x - P1.x, PQy = Q1.y - P1.y;
    alpha = (PQx * dPx + PQy * dPy) / (dPx * dPx + dPy * dPy);
    beta = -(PQx * dQx + PQy * dQy) / (dQx * dQx + dQy * dQy);
    bool a0 = false, a01 = false, an = false, b0 = false, b01 = false, bn = false;
    if (alpha > eps && alpha < 1.0 - eps) a01 = true;
    else if (std::fabs(alpha) <= eps) a0 = true;
    else an = true;
    if (beta > eps && beta < 1.0 - eps) b01 = true;
    else if (std::fabs(alpha) <= eps) b0 = true;
    else bn = true;
    if (a01 && b01) return 5;
    if (an && b01) return 6;
    if (bn && a01) return 7;
    if (a0 && b0) return 8;
  }
  return 0;
}

// ---- exact-predicate mode (the engine's precision option, not a reference behaviour)
//
// Exact signs of (a1-a0)(b1-b0) -/+ (c1-c0)(d1-d0), always through exact arithmetic:
// Two-Diff for the differences, Dekker's split-based Two-Product for the partial
// products, Grow-Expansion for the sum (Shewchuk 1997); the largest nonzero component
// of the nonoverlapping expansion carries the sign.  No error-bound shortcut here, so the
// engine's filtered evaluation is checked against the unconditional one.
inline void twoSum(double a, double b, double& s, double& e) {
  s = a + b;
  double bv = s - a, av = s - bv;
  e = (a - av) + (b - bv);
}
inline void dekkerSplit(double a, double& hi, double& lo) {      // Dekker: 2^27 + 1
  double c = 134217729.0 * a;
  double big = c - a;
  hi = c - big;
  lo = a - hi;
}
inline void twoProd(double a, double b, double& p, double& e) {
  p = a * b;
  double ah, al, bh, bl;
  dekkerSplit(a, ah, al);
  dekkerSplit(b, bh, bl);
  e = al * bl - (((p - ah * bh) - al * bh) - ah * bl);
}
int exactSign(double a1, double a0, double b1, double b0, double c1, double c0, double d1, double d0, bool sub) {
  double d[8];
  twoSum(a1, -a0, d[0], d[1]);
  twoSum(b1, -b0, d[2], d[3]);
  twoSum(c1, -c0, d[4], d[5]);
  twoSum(d1, -d0, d[6], d[7]);
  double h[16];
  int n = 0;
  auto grow = [&](double q) {
    for (int i = 0; i < n; ++i) { double s, r; twoSum(q, h[i], s, r); h[i] = r; q = s; }
    h[n++] = q;
  };
  for (int u = 0; u < 2; ++u)
    for (int v = 0; v < 2; ++v) {
      double p, e;
      twoProd(d[u], d[2 + v], p, e);
      grow(p); grow(e);
      twoProd(d[4 + u], d[6 + v], p, e);
      if (sub) { p = -p; e = -e; }
      grow(p); grow(e);
    }
  for (int i = n - 1; i >= 0; --i)
    if (h[i] != 0.0) return h[i] > 0 ? 1 : -1;
  return 0;
}
inline int orientExact(double px, double py, double qx, double qy, double rx, double ry) {
  return exactSign(qx, px, ry, py, qy, py, rx, px, true);   // sign of A3(P, Q, R)
}
inline int dotExact(Pt U1, Pt U0, Pt V1, Pt V0) {            // sign of (U1-U0).(V1-V0)
  return exactSign(U1.x, U0.x, V1.x, V0.x, U1.y, U0.y, V1.y, V0.y, false);
}
inline double crossingParam(double A1, double A2) {
  double t = A1 / (A1 - A2);
  if (!(t >= 0.0)) t = 0.0;
  if (t > 1.0) t = 1.0;
  return t;
}

// Edge classification with exact signs: the nine types of classify() with every
// tolerance test replaced by its exact counterpart (alpha in (0,1) <=> P1, P2 strictly on
// opposite sides of line Q; alpha == 0 <=> P1 on it; collinear order from exact dot
// signs; Q1 == P1 for the coincident-start cases).  alpha/beta are the FP64 expressions,
// clamped to [0,1].
int classifyExact(Pt P1, Pt P2, Pt Q1, Pt Q2, double& alpha, double& beta) {
  int s1 = orientExact(P1.x, P1.y, Q1.x, Q1.y, Q2.x, Q2.y);
  int s2 = orientExact(P2.x, P2.y, Q1.x, Q1.y, Q2.x, Q2.y);
  if (s1 != 0 || s2 != 0) {
    if (s1 == s2) return 0;
    int t1 = orientExact(Q1.x, Q1.y, P1.x, P1.y, P2.x, P2.y);
    int t2 = orientExact(Q2.x, Q2.y, P1.x, P1.y, P2.x, P2.y);
    bool a01 = s1 * s2 < 0, a0 = s1 == 0, b01 = t1 * t2 < 0, b0 = t1 == 0;
    if (!(a01 || a0) || !(b01 || b0)) return 0;
    double AP1 = A3(P1.x, P1.y, Q1.x, Q1.y, Q2.x, Q2.y), AP2 = A3(P2.x, P2.y, Q1.x, Q1.y, Q2.x, Q2.y);
    double AQ1 = A3(Q1.x, Q1.y, P1.x, P1.y, P2.x, P2.y), AQ2 = A3(Q2.x, Q2.y, P1.x, P1.y, P2.x, P2.y);
    alpha = a0 ? 0.0 : crossingParam(AP1, AP2);
    beta = b0 ? 0.0 : crossingParam(AQ1, AQ2);
    if (a01 && b01) return 1;
    if (a0 && b01) return 2;
    if (b0 && a01) return 3;
    return 4;
  }
  bool same = P1.x == Q1.x && P1.y == Q1.y;
  bool a01 = dotExact(Q1, P1, P2, P1) > 0 && dotExact(P2, Q1, P2, P1) > 0;
  bool b01 = dotExact(P1, Q1, Q2, Q1) > 0 && dotExact(Q2, P1, Q2, Q1) > 0;
  bool a0 = !a01 && same, an = !a01 && !same;
  bool b0 = !b01 && same, bn = !b01 && !same;
  int tp = 0;
  if (a01 && b01) tp = 5;
  else if (an && b01) tp = 6;
  else if (bn && a01) tp = 7;
  else if (a0 && b0) tp = 8;
  if (tp) {
    double dPx = P2.x - P1.x, dPy = P2.y - P1.y;
    double dQx = Q2.x - Q1.x, dQy = Q2.y - Q1.y;
    double PQx = Q1.x - P1.x, PQy = Q1.y - P1.y;
    alpha = (PQx * dPx + PQy * dPy) / (dPx * dPx + dPy * dPy);
    beta = -(PQx * dQx + PQy * dQy) / (dQx * dQx + dQy * dQy);
    if (a01) alpha = std::min(std::max(alpha, 0.0), 1.0);
    if (b01) beta = std::min(std::max(beta, 0.0), 1.0);
    if (a0) alpha = 0.0;
    if (b0) beta = 0.0;
  }
  return tp;
}

// sign of A3 in the selected mode
inline int orientSign(bool exact, double px, double py, double qx, double qy, double rx, double ry) {
  if (exact) return orientExact(px, py, qx, qy, rx, ry);
  double v = A3(px, py, qx, qy, rx, ry);
  return (v > 0) - (v < 0);
}

// gppolyclip_mDIV512.cu:345-371
inline bool edgeBoxesTouch(Pt P1, Pt P2, Pt Q1, Pt Q2) {
  double minPX = std::min(P1.x, P2.x), maxPX = std::max(P1.x, P2.x);
  double minPY = std::min(P1.y, P2.y), maxPY = std::max(P1.y, P2.y);
  double minQX = std::min(Q1.x, Q2.x), maxQX = std::max(Q1.x, Q2.x);
  double minQY = std::min(Q1.y, Q2.y), maxQY = std::max(Q1.y, Q2.y);
  if (minPX > maxQX || maxPX < minQX) return false;
  if (minPY > maxQY || maxPY < minQY) return false;
  return true;
}

// gppolyclip_mDIV512.cu:406-413 (same closed test as GPU_Join.h:576-577)
inline bool edgeTouchesBox(Pt P1, Pt P2, const double* c) {
  double minX = std::min(P1.x, P2.x), minY = std::min(P1.y, P2.y);
  double maxX = std::max(P1.x, P2.x), maxY = std::max(P1.y, P2.y);
  if (minX > c[2] || maxX < c[0]) return false;
  if (minY > c[3] || maxY < c[1]) return false;
  return true;
}

// ---- clean-up (polyclip.h:791-807): drop the root while it is collinear, then one
// forward pass over the remaining vertices; components left empty are dropped.
void cleanUp(std::vector<std::vector<Pt>>& out, double epsClean) {
    for (auto& comp : out) {
      int m = (int)comp.size();
      if (m == 0) continue;
      std::vector<int> nx(m), pv(m);
      for (int i = 0; i < m; ++i) { nx[i] = (i + 1) % m; pv[i] = (i + m - 1) % m; }
      int root = 0, alive = m;
      auto area = [&](int v) {
        return std::fabs(A3(comp[pv[v]].x, comp[pv[v]].y, comp[v].x, comp[v].y, comp[nx[v]].x, comp[nx[v]].y));
      };
      auto remove = [&](int v) {
        if (root == v) { root = nx[v]; if (nx[root] == root) root = -1; }
        nx[pv[v]] = nx[v]; pv[nx[v]] = pv[v];
        --alive;
      };
      while (root >= 0 && area(root) < epsClean) remove(root);
      std::vector<Pt> res;
      if (root >= 0) {
        int start = root, v = root;
        do {
          int nxt = nx[v];
          if (area(v) < epsClean) remove(v);
          v = nxt;
        } while (v != start && root >= 0);
        if (root >= 0) {
          v = root;
          do { res.push_back(comp[v]); v = nx[v]; } while (v != root);
        }
      }
      comp.swap(res);
    }
    std::vector<std::vector<Pt>> kept;
    for (auto& c : out) if (!c.empty()) kept.push_back(std::move(c));
    out.swap(kept);
}

struct Rec { int p, q; double a, b; int type; };

// One polygon ring with explicit links (polygon.h:40-113 vertex/insertVertex).
struct Ring {
  std::vector<double> x, y;
  std::vector<int> next, prev, nbr;
  std::vector<uint8_t> inter, source;
  std::vector<int8_t> label, enex;
  int root = 0;
  int add(double X, double Y, bool src) {
    x.push_back(X); y.push_back(Y); next.push_back(-1); prev.push_back(-1); nbr.push_back(-1);
    inter.push_back(0); source.push_back(src ? 1 : 0); label.push_back(NONE); enex.push_back(NEITHER);
    return (int)x.size() - 1;
  }
  void insertAfter(int v, int after) {   // insertVertex(V, curr) with alpha = -1 (polygon.h:106-112)
    int c = next[after];
    next[prev[c]] = v; prev[v] = prev[c]; next[v] = c; prev[c] = v;
  }
};

struct Clipper {
  double eps, epsClean;
  bool uni, filters;
  bool exact = false;                          // exact-predicate mode
  Ring R[2];                                   // R[0] = P, R[1] = Q
  std::vector<std::vector<Pt>> out;            // result components
  // When set, run() stops after the neighbour links and fills this with what the
  // reference's calculateIntersections returns (gppolyclip_mDIV512.cu:1298-1640).
  struct Export {
    int64_t np = 0, nq = 0;
    std::vector<double> xyP, xyQ;
    std::vector<int32_t> alP, alQ, lbP, lbQ, nbP, nbQ;
  };
  Export* ex = nullptr;
  long long count1P = 0, count1Q = 0, typeCount[9] = {0};
  int status = 0;                              // 0 ok, 1 invalid, 2 disjoint MBRs

  static void link(Ring& a, int i, Ring& b, int j) {   // polygon.h:89-94
    a.nbr[i] = j; b.nbr[j] = i; a.inter[i] = 1; b.inter[j] = 1;
  }

  // polygon.h:427-448 over the ring's current vertices (edges(ALL)).
  static bool pointInPoly(const Ring& Rg, double Rx, double Ry, bool ex) {
    int w = 0;
    int one = Rg.root;
    do {
      int two = Rg.next[one];
      double P0x = Rg.x[one], P0y = Rg.y[one], P1x = Rg.x[two], P1y = Rg.y[two];
      if ((P0y < Ry) != (P1y < Ry)) {
        if (P0x >= Rx) {
          if (P1x > Rx) w = w + 2 * (P1y > P0y) - 1;
          else if ((orientSign(ex, P0x, P0y, P1x, P1y, Rx, Ry) > 0) == (P1y > P0y)) w = w + 2 * (P1y > P0y) - 1;
        } else if (P1x > Rx) {
          if ((orientSign(ex, P0x, P0y, P1x, P1y, Rx, Ry) > 0) == (P1y > P0y)) w = w + 2 * (P1y > P0y) - 1;
        }
      }
      one = two;
    } while (one != Rg.root);
    return (w % 2) != 0;
  }

  RelPos oracleRel(int qv, const Ring& P, int p1, int p2, int p3) const {  // polyclip.h:297-326
    const Ring& Q = R[1];
    if (P.inter[p1] && P.nbr[p1] == qv) return IS_P_m;
    if (P.inter[p3] && P.nbr[p3] == qv) return IS_P_p;
    int s1 = orientSign(exact, Q.x[qv], Q.y[qv], P.x[p1], P.y[p1], P.x[p2], P.y[p2]);
    int s2 = orientSign(exact, Q.x[qv], Q.y[qv], P.x[p2], P.y[p2], P.x[p3], P.y[p3]);
    int s3 = orientSign(exact, P.x[p1], P.y[p1], P.x[p2], P.y[p2], P.x[p3], P.y[p3]);
    if (s3 > 0) return (s1 > 0 && s2 > 0) ? LEFT : RIGHT;
    return (s1 < 0 && s2 < 0) ? RIGHT : LEFT;
  }

  static Label initialLabel(RelPos m, RelPos p) {   // gppolyclip_mDIV512.cu:237-252
    auto has = [&](RelPos a, RelPos b) { return (m == a && p == b) || (m == b && p == a); };
    if (has(LEFT, RIGHT)) return CROSSING;
    if ((m == LEFT && p == LEFT) || (m == RIGHT && p == RIGHT)) return BOUNCING;
    if (has(IS_P_p, RIGHT)) return LEFT_ON;
    if (has(IS_P_p, LEFT)) return RIGHT_ON;
    if (has(IS_P_p, IS_P_m)) return ON_ON;
    if (has(IS_P_m, RIGHT)) return ON_LEFT;
    if (has(IS_P_m, LEFT)) return ON_RIGHT;
    return NONE;
  }

  // vertices of ring rg with intersection flag set, starting at `start` (inclusive if it
  // qualifies), in ring order, evaluated lazily like vertexIterator (polygon.h:194-264).
  template <class F> void forIntersections(Ring& rg, int start, F f) {
    int V = start;
    if (!rg.inter[V]) {
      do { V = rg.next[V]; } while (!rg.inter[V] && V != start);
      if (V == start) return;
    }
    for (;;) {
      f(V);
      do { V = rg.next[V]; } while (!rg.inter[V] && V != start);
      if (V == start) return;
    }
  }

  bool noCrossingVertex(const Ring& rg) const {      // polygon.h:465-475
    int v = rg.root;
    do {
      if (rg.inter[v]) {
        if (rg.label[v] == CROSSING || rg.label[v] == DELAYED_CROSSING) return false;
        if (uni && (rg.label[v] == BOUNCING || rg.label[v] == DELAYED_BOUNCING)) return false;
      }
      v = rg.next[v];
    } while (v != rg.root);
    return true;
  }
  static bool allOnOn(const Ring& rg) {                // polygon.h:453-458
    int v = rg.root;
    do { if (rg.label[v] != ON_ON) return false; v = rg.next[v]; } while (v != rg.root);
    return true;
  }
  // polygon.h:480-491 (first non-intersection vertex, else a safe edge midpoint)
  static bool nonIntersectionPoint(const Ring& rg, const Ring& other, double& px, double& py) {
    int v = rg.root;
    do { if (!rg.inter[v]) { px = rg.x[v]; py = rg.y[v]; return true; } v = rg.next[v]; } while (v != rg.root);
    v = rg.root;
    do {
      int nb = rg.nbr[v], nx = rg.next[v];
      if (nb >= 0 && rg.nbr[nx] != other.prev[nb] && rg.nbr[nx] != other.next[nb]) {
        px = 0.5 * (rg.x[v] + rg.x[nx]); py = 0.5 * (rg.y[v] + rg.y[nx]); return true;
      }
      v = rg.next[v];
    } while (v != rg.root);
    return false;
  }
  // polygon.h:496-512 (may insert a temporary midpoint vertex)
  static int nonIntersectionVertex(Ring& rg, const Ring& other) {
    int v = rg.root;
    do { if (!rg.inter[v]) return v; v = rg.next[v]; } while (v != rg.root);
    v = rg.root;
    do {
      int nb = rg.nbr[v], nx = rg.next[v];
      if (nb >= 0 && rg.nbr[nx] != other.prev[nb] && rg.nbr[nx] != other.next[nb]) {
        int t = rg.add(0.5 * (rg.x[v] + rg.x[nx]), 0.5 * (rg.y[v] + rg.y[nx]), false);
        rg.insertAfter(t, v);
        return t;
      }
      v = rg.next[v];
    } while (v != rg.root);
    return -1;
  }
  std::vector<Pt> ringPoints(const Ring& rg) const {
    std::vector<Pt> pts;
    int v = rg.root;
    do { pts.push_back({rg.x[v], rg.y[v]}); v = rg.next[v]; } while (v != rg.root);
    return pts;
  }

  // ---- calculateIntersections outputs
  void exportPlain(const double* P, int nP, const double* Q, int nQ) {
    ex->np = nP; ex->nq = nQ;
    ex->xyP.assign(P, P + 2 * nP); ex->xyQ.assign(Q, Q + 2 * nQ);
    ex->alP.assign(nP, -100); ex->lbP.assign(nP, -100); ex->nbP.assign(nP, 0);
    ex->alQ.assign(nQ, -100); ex->lbQ.assign(nQ, -100); ex->nbQ.assign(nQ, 0);
  }
  static int32_t alphaKey(double a) { return (int32_t)(10000000.0 * a); }   // (int)pow(10,7)*alpha
  // oracle(), gppolyclip_mDIV512.cu:195-215, with linked-ness read from the keys
  int relKeyed(int pMN, int pPN, int qId, int p1, int p2, int p3) const {
    const Ring& P = R[0];
    const Ring& Q = R[1];
    if (pMN != -100 && pMN == qId) return IS_P_m;
    if (pPN != -100 && pPN == qId) return IS_P_p;
    int s1 = orientSign(exact, Q.x[qId], Q.y[qId], P.x[p1], P.y[p1], P.x[p2], P.y[p2]);
    int s2 = orientSign(exact, Q.x[qId], Q.y[qId], P.x[p2], P.y[p2], P.x[p3], P.y[p3]);
    int s3 = orientSign(exact, P.x[p1], P.y[p1], P.x[p2], P.y[p2], P.x[p3], P.y[p3]);
    if (s3 > 0) return (s1 > 0 && s2 > 0) ? LEFT : RIGHT;
    return (s1 < 0 && s2 < 0) ? RIGHT : LEFT;
  }
  // getInitialLabel, gppolyclip_mDIV512.cu:237-252
  static int32_t labelKeyed(int m, int p) {
    auto has = [&](int a, int b) { return (m == a && p == b) || (m == b && p == a); };
    if (has(LEFT, RIGHT)) return CROSSING;
    if ((m == LEFT && p == LEFT) || (m == RIGHT && p == RIGHT)) return BOUNCING;
    if (has(IS_P_p, RIGHT)) return LEFT_ON;
    if (has(IS_P_p, LEFT)) return RIGHT_ON;
    if (has(IS_P_p, IS_P_m)) return ON_ON;
    if (has(IS_P_m, RIGHT)) return ON_LEFT;
    if (has(IS_P_m, LEFT)) return ON_RIGHT;
    return -102;
  }
  // Rings in slot order (= ring order before labelling).  Keys follow the reference's
  // writes (gppolyclip_mDIV512.cu:926-1053): an inserted vertex gets its record's key; a
  // source vertex gets the key of its last degenerate record in (P edge, Q edge) order --
  // P: types 2/4/6/8, Q: types 3/4/7/8; type 5 keys only its inserted vertices.  Labels
  // as gpuCalculateInitLabel (:1171-1223), in slot order.
  void exportRings(const std::vector<Rec>& recs, const std::vector<int>& srcP, const std::vector<int>& srcQ,
                   const std::vector<int>& insP, const std::vector<int>& insQ) {
    const Ring& RP = R[0];
    const Ring& RQ = R[1];
    const int np = (int)RP.x.size(), nq = (int)RQ.x.size();
    ex->np = np; ex->nq = nq;
    ex->xyP.resize(2 * np); ex->xyQ.resize(2 * nq);
    for (int v = 0; v < np; ++v) { ex->xyP[2 * v] = RP.x[v]; ex->xyP[2 * v + 1] = RP.y[v]; }
    for (int v = 0; v < nq; ++v) { ex->xyQ[2 * v] = RQ.x[v]; ex->xyQ[2 * v + 1] = RQ.y[v]; }
    ex->alP.assign(np, -100); ex->alQ.assign(nq, -100);
    for (size_t r = 0; r < recs.size(); ++r) {
      const Rec& rc = recs[r];
      const int t = rc.type;
      if (t == 1 || t == 3 || t == 5 || t == 7) ex->alP[insP[r]] = alphaKey(rc.a);
      else ex->alP[srcP[rc.p]] = alphaKey(rc.a);
      if (t == 1 || t == 2 || t == 5 || t == 6) ex->alQ[insQ[r]] = alphaKey(rc.b);
      else ex->alQ[srcQ[rc.q]] = alphaKey(rc.b);
    }
    ex->nbP.resize(np); ex->nbQ.resize(nq);
    for (int v = 0; v < np; ++v) ex->nbP[v] = RP.nbr[v] + 1;
    for (int v = 0; v < nq; ++v) ex->nbQ[v] = RQ.nbr[v] + 1;
    ex->lbP.assign(np, -100); ex->lbQ.assign(nq, -100);
    for (int i = 0; i < np; ++i) {
      if (ex->alP[i] == -100) continue;
      const int nId = RP.nbr[i];
      if (nId < 0 || nId >= nq) continue;
      const int pm = (i + np - 1) % np, pp = (i + 1) % np;
      const int pMN = ex->alP[pm] != -100 ? RP.nbr[pm] : -100;
      const int pPN = ex->alP[pp] != -100 ? RP.nbr[pp] : -100;
      const int a = relKeyed(pMN, pPN, (nId + nq - 1) % nq, pm, i, pp);
      const int b = relKeyed(pMN, pPN, (nId + 1) % nq, pm, i, pp);
      const int32_t L = labelKeyed(a, b);
      ex->lbP[i] = L;
      ex->lbQ[nId] = L;
    }
  }

  void run(const double* P, int nP, const double* Q, int nQ) {
    out.clear();
    // ---- MBRs and CMBR (ghcuda.cpp:94-125, readShapefile.h:304-330)
    double mb[2][4];
    const double* src[2] = {P, Q};
    int n[2] = {nP, nQ};
    for (int s = 0; s < 2; ++s) {
      double mnx = src[s][0], mny = src[s][1], mxx = mnx, mxy = mny;
      for (int i = 0; i < n[s]; ++i) {
        double X = src[s][2 * i], Y = src[s][2 * i + 1];
        if (mxx < X) mxx = X;
        if (mnx > X) mnx = X;
        if (mxy < Y) mxy = Y;
        if (mny > Y) mny = Y;
      }
      mb[s][0] = mnx; mb[s][1] = mny; mb[s][2] = mxx; mb[s][3] = mxy;
    }
    if (filters) {
      if (mb[0][0] > mb[1][2] || mb[0][2] < mb[1][0] || mb[0][1] > mb[1][3] || mb[0][3] < mb[1][1]) {
        status = 2;
        if (ex) exportPlain(P, nP, Q, nQ);
        return;
      }
    }
    double cmbr[4] = {std::max(mb[0][0], mb[1][0]), std::max(mb[0][1], mb[1][1]),
                      std::min(mb[0][2], mb[1][2]), std::min(mb[0][3], mb[1][3])};

    // ---- intersection records (gpuCountIntersections / polyclip.h:202-268)
    std::vector<uint8_t> cmP(nP, 1), cmQ(nQ, 1);
    auto ptP = [&](int i) { return Pt{P[2 * i], P[2 * i + 1]}; };
    auto ptQ = [&](int i) { return Pt{Q[2 * i], Q[2 * i + 1]}; };
    if (filters) {
      for (int i = 0; i < nP; ++i) cmP[i] = edgeTouchesBox(ptP(i), ptP((i + 1) % nP), cmbr);
      for (int j = 0; j < nQ; ++j) cmQ[j] = edgeTouchesBox(ptQ(j), ptQ((j + 1) % nQ), cmbr);
    }
    // With the box filter on, only Q edges whose boxes can touch P's edge box matter; for
    // large pairs they are found through a uniform grid of Q-edge boxes (the same set as
    // testing every j, visited in ascending j).  Cells hold about one Q edge each but are
    // never smaller than the Q edges' mean box.  P edges are processed in contiguous
    // blocks by worker threads; blocks are concatenated in P-edge order, so records and
    // counts are the same as one sequential pass.
    const bool gridded = filters && (double)nP * nQ > 4e6;
    int gx = 1, gy = 1;
    double gx0 = cmbr[0], gy0 = cmbr[1], gcw = 1, gch = 1;
    std::vector<int> cellStart, cellItems;
    auto cellOf = [](double v, double v0, double cs, int g) {
      double t = (v - v0) / cs;
      if (!(t > 0)) return 0;
      if (t >= g) return g - 1;
      return (int)t;
    };
    if (gridded) {
      double w = cmbr[2] - cmbr[0], h = cmbr[3] - cmbr[1];
      int target = std::max(1, nQ);
      double sw = 0, sh = 0;
      for (int j = 0; j < nQ; ++j) {
        Pt a = ptQ(j), b = ptQ((j + 1) % nQ);
        sw += std::fabs(b.x - a.x); sh += std::fabs(b.y - a.y);
      }
      if (w > 0 && h > 0) {
        gx = std::max(1, (int)std::ceil(std::sqrt(target * w / h)));
        gy = std::max(1, (int)std::ceil((double)target / gx));
        if (sw > 0) gx = std::min(gx, (int)std::ceil(w / (sw / target)));
        if (sh > 0) gy = std::min(gy, (int)std::ceil(h / (sh / target)));
        gx = std::min(4096, std::max(1, gx));
        gy = std::min(4096, std::max(1, gy));
      }
      gcw = w > 0 ? w / gx : 1;
      gch = h > 0 ? h / gy : 1;
      std::vector<int> cnt((size_t)gx * gy + 1, 0);
      auto span = [&](int j, int& x0, int& x1, int& y0, int& y1) {
        Pt a = ptQ(j), b = ptQ((j + 1) % nQ);
        x0 = cellOf(std::min(a.x, b.x), gx0, gcw, gx); x1 = cellOf(std::max(a.x, b.x), gx0, gcw, gx);
        y0 = cellOf(std::min(a.y, b.y), gy0, gch, gy); y1 = cellOf(std::max(a.y, b.y), gy0, gch, gy);
      };
      for (int j = 0; j < nQ; ++j) {
        if (!cmQ[j]) continue;
        int x0, x1, y0, y1;
        span(j, x0, x1, y0, y1);
        for (int y = y0; y <= y1; ++y)
          for (int x = x0; x <= x1; ++x) cnt[(size_t)y * gx + x]++;
      }
      cellStart.assign(cnt.size(), 0);
      for (size_t c = 1; c < cnt.size(); ++c) cellStart[c] = cellStart[c - 1] + cnt[c - 1];
      cellItems.assign(cellStart.back(), 0);
      std::vector<int> cur(cellStart.begin(), cellStart.end() - 1);
      for (int j = 0; j < nQ; ++j) {
        if (!cmQ[j]) continue;
        int x0, x1, y0, y1;
        span(j, x0, x1, y0, y1);
        for (int y = y0; y <= y1; ++y)
          for (int x = x0; x <= x1; ++x) cellItems[cur[(size_t)y * gx + x]++] = j;
      }
    }
    auto cls = [&](Pt A1, Pt A2, Pt B1, Pt B2, double& al, double& be) {
      return exact ? classifyExact(A1, A2, B1, B2, al, be) : classify(A1, A2, B1, B2, eps, al, be);
    };
    struct Part { std::vector<Rec> recs; long long c1P = 0, c1Q = 0, tc[9] = {0}; };
    auto runBlock = [&](int i0, int i1, Part& out) {
      std::vector<int> qcand;
      for (int i = i0; i < i1; ++i) {
        Pt P1 = ptP(i), P2 = ptP((i + 1) % nP);
        int ncand = nQ;
        if (gridded) {
          qcand.clear();
          if (cmP[i]) {
            int x0 = cellOf(std::min(P1.x, P2.x), gx0, gcw, gx), x1 = cellOf(std::max(P1.x, P2.x), gx0, gcw, gx);
            int y0 = cellOf(std::min(P1.y, P2.y), gy0, gch, gy), y1 = cellOf(std::max(P1.y, P2.y), gy0, gch, gy);
            for (int y = y0; y <= y1; ++y)
              for (int x = x0; x <= x1; ++x) {
                size_t c = (size_t)y * gx + x;
                qcand.insert(qcand.end(), cellItems.begin() + cellStart[c], cellItems.begin() + cellStart[c + 1]);
              }
            std::sort(qcand.begin(), qcand.end());
            qcand.erase(std::unique(qcand.begin(), qcand.end()), qcand.end());
          }
          ncand = (int)qcand.size();
        }
        for (int jj = 0; jj < ncand; ++jj) {
          const int j = gridded ? qcand[jj] : jj;
          Pt Q1 = ptQ(j), Q2 = ptQ((j + 1) % nQ);
          double a = 0, b = 0;
          if (filters) {
            if (!edgeBoxesTouch(P1, P2, Q1, Q2)) continue;
            int tp = (cmP[i] || cmQ[j]) ? cls(P1, P2, Q1, Q2, a, b) : 0;
            if (cmP[i] && tp) out.c1P++;
            if (cmQ[j]) {
              double a2, b2;
              if (cls(Q1, Q2, P1, P2, a2, b2)) out.c1Q++;
            }
            if (tp && cmP[i] && cmQ[j]) { out.recs.push_back({i, j, a, b, tp}); out.tc[tp]++; }
          } else {
            int tp = cls(P1, P2, Q1, Q2, a, b);
            if (tp) { out.recs.push_back({i, j, a, b, tp}); out.tc[tp]++; out.c1P++; out.c1Q++; }
          }
        }
      }
    };
    std::vector<Rec> recs;
    {
      int nth = 1;
      if ((double)nP * nQ > 4e7) {
        unsigned hc = std::thread::hardware_concurrency();
        nth = (int)std::max(1u, std::min(hc ? hc : 1u, 64u));
        if (const char* e = std::getenv("GCMFGH_ORACLE_THREADS")) nth = std::max(1, std::atoi(e));
      }
      nth = std::min(nth, std::max(1, nP));
      std::vector<Part> parts(nth);
      if (nth == 1) {
        runBlock(0, nP, parts[0]);
      } else {
        std::vector<std::thread> th;
        for (int t = 0; t < nth; ++t) {
          int i0 = (int)((int64_t)nP * t / nth), i1 = (int)((int64_t)nP * (t + 1) / nth);
          th.emplace_back(runBlock, i0, i1, std::ref(parts[t]));
        }
        for (auto& x : th) x.join();
      }
      size_t tot = 0;
      for (auto& pt : parts) tot += pt.recs.size();
      recs.reserve(tot);
      for (auto& pt : parts) {
        recs.insert(recs.end(), pt.recs.begin(), pt.recs.end());
        std::vector<Rec>().swap(pt.recs);
        count1P += pt.c1P; count1Q += pt.c1Q;
        for (int t = 0; t < 9; ++t) typeCount[t] += pt.tc[t];
      }
    }
    if (filters && count1P != count1Q) {                         // gppolyclip_mDIV512.cu:1461
      status = 1;
      if (ex) {
        ex->np = nP; ex->nq = nQ;
        for (const Rec& rc : recs) {
          if (rc.type == 1 || rc.type == 3 || rc.type == 5 || rc.type == 7) ex->np++;
          if (rc.type == 1 || rc.type == 2 || rc.type == 5 || rc.type == 6) ex->nq++;
        }
      }
      return;
    }

    // ---- merged rings: source vertex of each edge followed by inserted vertices in
    // ascending parameter; equal parameters keep the later-inserted vertex first
    // (insertVertex, polygon.h:101-113, over the loop order of polyclip.h:202-205).
    Ring& RP = R[0];
    Ring& RQ = R[1];
    RP = Ring(); RQ = Ring();
    std::vector<std::vector<int>> onP(nP), onQ(nQ);
    for (int r = 0; r < (int)recs.size(); ++r) {
      int t = recs[r].type;
      if (t == 1 || t == 3 || t == 5 || t == 7) onP[recs[r].p].push_back(r);
      if (t == 1 || t == 2 || t == 5 || t == 6) onQ[recs[r].q].push_back(r);
    }
    std::vector<int> srcP(nP), srcQ(nQ), insP(recs.size(), -1), insQ(recs.size(), -1);
    for (int i = 0; i < nP; ++i) {
      srcP[i] = RP.add(P[2 * i], P[2 * i + 1], true);
      std::vector<int>& L = onP[i];
      std::stable_sort(L.begin(), L.end(), [&](int u, int v) {
        if (recs[u].a != recs[v].a) return recs[u].a < recs[v].a;
        return recs[u].q > recs[v].q;
      });
      for (int r : L) {
        const Rec& rc = recs[r];
        double X, Y;
        if (rc.type == 1) {
          Pt P1 = ptP(rc.p), P2 = ptP((rc.p + 1) % nP);
          X = (1.0 - rc.a) * P1.x + rc.a * P2.x;
          Y = (1.0 - rc.a) * P1.y + rc.a * P2.y;
        } else {                                   // copy of Q1 (types 3, 5, 7)
          X = Q[2 * rc.q]; Y = Q[2 * rc.q + 1];
        }
        insP[r] = RP.add(X, Y, false);
      }
    }
    for (int j = 0; j < nQ; ++j) {
      srcQ[j] = RQ.add(Q[2 * j], Q[2 * j + 1], true);
      std::vector<int>& L = onQ[j];
      std::stable_sort(L.begin(), L.end(), [&](int u, int v) {
        if (recs[u].b != recs[v].b) return recs[u].b < recs[v].b;
        return recs[u].p > recs[v].p;
      });
      for (int r : L) {
        const Rec& rc = recs[r];
        double X, Y;
        if (rc.type == 1) { X = RP.x[insP[r]]; Y = RP.y[insP[r]]; }
        else { X = P[2 * rc.p]; Y = P[2 * rc.p + 1]; }   // copy of P1 (types 2, 5, 6)
        insQ[r] = RQ.add(X, Y, false);
      }
    }
    for (Ring* rg : {&RP, &RQ}) {
      int m = (int)rg->x.size();
      for (int v = 0; v < m; ++v) { rg->next[v] = (v + 1) % m; rg->prev[v] = (v + m - 1) % m; }
      rg->root = 0;
    }
    // links in the reference's loop order (p outer, q inner): polyclip.h:215-267
    for (int r = 0; r < (int)recs.size(); ++r) {
      const Rec& rc = recs[r];
      switch (rc.type) {
        case 1: link(RP, insP[r], RQ, insQ[r]); break;
        case 5: link(RP, srcP[rc.p], RQ, insQ[r]); link(RP, insP[r], RQ, srcQ[rc.q]); break;
        case 2: case 6: link(RP, srcP[rc.p], RQ, insQ[r]); break;
        case 3: case 7: link(RP, insP[r], RQ, srcQ[rc.q]); break;
        case 4: case 8: link(RP, srcP[rc.p], RQ, srcQ[rc.q]); break;
      }
    }

    if (ex) { exportRings(recs, srcP, srcQ, insP, insQ); return; }

    // ---- step 1: initial labels on P, copied to the neighbour on Q
    forIntersections(RP, RP.root, [&](int I) {
      int nb = RP.nbr[I];
      RelPos qm = oracleRel(RQ.prev[nb], RP, RP.prev[I], I, RP.next[I]);
      RelPos qp = oracleRel(RQ.next[nb], RP, RP.prev[I], I, RP.next[I]);
      Label L = initialLabel(qm, qp);
      if (L != NONE) { RP.label[I] = L; RQ.label[nb] = L; }
    });

    // ---- step 2: intersection chains (polyclip.h:405-451)
    forIntersections(RP, RP.root, [&](int I0) {
      if (RP.label[I0] == LEFT_ON || RP.label[I0] == RIGHT_ON) {
        RelPos x = RP.label[I0] == LEFT_ON ? LEFT : RIGHT;
        int X = I0, I = I0;
        do {
          RP.label[I] = NONE;
          RQ.label[RP.nbr[I]] = NONE;
          I = RP.next[I];
        } while (RP.label[I] == ON_ON);
        RelPos y = RP.label[I] == ON_LEFT ? LEFT : RIGHT;
        Label ct = (x != y) ? DELAYED_CROSSING : DELAYED_BOUNCING;
        RP.label[X] = ct; RP.label[I] = ct;
        RQ.label[RP.nbr[X]] = ct; RQ.label[RP.nbr[I]] = ct;
      }
    });

    // ---- step 3.5: components without crossings (polyclip.h:474-541)
    bool noInter[2] = {false, false}, ident[2] = {false, false};
    for (int s = 0; s < 2; ++s) {
      Ring& A = R[s];
      Ring& B = R[1 - s];
      if (noCrossingVertex(A)) {
        noInter[s] = true;
        if (allOnOn(A)) ident[s] = true;
        else {
          double px = 0, py = 0;
          nonIntersectionPoint(A, B, px, py);
          bool inside = pointInPoly(B, px, py, exact);
          if (inside ^ uni) out.push_back(ringPoints(A));
        }
      }
    }
    if (ident[0] && ident[1]) out.push_back(ringPoints(RP));

    // ---- step 4: entry/exit flags (polyclip.h:549-655)
    std::vector<int> split[2], cand[2];
    for (int s = 0; s < 2; ++s) {
      if (noInter[s]) continue;
      Ring& A = R[s];
      Ring& B = R[1 - s];
      int V = nonIntersectionVertex(A, B);
      if (V < 0) continue;
      int st = ENTRY;
      if (pointInPoly(B, A.x[V], A.y[V], exact)) st = EXIT;
      bool first = true;
      auto toggle = [&]() { st = (st == ENTRY) ? EXIT : ENTRY; };
      forIntersections(A, V, [&](int I) {
        if (A.label[I] == CROSSING) { A.enex[I] = st; toggle(); }
        if (A.label[I] == BOUNCING && ((st == EXIT) ^ uni)) split[s].push_back(I);
        if (A.label[I] == DELAYED_CROSSING) {
          A.enex[I] = st;
          if (first) { if ((st == EXIT) ^ uni) A.label[I] = CROSSING; first = false; }
          else { if ((st == ENTRY) ^ uni) A.label[I] = CROSSING; first = true; toggle(); }
        }
        if (A.label[I] == DELAYED_BOUNCING) {
          A.enex[I] = st;
          if (first) { if ((st == EXIT) ^ uni) cand[s].push_back(I); first = false; }
          else { if ((st == ENTRY) ^ uni) cand[s].push_back(I); first = true; }
          toggle();
        }
      });
    }

    // ---- step 5: split vertex pairs (polyclip.h:661-714), processed in P ring order
    {
      std::vector<uint8_t> inSplitQ(RQ.x.size(), 0);
      for (int v : split[1]) inSplitQ[v] = 1;
      std::vector<int> order = split[0];
      for (int IP : order) {
        int IQ = RP.nbr[IP];
        if (IQ < 0 || IQ >= (int)inSplitQ.size() || !inSplitQ[IQ]) continue;
        int VP = RP.add(RP.x[IP], RP.y[IP], false);
        int VQ = RQ.add(RQ.x[IQ], RQ.y[IQ], false);
        double sP = A3(RP.x[RP.prev[IP]], RP.y[RP.prev[IP]], RP.x[IP], RP.y[IP], RP.x[RP.next[IP]], RP.y[RP.next[IP]]);
        double sQ = A3(RQ.x[RQ.prev[IQ]], RQ.y[RQ.prev[IQ]], RQ.x[IQ], RQ.y[IQ], RQ.x[RQ.next[IQ]], RQ.y[RQ.next[IQ]]);
        bool same = exact ? orientSign(true, RP.x[RP.prev[IP]], RP.y[RP.prev[IP]], RP.x[IP], RP.y[IP],
                                       RP.x[RP.next[IP]], RP.y[RP.next[IP]]) *
                                orientSign(true, RQ.x[RQ.prev[IQ]], RQ.y[RQ.prev[IQ]], RQ.x[IQ], RQ.y[IQ],
                                       RQ.x[RQ.next[IQ]], RQ.y[RQ.next[IQ]]) > 0
                          : sP * sQ > 0;
        if (same) { link(RP, IP, RQ, VQ); link(RP, VP, RQ, IQ); }
        else link(RP, VP, RQ, VQ);
        RP.insertAfter(VP, IP);
        RQ.insertAfter(VQ, IQ);
        int8_t e1 = uni ? ENTRY : EXIT, e2 = uni ? EXIT : ENTRY;
        RP.enex[IP] = e1; RP.enex[VP] = e2; RQ.enex[IQ] = e1; RQ.enex[VQ] = e2;
        RP.label[IP] = CROSSING; RP.label[VP] = CROSSING; RQ.label[IQ] = CROSSING; RQ.label[VQ] = CROSSING;
      }
    }
    // ---- step 6: crossing candidates (polyclip.h:723-734)
    {
      std::vector<uint8_t> inCandQ(RQ.x.size(), 0);
      for (int v : cand[1]) inCandQ[v] = 1;
      for (int IP : cand[0]) {
        int IQ = RP.nbr[IP];
        if (IQ >= 0 && inCandQ[IQ]) { RP.label[IP] = CROSSING; RQ.label[IQ] = CROSSING; }
      }
    }

    // ---- tracing (polyclip.h:743-783)
    {
      int V0 = RP.root;
      auto isStart = [&](int v) { return RP.inter[v] && RP.label[v] == CROSSING; };
      int I = V0;
      bool have = isStart(I);
      if (!have) {
        do { I = RP.next[I]; } while (!isStart(I) && I != V0);
        have = (I != V0);
      }
      // The reference walks until it is back at I; a malformed labelling can make that
      // walk endless, so it is bounded here and reported as status 3.
      long long budget = 4 * (long long)(RP.x.size() + RQ.x.size()) + 16;
      while (have) {
        std::vector<Pt> comp;
        int side = 0, V = I;
        RP.inter[V] = 0;
        do {
          if (--budget < 0) { status = 3; out.clear(); return; }
          Ring* cur = &R[side];
          int st = cur->enex[V];
          if (st == ENTRY) st = EXIT; else if (st == EXIT) st = ENTRY;
          do {
            if (--budget < 0) { status = 3; out.clear(); return; }
            if ((st == EXIT) ^ uni) V = cur->next[V]; else V = cur->prev[V];
            cur->inter[V] = 0;
            comp.push_back({cur->x[V], cur->y[V]});
          } while (!(cur->enex[V] == st) && !(side == 0 && V == I));
          if (!(side == 0 && V == I)) {
            if (cur->nbr[V] < 0) { status = 3; out.clear(); return; }
            V = cur->nbr[V];
            side = 1 - side;
            R[side].inter[V] = 0;
          }
        } while (!(side == 0 && V == I));
        out.push_back(comp);
        // advance the CROSSING_INTERSECTION iterator from I
        do { I = RP.next[I]; } while (!isStart(I) && I != V0);
        have = (I != V0);
      }
    }

    cleanUp(out, epsClean);
  }
};

// ------------------------------------------------------------------ multi-component pairs
// P and Q each made of several rings (outer boundaries and holes, even-odd).  The
// reference's CPU clipper handles them by looping over components in every phase
// (GH-CUDA/lib/polyclip.h: computeIntersections :202-268 over all component pairs, step 1
// and the chains per component, special cases :474-541 per component with the inside
// test's parity over all components of the other polygon and the hole test for identical
// components, entry/exit :549-655 per component, split pairs and crossing candidates over
// all components, tracing :743-783 from every component of P).  The GPU intersection
// phase has no multi-component form (calculateIntersectionsMultipleComponents is declared
// in GH-CUDA/ghcuda.h:15 and defined nowhere).  With filters on, every (P ring, Q ring)
// pair gets the GPU path's common-MBR edge filter, edge-box test and P/Q count check; a
// failing ring pair makes the whole pair invalid.
struct MultiClipper {
  double eps, epsClean;
  bool uni, filters, exact = false;
  Ring R[2];
  std::vector<int> roots[2];                   // root slot of every component
  std::vector<std::vector<Pt>> out;
  long long count1P = 0, nrec = 0;
  int status = 0;

  static void link(Ring& a, int i, Ring& b, int j) { a.nbr[i] = j; b.nbr[j] = i; a.inter[i] = 1; b.inter[j] = 1; }

  bool pointInComp(const Ring& Rg, int root, double Rx, double Ry) const {   // polygon.h:427-448
    int w = 0, one = root;
    do {
      int two = Rg.next[one];
      double P0x = Rg.x[one], P0y = Rg.y[one], P1x = Rg.x[two], P1y = Rg.y[two];
      if ((P0y < Ry) != (P1y < Ry)) {
        if (P0x >= Rx) {
          if (P1x > Rx) w = w + 2 * (P1y > P0y) - 1;
          else if ((orientSign(exact, P0x, P0y, P1x, P1y, Rx, Ry) > 0) == (P1y > P0y)) w = w + 2 * (P1y > P0y) - 1;
        } else if (P1x > Rx) {
          if ((orientSign(exact, P0x, P0y, P1x, P1y, Rx, Ry) > 0) == (P1y > P0y)) w = w + 2 * (P1y > P0y) - 1;
        }
      }
      one = two;
    } while (one != root);
    return (w % 2) != 0;
  }
  RelPos rel(int qv, int p1, int p2, int p3) const {                      // polyclip.h:297-326
    const Ring& P = R[0];
    const Ring& Q = R[1];
    if (P.inter[p1] && P.nbr[p1] == qv) return IS_P_m;
    if (P.inter[p3] && P.nbr[p3] == qv) return IS_P_p;
    int s1 = orientSign(exact, Q.x[qv], Q.y[qv], P.x[p1], P.y[p1], P.x[p2], P.y[p2]);
    int s2 = orientSign(exact, Q.x[qv], Q.y[qv], P.x[p2], P.y[p2], P.x[p3], P.y[p3]);
    int s3 = orientSign(exact, P.x[p1], P.y[p1], P.x[p2], P.y[p2], P.x[p3], P.y[p3]);
    if (s3 > 0) return (s1 > 0 && s2 > 0) ? LEFT : RIGHT;
    return (s1 < 0 && s2 < 0) ? RIGHT : LEFT;
  }
  template <class F> static void forInter(const Ring& rg, int start, F f) {   // vertexIterator
    int V = start;
    if (!rg.inter[V]) {
      do { V = rg.next[V]; } while (!rg.inter[V] && V != start);
      if (V == start) return;
    }
    for (;;) {
      f(V);
      do { V = rg.next[V]; } while (!rg.inter[V] && V != start);
      if (V == start) return;
    }
  }
  bool noCrossing(const Ring& rg, int root) const {                      // polygon.h:465-475
    int v = root;
    do {
      if (rg.inter[v]) {
        if (rg.label[v] == CROSSING || rg.label[v] == DELAYED_CROSSING) return false;
        if (uni && (rg.label[v] == BOUNCING || rg.label[v] == DELAYED_BOUNCING)) return false;
      }
      v = rg.next[v];
    } while (v != root);
    return true;
  }
  static bool allOnOn(const Ring& rg, int root) {                       // polygon.h:453-458
    int v = root;
    do { if (rg.label[v] != ON_ON) return false; v = rg.next[v]; } while (v != root);
    return true;
  }
  static bool nonInterPoint(const Ring& rg, int root, const Ring& other, double& px, double& py) {
    int v = root;                                                       // polygon.h:480-491
    do { if (!rg.inter[v]) { px = rg.x[v]; py = rg.y[v]; return true; } v = rg.next[v]; } while (v != root);
    v = root;
    do {
      int nb = rg.nbr[v], nx = rg.next[v];
      if (nb >= 0 && rg.nbr[nx] != other.prev[nb] && rg.nbr[nx] != other.next[nb]) {
        px = 0.5 * (rg.x[v] + rg.x[nx]); py = 0.5 * (rg.y[v] + rg.y[nx]); return true;
      }
      v = rg.next[v];
    } while (v != root);
    return false;
  }
  static int nonInterVertex(Ring& rg, int root, const Ring& other) {    // polygon.h:496-512
    int v = root;
    do { if (!rg.inter[v]) return v; v = rg.next[v]; } while (v != root);
    v = root;
    do {
      int nb = rg.nbr[v], nx = rg.next[v];
      if (nb >= 0 && rg.nbr[nx] != other.prev[nb] && rg.nbr[nx] != other.next[nb]) {
        int t = rg.add(0.5 * (rg.x[v] + rg.x[nx]), 0.5 * (rg.y[v] + rg.y[nx]), false);
        rg.insertAfter(t, v);
        return t;
      }
      v = rg.next[v];
    } while (v != root);
    return -1;
  }
  std::vector<Pt> compPoints(const Ring& rg, int root) const {
    std::vector<Pt> pts;
    int v = root;
    do { pts.push_back({rg.x[v], rg.y[v]}); v = rg.next[v]; } while (v != root);
    return pts;
  }

  // rings: interleaved open rings, ring k has sizes[k] vertices
  void run(const double* P, const int32_t* sizesP, int kP, const double* Q, const int32_t* sizesQ, int kQ) {
    out.clear();
    std::vector<int64_t> offP(kP + 1, 0), offQ(kQ + 1, 0);
    for (int i = 0; i < kP; ++i) offP[i + 1] = offP[i] + sizesP[i];
    for (int j = 0; j < kQ; ++j) offQ[j + 1] = offQ[j] + sizesQ[j];
    auto vP = [&](int i, int e) { int n = sizesP[i]; e %= n; return Pt{P[2 * (offP[i] + e)], P[2 * (offP[i] + e) + 1]}; };
    auto vQ = [&](int j, int e) { int n = sizesQ[j]; e %= n; return Pt{Q[2 * (offQ[j] + e)], Q[2 * (offQ[j] + e) + 1]}; };
    auto mbrOf = [&](const double* xy, int64_t o, int n, double* m) {
      m[0] = m[2] = xy[2 * o]; m[1] = m[3] = xy[2 * o + 1];
      for (int k = 0; k < n; ++k) {
        double X = xy[2 * (o + k)], Y = xy[2 * (o + k) + 1];
        m[0] = std::min(m[0], X); m[2] = std::max(m[2], X); m[1] = std::min(m[1], Y); m[3] = std::max(m[3], Y);
      }
    };
    std::vector<std::array<double, 4>> mbP(kP), mbQ(kQ);
    for (int i = 0; i < kP; ++i) mbrOf(P, offP[i], sizesP[i], mbP[i].data());
    for (int j = 0; j < kQ; ++j) mbrOf(Q, offQ[j], sizesQ[j], mbQ[j].data());
    auto cls = [&](Pt A1, Pt A2, Pt B1, Pt B2, double& al, double& be) {
      return exact ? classifyExact(A1, A2, B1, B2, al, be) : classify(A1, A2, B1, B2, eps, al, be);
    };
    // ---- records in the reference's loop order: P component, P edge, Q component, Q edge
    struct MRec { int i, p, j, q; double a, b; int type; };
    std::vector<MRec> recs;
    std::vector<long long> c1P((size_t)kP * kQ, 0), c1Q((size_t)kP * kQ, 0);
    for (int i = 0; i < kP; ++i)
      for (int e = 0; e < sizesP[i]; ++e) {
        Pt P1 = vP(i, e), P2 = vP(i, e + 1);
        for (int j = 0; j < kQ; ++j) {
          const double* a = mbP[i].data();
          const double* b = mbQ[j].data();
          bool disjoint = a[0] > b[2] || a[2] < b[0] || a[1] > b[3] || a[3] < b[1];
          if (filters && disjoint) continue;                       // ghcuda.cpp:109-116 per ring pair
          double cm[4] = {std::max(a[0], b[0]), std::max(a[1], b[1]), std::min(a[2], b[2]), std::min(a[3], b[3])};
          bool cmP = !filters || edgeTouchesBox(P1, P2, cm);
          for (int q = 0; q < sizesQ[j]; ++q) {
            Pt Q1 = vQ(j, q), Q2 = vQ(j, q + 1);
            double al = 0, be = 0;
            int tp;
            if (filters) {
              if (!edgeBoxesTouch(P1, P2, Q1, Q2)) continue;
              bool cmQ = edgeTouchesBox(Q1, Q2, cm);
              tp = (cmP || cmQ) ? cls(P1, P2, Q1, Q2, al, be) : 0;
              if (cmP && tp) c1P[(size_t)i * kQ + j]++;
              if (cmQ) { double a2, b2; if (cls(Q1, Q2, P1, P2, a2, b2)) c1Q[(size_t)i * kQ + j]++; }
              if (!(tp && cmP && cmQ)) continue;
            } else {
              tp = cls(P1, P2, Q1, Q2, al, be);
              if (!tp) continue;
              c1P[(size_t)i * kQ + j]++; c1Q[(size_t)i * kQ + j]++;
            }
            recs.push_back({i, e, j, q, al, be, tp});
          }
        }
      }
    bool counts_differ = false;
    for (size_t k = 0; k < c1P.size(); ++k) {
      count1P += c1P[k];
      if (c1P[k] != c1Q[k]) counts_differ = true;
    }
    if (filters && counts_differ) { status = 1; return; }     // per ring pair, gppolyclip_mDIV512.cu:1461
    nrec = (long long)recs.size();
    // ---- merged rings, component by component
    Ring& RP = R[0];
    Ring& RQ = R[1];
    RP = Ring(); RQ = Ring();
    roots[0].clear(); roots[1].clear();
    std::vector<std::vector<int>> onP(offP[kP]), onQ(offQ[kQ]);
    for (int r = 0; r < (int)recs.size(); ++r) {
      int t = recs[r].type;
      if (t == 1 || t == 3 || t == 5 || t == 7) onP[offP[recs[r].i] + recs[r].p].push_back(r);
      if (t == 1 || t == 2 || t == 5 || t == 6) onQ[offQ[recs[r].j] + recs[r].q].push_back(r);
    }
    std::vector<int> srcP(offP[kP]), srcQ(offQ[kQ]), insP(recs.size(), -1), insQ(recs.size(), -1);
    for (int i = 0; i < kP; ++i) {
      int first = (int)RP.x.size();
      roots[0].push_back(first);
      for (int e = 0; e < sizesP[i]; ++e) {
        srcP[offP[i] + e] = RP.add(vP(i, e).x, vP(i, e).y, true);
        std::vector<int>& L = onP[offP[i] + e];
        // ascending parameter; equal parameters: the later-inserted record (larger
        // (Q component, Q edge)) first, as insertVertex does (polygon.h:101-113)
        std::stable_sort(L.begin(), L.end(), [&](int u, int v) {
          if (recs[u].a != recs[v].a) return recs[u].a < recs[v].a;
          return std::make_pair(recs[u].j, recs[u].q) > std::make_pair(recs[v].j, recs[v].q);
        });
        for (int r : L) {
          const MRec& rc = recs[r];
          double X, Y;
          if (rc.type == 1) {
            Pt P1 = vP(i, e), P2 = vP(i, e + 1);
            X = (1.0 - rc.a) * P1.x + rc.a * P2.x;
            Y = (1.0 - rc.a) * P1.y + rc.a * P2.y;
          } else {
            X = vQ(rc.j, rc.q).x; Y = vQ(rc.j, rc.q).y;
          }
          insP[r] = RP.add(X, Y, false);
        }
      }
      int last = (int)RP.x.size();
      for (int v = first; v < last; ++v) { RP.next[v] = v + 1 < last ? v + 1 : first; RP.prev[v] = v > first ? v - 1 : last - 1; }
    }
    for (int j = 0; j < kQ; ++j) {
      int first = (int)RQ.x.size();
      roots[1].push_back(first);
      for (int e = 0; e < sizesQ[j]; ++e) {
        srcQ[offQ[j] + e] = RQ.add(vQ(j, e).x, vQ(j, e).y, true);
        std::vector<int>& L = onQ[offQ[j] + e];
        std::stable_sort(L.begin(), L.end(), [&](int u, int v) {
          if (recs[u].b != recs[v].b) return recs[u].b < recs[v].b;
          return std::make_pair(recs[u].i, recs[u].p) > std::make_pair(recs[v].i, recs[v].p);
        });
        for (int r : L) {
          const MRec& rc = recs[r];
          double X, Y;
          if (rc.type == 1) { X = RP.x[insP[r]]; Y = RP.y[insP[r]]; }
          else { X = vP(rc.i, rc.p).x; Y = vP(rc.i, rc.p).y; }
          insQ[r] = RQ.add(X, Y, false);
        }
      }
      int last = (int)RQ.x.size();
      for (int v = first; v < last; ++v) { RQ.next[v] = v + 1 < last ? v + 1 : first; RQ.prev[v] = v > first ? v - 1 : last - 1; }
    }
    for (int r = 0; r < (int)recs.size(); ++r) {                  // polyclip.h:215-267
      const MRec& rc = recs[r];
      const int sp = srcP[offP[rc.i] + rc.p], sq = srcQ[offQ[rc.j] + rc.q];
      switch (rc.type) {
        case 1: link(RP, insP[r], RQ, insQ[r]); break;
        case 5: link(RP, sp, RQ, insQ[r]); link(RP, insP[r], RQ, sq); break;
        case 2: case 6: link(RP, sp, RQ, insQ[r]); break;
        case 3: case 7: link(RP, insP[r], RQ, sq); break;
        case 4: case 8: link(RP, sp, RQ, sq); break;
      }
    }
    // ---- step 1 and step 2, per component of P
    for (int root : roots[0])
      forInter(RP, root, [&](int I) {
        int nb = RP.nbr[I];
        Label L = Clipper::initialLabel(rel(RQ.prev[nb], RP.prev[I], I, RP.next[I]),
                                        rel(RQ.next[nb], RP.prev[I], I, RP.next[I]));
        if (L != NONE) { RP.label[I] = L; RQ.label[nb] = L; }
      });
    for (int root : roots[0])
      forInter(RP, root, [&](int I0) {
        if (RP.label[I0] == LEFT_ON || RP.label[I0] == RIGHT_ON) {
          RelPos x = RP.label[I0] == LEFT_ON ? LEFT : RIGHT;
          int X = I0, I = I0;
          do {
            RP.label[I] = NONE;
            RQ.label[RP.nbr[I]] = NONE;
            I = RP.next[I];
          } while (RP.label[I] == ON_ON);
          RelPos y = RP.label[I] == ON_LEFT ? LEFT : RIGHT;
          Label ct = (x != y) ? DELAYED_CROSSING : DELAYED_BOUNCING;
          RP.label[X] = ct; RP.label[I] = ct;
          RQ.label[RP.nbr[X]] = ct; RQ.label[RP.nbr[I]] = ct;
        }
      });
    // ---- step 3.5, per component (polyclip.h:474-541)
    std::vector<uint8_t> noInter[2], ident[2];
    for (int s = 0; s < 2; ++s) {
      noInter[s].assign(roots[s].size(), 0);
      ident[s].assign(roots[s].size(), 0);
      Ring& A = R[s];
      Ring& B = R[1 - s];
      for (size_t c = 0; c < roots[s].size(); ++c) {
        int root = roots[s][c];
        if (!noCrossing(A, root)) continue;
        noInter[s][c] = 1;
        if (allOnOn(A, root)) { ident[s][c] = 1; continue; }
        double px = 0, py = 0;
        nonInterPoint(A, root, B, px, py);
        bool inside = false;
        for (int rb : roots[1 - s]) if (pointInComp(B, rb, px, py)) inside = !inside;
        if (inside ^ uni) out.push_back(compPoints(A, root));
      }
    }
    for (size_t c = 0; c < roots[0].size(); ++c) {                  // identical components
      if (!ident[0][c]) continue;
      const int pr = roots[0][c];
      bool pHole = false;
      for (int r2 : roots[0]) if (r2 != pr && pointInComp(RP, r2, RP.x[pr], RP.y[pr])) pHole = !pHole;
      for (size_t d = 0; d < roots[1].size(); ++d) {
        if (!ident[1][d]) continue;
        const int qr = roots[1][d];
        bool match = false;
        int v = qr;
        do { if (v == RP.nbr[pr]) { match = true; break; } v = RQ.next[v]; } while (v != qr);
        if (!match) continue;
        bool qHole = false;
        for (int r2 : roots[1]) if (r2 != qr && pointInComp(RQ, r2, RQ.x[qr], RQ.y[qr])) qHole = !qHole;
        if (pHole == qHole) out.push_back(compPoints(RP, pr));
        break;
      }
    }
    // ---- step 4, per component (polyclip.h:549-655)
    std::vector<int> split[2], cand[2];
    for (int s = 0; s < 2; ++s) {
      Ring& A = R[s];
      Ring& B = R[1 - s];
      for (size_t c = 0; c < roots[s].size(); ++c) {
        if (noInter[s][c]) continue;
        int V = nonInterVertex(A, roots[s][c], B);
        if (V < 0) continue;
        int st = ENTRY;
        for (int rb : roots[1 - s]) if (pointInComp(B, rb, A.x[V], A.y[V])) st = (st == ENTRY) ? EXIT : ENTRY;
        bool first = true;
        auto toggle = [&]() { st = (st == ENTRY) ? EXIT : ENTRY; };
        forInter(A, V, [&](int I) {
          if (A.label[I] == CROSSING) { A.enex[I] = st; toggle(); }
          if (A.label[I] == BOUNCING && ((st == EXIT) ^ uni)) split[s].push_back(I);
          if (A.label[I] == DELAYED_CROSSING) {
            A.enex[I] = st;
            if (first) { if ((st == EXIT) ^ uni) A.label[I] = CROSSING; first = false; }
            else { if ((st == ENTRY) ^ uni) A.label[I] = CROSSING; first = true; toggle(); }
          }
          if (A.label[I] == DELAYED_BOUNCING) {
            A.enex[I] = st;
            if (first) { if ((st == EXIT) ^ uni) cand[s].push_back(I); first = false; }
            else { if ((st == ENTRY) ^ uni) cand[s].push_back(I); first = true; }
            toggle();
          }
        });
      }
    }
    // ---- step 5: split vertex pairs, in the order P's components found them
    {
      std::vector<uint8_t> inSplitQ(RQ.x.size(), 0);
      for (int v : split[1]) inSplitQ[v] = 1;
      std::vector<int> order = split[0];
      for (int IP : order) {
        int IQ = RP.nbr[IP];
        if (IQ < 0 || IQ >= (int)inSplitQ.size() || !inSplitQ[IQ]) continue;
        int VP = RP.add(RP.x[IP], RP.y[IP], false);
        int VQ = RQ.add(RQ.x[IQ], RQ.y[IQ], false);
        double sP = A3(RP.x[RP.prev[IP]], RP.y[RP.prev[IP]], RP.x[IP], RP.y[IP], RP.x[RP.next[IP]], RP.y[RP.next[IP]]);
        double sQ = A3(RQ.x[RQ.prev[IQ]], RQ.y[RQ.prev[IQ]], RQ.x[IQ], RQ.y[IQ], RQ.x[RQ.next[IQ]], RQ.y[RQ.next[IQ]]);
        bool same = exact ? orientSign(true, RP.x[RP.prev[IP]], RP.y[RP.prev[IP]], RP.x[IP], RP.y[IP],
                                       RP.x[RP.next[IP]], RP.y[RP.next[IP]]) *
                                orientSign(true, RQ.x[RQ.prev[IQ]], RQ.y[RQ.prev[IQ]], RQ.x[IQ], RQ.y[IQ],
                                       RQ.x[RQ.next[IQ]], RQ.y[RQ.next[IQ]]) > 0
                          : sP * sQ > 0;
        if (same) { link(RP, IP, RQ, VQ); link(RP, VP, RQ, IQ); }
        else link(RP, VP, RQ, VQ);
        RP.insertAfter(VP, IP);
        RQ.insertAfter(VQ, IQ);
        int8_t e1 = uni ? ENTRY : EXIT, e2 = uni ? EXIT : ENTRY;
        RP.enex[IP] = e1; RP.enex[VP] = e2; RQ.enex[IQ] = e1; RQ.enex[VQ] = e2;
        RP.label[IP] = CROSSING; RP.label[VP] = CROSSING; RQ.label[IQ] = CROSSING; RQ.label[VQ] = CROSSING;
      }
    }
    // ---- step 6: crossing candidates
    {
      std::vector<uint8_t> inCandQ(RQ.x.size(), 0);
      for (int v : cand[1]) inCandQ[v] = 1;
      for (int IP : cand[0]) {
        int IQ = RP.nbr[IP];
        if (IQ >= 0 && inCandQ[IQ]) { RP.label[IP] = CROSSING; RQ.label[IQ] = CROSSING; }
      }
    }
    // ---- tracing from every component of P (polyclip.h:743-783)
    long long budget = 4 * (long long)(RP.x.size() + RQ.x.size()) + 16;
    for (int V0 : roots[0]) {
      auto isStart = [&](int v) { return RP.inter[v] && RP.label[v] == CROSSING; };
      int I = V0;
      bool have = isStart(I);
      if (!have) {
        do { I = RP.next[I]; } while (!isStart(I) && I != V0);
        have = (I != V0);
      }
      while (have) {
        std::vector<Pt> comp;
        int side = 0, V = I;
        RP.inter[V] = 0;
        do {
          if (--budget < 0) { status = 3; out.clear(); return; }
          Ring* cur = &R[side];
          int st = cur->enex[V];
          if (st == ENTRY) st = EXIT; else if (st == EXIT) st = ENTRY;
          do {
            if (--budget < 0) { status = 3; out.clear(); return; }
            if ((st == EXIT) ^ uni) V = cur->next[V]; else V = cur->prev[V];
            cur->inter[V] = 0;
            comp.push_back({cur->x[V], cur->y[V]});
          } while (!(cur->enex[V] == st) && !(side == 0 && V == I));
          if (!(side == 0 && V == I)) {
            if (cur->nbr[V] < 0) { status = 3; out.clear(); return; }
            V = cur->nbr[V];
            side = 1 - side;
            R[side].inter[V] = 0;
          }
        } while (!(side == 0 && V == I));
        out.push_back(comp);
        do { I = RP.next[I]; } while (!isStart(I) && I != V0);
        have = (I != V0);
      }
    }
    cleanUp(out, epsClean);
  }
};

// ------------------------------------------------------------------ result store
struct Store {
  std::vector<int32_t> status, ncomp;
  std::vector<int64_t> count1, nrec;
  std::vector<int32_t> compSize;
  std::vector<double> xy;
  void clear() { status.clear(); ncomp.clear(); count1.clear(); nrec.clear(); compSize.clear(); xy.clear(); }
} g_store;

void storeResult(const Clipper& c) {
  g_store.status.push_back(c.status);
  g_store.ncomp.push_back((int32_t)c.out.size());
  g_store.count1.push_back(c.count1P);
  long long nr = 0;
  for (int t = 1; t < 9; ++t) nr += c.typeCount[t];
  g_store.nrec.push_back(nr);
  for (auto& comp : c.out) {
    g_store.compSize.push_back((int32_t)comp.size());
    for (auto& p : comp) { g_store.xy.push_back(p.x); g_store.xy.push_back(p.y); }
  }
}

}  // namespace

extern "C" {

// Clip one pair.  P, Q: open rings (no closing vertex), interleaved x,y.
// flags bit0: union instead of intersection.  bit1: GPU-path semantics (CMBR and edge-box
// filters, P/Q count cross-check); without it, the reference's CPU path (every edge pair).
// bit2: exact-predicate mode (eps unused for classification; epsClean still applies).
int orc_clip_pair(const double* P, int nP, const double* Q, int nQ, double eps, double epsClean, int flags) {
  g_store.clear();
  Clipper c;
  c.eps = eps; c.epsClean = epsClean; c.uni = flags & 1; c.filters = (flags >> 1) & 1;
  c.exact = (flags >> 2) & 1;
  c.run(P, nP, Q, nQ);
  storeResult(c);
  return c.status;
}

// Clip a batch of layer pairs with the GCMF-GH swap rule (ghcuda.cpp:64-91): the
// polygon with more vertices becomes P, ties keep the base polygon as P.
// Layers use the reference's join layout: interleaved coordinates with the closing
// vertex stored, vnum counts it, vps is the inclusive prefix sum of vnum.
int64_t orc_clip_batch(const double* bxy, const int32_t* bvnum, const int64_t* bvps,
                       const double* oxy, const int32_t* ovnum, const int64_t* ovps,
                       const int32_t* pid, const int32_t* qid, int64_t npairs,
                       double eps, double epsClean, int flags) {
  g_store.clear();
  for (int64_t k = 0; k < npairs; ++k) {
    int b = pid[k], o = qid[k];
    int nb = bvnum[b] - 1, no = ovnum[o] - 1;
    const double* pb = bxy + 2 * (bvps[b] - bvnum[b]);
    const double* po = oxy + 2 * (ovps[o] - ovnum[o]);
    Clipper c;
    c.eps = eps; c.epsClean = epsClean; c.uni = flags & 1; c.filters = (flags >> 1) & 1;
    c.exact = (flags >> 2) & 1;
    if (nb < no) c.run(po, no, pb, nb);
    else c.run(pb, nb, po, no);
    storeResult(c);
  }
  return (int64_t)g_store.status.size();
}

int64_t orc_result_sizes(int64_t* out3) {   // npairs, ncomponents, nvertices
  out3[0] = (int64_t)g_store.status.size();
  out3[1] = (int64_t)g_store.compSize.size();
  out3[2] = (int64_t)g_store.xy.size() / 2;
  return out3[0];
}

void orc_result_copy(int32_t* status, int32_t* ncomp, int64_t* count1, int64_t* nrec,
                     int32_t* compSize, double* xy) {
  if (status) std::copy(g_store.status.begin(), g_store.status.end(), status);
  if (ncomp) std::copy(g_store.ncomp.begin(), g_store.ncomp.end(), ncomp);
  if (count1) std::copy(g_store.count1.begin(), g_store.count1.end(), count1);
  if (nrec) std::copy(g_store.nrec.begin(), g_store.nrec.end(), nrec);
  if (compSize) std::copy(g_store.compSize.begin(), g_store.compSize.end(), compSize);
  if (xy) std::copy(g_store.xy.begin(), g_store.xy.end(), xy);
}

// Multi-component pair: P and Q as interleaved open rings, ring k of sizes[k] vertices,
// P clipped against Q as given.  flags as orc_clip_pair.  Returns the status.
int orc_clip_multi(const double* P, const int32_t* sizesP, int kP, const double* Q, const int32_t* sizesQ, int kQ,
                   double eps, double epsClean, int flags) {
  g_store.clear();
  MultiClipper c;
  c.eps = eps; c.epsClean = epsClean; c.uni = flags & 1; c.filters = (flags >> 1) & 1;
  c.exact = (flags >> 2) & 1;
  c.run(P, sizesP, kP, Q, sizesQ, kQ);
  g_store.status.push_back(c.status);
  g_store.ncomp.push_back((int32_t)c.out.size());
  g_store.count1.push_back(c.count1P);
  g_store.nrec.push_back(c.nrec);
  for (auto& comp : c.out) {
    g_store.compSize.push_back((int32_t)comp.size());
    for (auto& p : comp) { g_store.xy.push_back(p.x); g_store.xy.push_back(p.y); }
  }
  return c.status;
}

static Clipper::Export g_export;
static int32_t g_export_status = 0;

// The reference's calculateIntersections for one pair (GPU-path semantics: CMBR and
// edge-box filters, P/Q count cross-check).  P, Q: open rings; P is not swapped.
// flags bit2: exact-predicate mode.  out3 = merged sizes n_p, n_q and the invalid flag.
// Returns the pair status (0 ok, 1 invalid, 2 disjoint MBRs).
int orc_pair_intersections(const double* P, int nP, const double* Q, int nQ, double eps, int flags,
                           int64_t* out3) {
  Clipper c;
  c.eps = eps; c.epsClean = 0; c.uni = false; c.filters = true; c.exact = (flags >> 2) & 1;
  g_export = Clipper::Export();
  c.ex = &g_export;
  c.run(P, nP, Q, nQ);
  g_export_status = c.status;
  out3[0] = g_export.np;
  out3[1] = g_export.nq;
  out3[2] = c.status == 1 ? 1 : 0;
  return c.status;
}

// arrays of the last orc_pair_intersections (sizes 2 n_p, 2 n_q, then n_p / n_q each);
// nothing is written for an invalid pair
void orc_pair_intersections_copy(double* xyP, double* xyQ, int32_t* alP, int32_t* alQ, int32_t* lbP,
                                 int32_t* lbQ, int32_t* nbP, int32_t* nbQ) {
  if (g_export_status == 1) return;
  const Clipper::Export& e = g_export;
  std::copy(e.xyP.begin(), e.xyP.end(), xyP); std::copy(e.xyQ.begin(), e.xyQ.end(), xyQ);
  std::copy(e.alP.begin(), e.alP.end(), alP); std::copy(e.alQ.begin(), e.alQ.end(), alQ);
  std::copy(e.lbP.begin(), e.lbP.end(), lbP); std::copy(e.lbQ.begin(), e.lbQ.end(), lbQ);
  std::copy(e.nbP.begin(), e.nbP.end(), nbP); std::copy(e.nbQ.begin(), e.nbQ.end(), nbQ);
}

// exact sign of A3(P, Q, R) for n point triples (v: 6 doubles per triple), and of the
// dot product (U1-U0).(V1-V0) when dot != 0 (v: 8 doubles per entry)
void orc_exact_signs(const double* v, int64_t n, int dot, int32_t* out) {
  for (int64_t i = 0; i < n; ++i) {
    if (dot) {
      const double* w = v + 8 * i;
      out[i] = dotExact(Pt{w[0], w[1]}, Pt{w[2], w[3]}, Pt{w[4], w[5]}, Pt{w[6], w[7]});
    } else {
      const double* w = v + 6 * i;
      out[i] = orientExact(w[0], w[1], w[2], w[3], w[4], w[5]);
    }
  }
}

}  // extern "C"

// ======================================================================= join oracle
namespace {

struct LayerView {
  const double* xy; const int32_t* vnum; const int64_t* vps; int64_t n;
  int64_t start(int64_t i) const { return vps[i] - vnum[i]; }    // first vertex index
};

// MBR over every stored vertex (SEQ_Overlay.h:316-344); a polygon whose MBR has zero
// width or height is rejected by the reference reader (":337-344 MBR Error!") and is
// marked invalid here so it never joins.
void mbrOf(const LayerView& L, int64_t i, double* m, uint8_t* valid) {
  int64_t s = L.start(i);
  int nv = L.vnum[i];
  double x1 = L.xy[2 * s], y1 = L.xy[2 * s + 1], x2 = x1, y2 = y1;
  for (int k = 1; k < nv; ++k) {
    double X = L.xy[2 * (s + k)], Y = L.xy[2 * (s + k) + 1];
    if (X < x1) x1 = X;
    if (Y < y1) y1 = Y;
    if (X > x2) x2 = X;
    if (Y > y2) y2 = Y;
  }
  m[0] = x1; m[1] = y1; m[2] = x2; m[3] = y2;
  *valid = (nv >= 2 && x1 != x2 && y1 != y2) ? 1 : 0;
}

inline bool mbrCandidate(const double* b, const double* o) {
  // sort-based sweep acceptance (GPU_MBR.h:339-415) on exact values, see file header
  return o[0] <= b[2] && b[0] <= o[2] && !(o[0] == b[2]) && o[1] <= b[3] && b[1] <= o[3];
}

struct JoinStore {
  std::vector<int32_t> b, o;
  std::vector<double> cmbr;
  std::vector<int8_t> pipType, pipFlag, joinFlag, segFlag, clip;
  std::vector<int32_t> bE, oE;
  std::vector<double> mbrB, mbrO;
  std::vector<uint8_t> validB, validO;
} g_join;

// point-in-polygon crossing parity of (px,py) against the stored ring of polygon i
// (GPU_Join.h:882-915 per edge (i, i-1), parity combined by XOR :920-938).
int pipParity(const LayerView& L, int64_t i, double px, double py) {
  const double* c = L.xy + 2 * L.start(i);
  int n = L.vnum[i];
  int par = 0;
  for (int a = 0; a < n; ++a) {
    int j = (a == 0) ? n - 1 : a - 1;
    double Y1 = c[2 * a + 1], Y2 = c[2 * j + 1], X1 = c[2 * a], X2 = c[2 * j];
    if ((Y1 > py) == (Y2 > py)) continue;
    if (px < (X2 - X1) * (py - Y1) / (Y2 - Y1) + X1) par ^= 1;
  }
  return par;
}

// edges of polygon i whose box touches the common MBR (GPU_Join.h:564-580): edge k
// runs from vertex k to k+1, the last one from the closing vertex back to vertex 0.
void cmfEdges(const LayerView& L, int64_t i, const double* c, std::vector<int>& out) {
  const double* v = L.xy + 2 * L.start(i);
  int n = L.vnum[i];
  out.clear();
  for (int k = 0; k < n; ++k) {
    double x1 = v[2 * k], y1 = v[2 * k + 1];
    int k2 = (k < n - 1) ? k + 1 : 0;
    double x2 = v[2 * k2], y2 = v[2 * k2 + 1];
    if ((c[0] > x1 && c[0] > x2) || (c[2] < x1 && c[2] < x2)) continue;
    if ((c[1] > y1 && c[1] > y2) || (c[3] < y1 && c[3] < y2)) continue;
    out.push_back(k);
  }
}

// any intersecting pair among the surviving edges (GPU_Join.h:369-446)
int segmentsIntersect(const LayerView& B, int64_t bi, const std::vector<int>& bl,
                      const LayerView& O, int64_t oi, const std::vector<int>& ol) {
  const double* bv = B.xy + 2 * B.start(bi);
  const double* ov = O.xy + 2 * O.start(oi);
  int bV = B.vnum[bi], oV = O.vnum[oi];
  for (int be : bl) {
    double bX1 = bv[2 * be], bY1 = bv[2 * be + 1];
    int b2 = (be < bV - 1) ? be + 1 : 0;
    double bX2 = bv[2 * b2], bY2 = bv[2 * b2 + 1];
    if (bX1 == bX2 && bY1 == bY2) continue;
    for (int oe : ol) {
      double oX1 = ov[2 * oe], oY1 = ov[2 * oe + 1];
      int o2 = (oe < oV - 1) ? oe + 1 : 0;
      double oX2 = ov[2 * o2], oY2 = ov[2 * o2 + 1];
      if (((bX2 < oX1) && (bX2 < oX2)) && ((bX1 < oX1) && (bX1 < oX2))) continue;
      if (((bX2 > oX1) && (bX2 > oX2)) && ((bX1 > oX1) && (bX1 > oX2))) continue;
      if (((bY2 < oY1) && (bY2 < oY2)) && ((bY1 < oY1) && (bY1 < oY2))) continue;
      if (((bY2 > oY1) && (bY2 > oY2)) && ((bY1 > oY1) && (bY1 > oY2))) continue;
      double denom = ((bX1 - bX2) * (oY1 - oY2)) - ((bY1 - bY2) * (oX1 - oX2));
      if (denom == 0) {
        if ((oX1 == oX2 && oX1 == bX1) || (bX1 == bX2 && bX1 == oX1)) return 1;
        double oM = (oY2 - oY1) / (oX2 - oX1);
        double bM = (bY2 - bY1) / (bX2 - bX1);
        double oB = oY1 - oM * oX1;
        double bB = bY1 - bM * bX1;
        if (oB == bB) return 1;
        continue;
      }
      double nomX = (((bX1 * bY2) - (bY1 * bX2)) * (oX1 - oX2)) - ((bX1 - bX2) * ((oX1 * oY2) - (oY1 * oX2)));
      double nomY = ((((bX1 * bY2) - (bY1 * bX2)) * (oY1 - oY2)) - (((bY1 - bY2) * ((oX1 * oY2) - (oY1 * oX2)))));
      double x0 = nomX / denom, y0 = nomY / denom;
      if ((x0 > bX1 && x0 > bX2) || (x0 < bX1 && x0 < bX2)) continue;
      if ((x0 > oX1 && x0 > oX2) || (x0 < oX1 && x0 < oX2)) continue;
      if ((y0 > bY1 && y0 > bY2) || (y0 < bY1 && y0 < bY2)) continue;
      if ((y0 > oY1 && y0 > oY2) || (y0 < oY1 && y0 < oY2)) continue;
      return 1;
    }
  }
  return 0;
}

}  // namespace

extern "C" {

void orc_mbr(const double* xy, const int32_t* vnum, const int64_t* vps, int64_t n,
             double* mbr, uint8_t* valid) {
  LayerView L{xy, vnum, vps, n};
  for (int64_t i = 0; i < n; ++i) mbrOf(L, i, mbr + 4 * i, valid + i);
}

// Candidate pairs by testing every (base, overlay) combination: the pin for the
// decomposed search in orc_join.  Writes up to cap pairs, returns the count.
int64_t orc_join_bruteforce(const double* bxy, const int32_t* bvnum, const int64_t* bvps, int64_t nb,
                            const double* oxy, const int32_t* ovnum, const int64_t* ovps, int64_t no,
                            int32_t* outB, int32_t* outO, int64_t cap) {
  LayerView B{bxy, bvnum, bvps, nb}, O{oxy, ovnum, ovps, no};
  std::vector<double> mb(4 * nb), mo(4 * no);
  std::vector<uint8_t> vb(nb), vo(no);
  for (int64_t i = 0; i < nb; ++i) mbrOf(B, i, &mb[4 * i], &vb[i]);
  for (int64_t i = 0; i < no; ++i) mbrOf(O, i, &mo[4 * i], &vo[i]);
  int64_t k = 0;
  for (int64_t i = 0; i < nb; ++i) {
    if (!vb[i]) continue;
    for (int64_t j = 0; j < no; ++j) {
      if (!vo[j] || !mbrCandidate(&mb[4 * i], &mo[4 * j])) continue;
      if (k < cap) { outB[k] = (int32_t)i; outO[k] = (int32_t)j; }
      ++k;
    }
  }
  return k;
}

// The GCMF join: MBR candidates (sorted by base then overlay id), common MBRs,
// containment candidates and test, common-MBR edge filter, segment refine, and the
// clip set = contained pairs + pairs with intersecting edges.  Candidates are found by
// splitting the sweep's two acceptance cases: overlay starts in [x1b, x2b) for each
// base, base starts in (x1o, x2o] for each overlay; the exact predicate then decides.
int64_t orc_join(const double* bxy, const int32_t* bvnum, const int64_t* bvps, int64_t nb,
                 const double* oxy, const int32_t* ovnum, const int64_t* ovps, int64_t no) {
  LayerView B{bxy, bvnum, bvps, nb}, O{oxy, ovnum, ovps, no};
  JoinStore& J = g_join;
  J = JoinStore();
  J.mbrB.resize(4 * nb); J.mbrO.resize(4 * no); J.validB.resize(nb); J.validO.resize(no);
  for (int64_t i = 0; i < nb; ++i) mbrOf(B, i, &J.mbrB[4 * i], &J.validB[i]);
  for (int64_t i = 0; i < no; ++i) mbrOf(O, i, &J.mbrO[4 * i], &J.validO[i]);
  std::vector<int32_t> sb, so;
  for (int64_t i = 0; i < nb; ++i) if (J.validB[i]) sb.push_back((int32_t)i);
  for (int64_t i = 0; i < no; ++i) if (J.validO[i]) so.push_back((int32_t)i);
  auto byX1 = [](const std::vector<double>& m) {
    return [&m](int32_t a, int32_t b) { return m[4 * a] < m[4 * b] || (m[4 * a] == m[4 * b] && a < b); };
  };
  std::sort(sb.begin(), sb.end(), byX1(J.mbrB));
  std::sort(so.begin(), so.end(), byX1(J.mbrO));
  std::vector<double> sbx(sb.size()), sox(so.size());
  for (size_t i = 0; i < sb.size(); ++i) sbx[i] = J.mbrB[4 * sb[i]];
  for (size_t i = 0; i < so.size(); ++i) sox[i] = J.mbrO[4 * so[i]];
  std::vector<std::pair<int32_t, int32_t>> pairs;
  for (int32_t b : sb) {
    const double* mb = &J.mbrB[4 * b];
    size_t lo = std::lower_bound(sox.begin(), sox.end(), mb[0]) - sox.begin();
    size_t hi = std::lower_bound(sox.begin(), sox.end(), mb[2]) - sox.begin();
    for (size_t k = lo; k < hi; ++k)
      if (mbrCandidate(mb, &J.mbrO[4 * so[k]])) pairs.push_back({b, so[k]});
  }
  for (int32_t o : so) {
    const double* mo = &J.mbrO[4 * o];
    size_t lo = std::upper_bound(sbx.begin(), sbx.end(), mo[0]) - sbx.begin();
    size_t hi = std::upper_bound(sbx.begin(), sbx.end(), mo[2]) - sbx.begin();
    for (size_t k = lo; k < hi; ++k)
      if (mbrCandidate(&J.mbrB[4 * sb[k]], mo)) pairs.push_back({sb[k], o});
  }
  std::sort(pairs.begin(), pairs.end());
  int64_t K = (int64_t)pairs.size();
  J.b.resize(K); J.o.resize(K); J.cmbr.resize(4 * K); J.pipType.resize(K); J.pipFlag.resize(K);
  J.joinFlag.resize(K); J.segFlag.resize(K); J.clip.resize(K); J.bE.resize(K); J.oE.resize(K);
  std::vector<int> bl, ol;
  for (int64_t k = 0; k < K; ++k) {
    int32_t b = pairs[k].first, o = pairs[k].second;
    J.b[k] = b; J.o[k] = o;
    const double* m1 = &J.mbrB[4 * b];
    const double* m2 = &J.mbrO[4 * o];
    double* c = &J.cmbr[4 * k];
    // GPU_Join.h:475-506
    double x1 = m1[0], x2 = m1[2], y1 = m1[1], y2 = m1[3];
    double a1 = m2[0], a2 = m2[2], b1 = m2[1], b2 = m2[3];
    c[0] = (a1 > x1 ? a1 : x1);
    c[2] = (a2 < x2 ? a2 : x2);
    c[1] = (b1 > y1 ? b1 : y1);
    c[3] = (b2 < y2 ? b2 : y2);
    int type = 0;
    if (x1 == c[0] && x2 == c[2] && y1 == c[1] && y2 == c[3]) type = 1;
    else if (a1 == c[0] && a2 == c[2] && b1 == c[1] && b2 == c[3]) type = 2;
    J.pipType[k] = (int8_t)type;
    int join = 1, pip = 0;
    if (type == 1) {
      const double* p = B.xy + 2 * B.start(b);
      pip = pipParity(O, o, p[0], p[1]);
    } else if (type == 2) {
      const double* p = O.xy + 2 * O.start(o);
      pip = pipParity(B, b, p[0], p[1]);
    }
    if (pip) join = 0;
    J.pipFlag[k] = (int8_t)pip;
    int seg = 0;
    J.bE[k] = 0; J.oE[k] = 0;
    if (join) {
      cmfEdges(B, b, c, bl);
      cmfEdges(O, o, c, ol);
      if (bl.empty() || ol.empty()) join = 0;
      else { J.bE[k] = (int32_t)bl.size(); J.oE[k] = (int32_t)ol.size(); }
      if (join) seg = segmentsIntersect(B, b, bl, O, o, ol);
    }
    J.joinFlag[k] = (int8_t)join;
    J.segFlag[k] = (int8_t)seg;
    J.clip[k] = (int8_t)(pip || seg);
  }
  return K;
}

// Copies the last orc_join result; any pointer may be null.
void orc_join_copy(int32_t* b, int32_t* o, double* cmbr, int8_t* pipType, int8_t* pipFlag,
                   int8_t* joinFlag, int32_t* bE, int32_t* oE, int8_t* segFlag, int8_t* clip,
                   double* mbrB, uint8_t* validB, double* mbrO, uint8_t* validO) {
  JoinStore& J = g_join;
  if (b) std::copy(J.b.begin(), J.b.end(), b);
  if (o) std::copy(J.o.begin(), J.o.end(), o);
  if (cmbr) std::copy(J.cmbr.begin(), J.cmbr.end(), cmbr);
  if (pipType) std::copy(J.pipType.begin(), J.pipType.end(), pipType);
  if (pipFlag) std::copy(J.pipFlag.begin(), J.pipFlag.end(), pipFlag);
  if (joinFlag) std::copy(J.joinFlag.begin(), J.joinFlag.end(), joinFlag);
  if (bE) std::copy(J.bE.begin(), J.bE.end(), bE);
  if (oE) std::copy(J.oE.begin(), J.oE.end(), oE);
  if (segFlag) std::copy(J.segFlag.begin(), J.segFlag.end(), segFlag);
  if (clip) std::copy(J.clip.begin(), J.clip.end(), clip);
  if (mbrB) std::copy(J.mbrB.begin(), J.mbrB.end(), mbrB);
  if (validB) std::copy(J.validB.begin(), J.validB.end(), validB);
  if (mbrO) std::copy(J.mbrO.begin(), J.mbrO.end(), mbrO);
  if (validO) std::copy(J.validO.begin(), J.validO.end(), validO);
}

}  // extern "C"
