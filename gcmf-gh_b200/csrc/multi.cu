// multi.cu -- pairs of multi-component polygons: outer rings and holes, even-odd.
//
// The reference's CPU clipper takes P and Q as lists of components and loops over them in
// every phase (GH-CUDA/lib/polyclip.h): intersections over all component pairs
// (:202-268), step-1 labels and chains per component, special cases per component with
// the inside test's parity over all components of the other polygon and the hole test for
// identical components (:474-541), entry/exit per component (:549-655), split pairs and
// crossing candidates over all components (:661-734), tracing from every component of P
// (:743-783) and the clean-up (:791-807).  Its GPU intersection phase has no
// multi-component form (calculateIntersectionsMultipleComponents, GH-CUDA/ghcuda.h:15, is
// declared and never defined).
//
// Here the intersection records come from the batched clip stages G0-G3 run over every
// (P ring, Q ring) pair, so each ring pair gets the GPU path's common-MBR edge filter,
// edge-box test and P/Q count check (a failing ring pair makes the pair invalid).  One
// thread then builds the component rings, links them, labels them and traces the result:
// this path is for the occasional polygon with holes, and the phases after the
// intersections are a chain of dependent steps over linked lists.
#include <algorithm>
#include <cstring>
#include <vector>
#include "common.cuh"
#include "engine.cuh"
#include "prims.cuh"

namespace gcmfgh {

namespace {

// vertices of one side: all components in one slot array, each component a cycle
struct MRing {
  double* x; double* y;
  int32_t* nx; int32_t* pv; int32_t* nb;
  uint8_t* it; int8_t* lb; int8_t* ee;
  int used, cap;
};

struct MultiArgs {
  const double2* P; const double2* Q;        // layer vertices (closing vertex stored)
  const int64_t* startP; const int64_t* startQ;   // first layer vertex of each ring
  const int32_t* sizeP; const int32_t* sizeQ;     // open-ring sizes
  const int64_t* edgeP; const int64_t* edgeQ;     // first global edge of each ring (k + 1 entries)
  int kP, kQ;
  // intersection records of the ring pairs (pair k = i * kQ + j)
  const int32_t* rp; const int32_t* rq; const double* ra; const double* rb; const int8_t* rt;
  const int32_t* rk;                         // ring pair of each record (absolute; k0 is this pair's first)
  int64_t nR, k0;
  const int32_t* pairStatus; int64_t nPairs;
  // work arrays
  int32_t* cntP; int32_t* cntQ;              // per global edge (+1): insertion counts, then offsets
  int32_t* lstP; int32_t* lstQ;              // per edge, its inserting records
  int32_t* srcP; int32_t* srcQ;              // per global edge: slot of its source vertex
  int32_t* insP; int32_t* insQ;              // per record: its inserted slot on P / Q (-1 none)
  long long* winP; long long* winQ;          // per global edge: key of the source vertex's link
  MRing R[2];
  int32_t* root[2];                          // per component: root slot
  uint8_t* noInter[2]; uint8_t* ident[2];
  int32_t* split[2]; int32_t* cand[2];
  uint8_t* mark;                             // per Q slot
  // result
  double* oxy; int64_t vcap; int32_t* ocs; int ccap;
  int32_t* onx; int32_t* opv;                // clean-up scratch, vcap each
  double* otmp;                              // clean-up scratch, 2 vcap
  int32_t* status; int32_t* outNC; int64_t* outNV;
  double epsClean; int uni; int exact;
  int* err;
};

// the record's ring pair within this polygon pair, i * kQ + j
__device__ __forceinline__ int m_k(const MultiArgs& a, int64_t r) { return (int)(a.rk[r] - a.k0); }

__device__ int m_add(MRing& R, double X, double Y) {
  if (R.used >= R.cap) return -1;
  const int v = R.used++;
  R.x[v] = X; R.y[v] = Y; R.nx[v] = v; R.pv[v] = v; R.nb[v] = -1;
  R.it[v] = 0; R.lb[v] = L_NONE; R.ee[v] = E_NEITHER;
  return v;
}

__device__ void m_insert_after(MRing& R, int v, int after) {
  const int c = R.nx[after];
  R.nx[R.pv[c]] = v; R.pv[v] = R.pv[c]; R.nx[v] = c; R.pv[c] = v;
}

__device__ void m_link(MRing& A, int i, MRing& B, int j) {
  A.nb[i] = j; B.nb[j] = i; A.it[i] = 1; B.it[j] = 1;
}

// winding-number parity of (Rx, Ry) in one component (polygon.h:427-448)
__device__ bool m_point_in(const MRing& R, int root, double Rx, double Ry, int ex) {
  int w = 0, one = root;
  do {
    const int two = R.nx[one];
    const double P0x = R.x[one], P0y = R.y[one], P1x = R.x[two], P1y = R.y[two];
    if ((P0y < Ry) != (P1y < Ry)) {
      if (P0x >= Rx) {
        if (P1x > Rx) w = w + 2 * (P1y > P0y) - 1;
        else if ((orient_sign(ex, P0x, P0y, P1x, P1y, Rx, Ry) > 0) == (P1y > P0y)) w = w + 2 * (P1y > P0y) - 1;
      } else if (P1x > Rx) {
        if ((orient_sign(ex, P0x, P0y, P1x, P1y, Rx, Ry) > 0) == (P1y > P0y)) w = w + 2 * (P1y > P0y) - 1;
      }
    }
    one = two;
  } while (one != root);
  return (w % 2) != 0;
}

// parity of (Rx, Ry) over every component of a side, skipping the one rooted at `skip`
__device__ bool m_inside(const MRing& R, const int32_t* roots, int k, double Rx, double Ry, int ex, int skip = -1) {
  bool in = false;
  for (int c = 0; c < k; ++c)
    if (roots[c] != skip && m_point_in(R, roots[c], Rx, Ry, ex)) in = !in;
  return in;
}

// polyclip.h:297-326
__device__ int m_rel(const MultiArgs& a, int qv, int p1, int p2, int p3) {
  const MRing& P = a.R[0];
  const MRing& Q = a.R[1];
  if (P.it[p1] && P.nb[p1] == qv) return R_IS_P_M;
  if (P.it[p3] && P.nb[p3] == qv) return R_IS_P_P;
  const int s1 = orient_sign(a.exact, Q.x[qv], Q.y[qv], P.x[p1], P.y[p1], P.x[p2], P.y[p2]);
  const int s2 = orient_sign(a.exact, Q.x[qv], Q.y[qv], P.x[p2], P.y[p2], P.x[p3], P.y[p3]);
  const int s3 = orient_sign(a.exact, P.x[p1], P.y[p1], P.x[p2], P.y[p2], P.x[p3], P.y[p3]);
  if (s3 > 0) return (s1 > 0 && s2 > 0) ? R_LEFT : R_RIGHT;
  return (s1 < 0 && s2 < 0) ? R_RIGHT : R_LEFT;
}

// gppolyclip_mDIV512.cu:237-252
__device__ int8_t m_initial_label(int m, int p) {
  auto is = [&](int x, int y) { return (m == x && p == y) || (m == y && p == x); };
  if (is(R_LEFT, R_RIGHT)) return L_CROSSING;
  if ((m == R_LEFT && p == R_LEFT) || (m == R_RIGHT && p == R_RIGHT)) return L_BOUNCING;
  if (is(R_IS_P_P, R_RIGHT)) return L_LEFT_ON;
  if (is(R_IS_P_P, R_LEFT)) return L_RIGHT_ON;
  if (is(R_IS_P_P, R_IS_P_M)) return L_ON_ON;
  if (is(R_IS_P_M, R_RIGHT)) return L_ON_LEFT;
  if (is(R_IS_P_M, R_LEFT)) return L_ON_RIGHT;
  return L_NONE;
}

__device__ bool m_no_crossing(const MRing& R, int root, int uni) {     // polygon.h:465-475
  int v = root;
  do {
    if (R.it[v]) {
      if (R.lb[v] == L_CROSSING || R.lb[v] == L_DELAYED_CROSSING) return false;
      if (uni && (R.lb[v] == L_BOUNCING || R.lb[v] == L_DELAYED_BOUNCING)) return false;
    }
    v = R.nx[v];
  } while (v != root);
  return true;
}

__device__ bool m_all_on_on(const MRing& R, int root) {                // polygon.h:453-458
  int v = root;
  do { if (R.lb[v] != L_ON_ON) return false; v = R.nx[v]; } while (v != root);
  return true;
}

// polygon.h:480-491
__device__ void m_non_inter_point(const MRing& R, int root, const MRing& O, double& px, double& py) {
  int v = root;
  do { if (!R.it[v]) { px = R.x[v]; py = R.y[v]; return; } v = R.nx[v]; } while (v != root);
  v = root;
  do {
    const int nb = R.nb[v], nx = R.nx[v];
    if (nb >= 0 && R.nb[nx] != O.pv[nb] && R.nb[nx] != O.nx[nb]) {
      px = 0.5 * (R.x[v] + R.x[nx]); py = 0.5 * (R.y[v] + R.y[nx]); return;
    }
    v = R.nx[v];
  } while (v != root);
  px = py = 0.0;
}

// polygon.h:496-512 (may add a temporary midpoint vertex); -1 if none, -2 when full
__device__ int m_non_inter_vertex(MRing& R, int root, const MRing& O) {
  int v = root;
  do { if (!R.it[v]) return v; v = R.nx[v]; } while (v != root);
  v = root;
  do {
    const int nb = R.nb[v], nx = R.nx[v];
    if (nb >= 0 && R.nb[nx] != O.pv[nb] && R.nb[nx] != O.nx[nb]) {
      const int t = m_add(R, 0.5 * (R.x[v] + R.x[nx]), 0.5 * (R.y[v] + R.y[nx]));
      if (t < 0) return -2;
      m_insert_after(R, t, v);
      return t;
    }
    v = R.nx[v];
  } while (v != root);
  return -1;
}

// the intersection vertices of start's component in ring order from start (vertexIterator
// with INTERSECTION, polygon.h:194-264); f returns false to stop with an error.  The walk
// is bounded by guard; returns false when f failed or the guard ran out
template <class F>
__device__ bool m_for_inter(const MRing& R, int start, long long& guard, F f) {
  int V = start;
  if (!R.it[V]) {
    do { V = R.nx[V]; if (--guard < 0) return false; } while (!R.it[V] && V != start);
    if (V == start) return true;
  }
  for (;;) {
    if (!f(V)) return false;
    do { V = R.nx[V]; if (--guard < 0) return false; } while (!R.it[V] && V != start);
    if (V == start) return true;
  }
}

struct MOut {
  double* xy; int32_t* csz; int64_t vcap; int ccap;
  int64_t nv; int nc; bool overflow;
  __device__ void begin() { if (nc >= ccap) overflow = true; else csz[nc] = 0; }
  __device__ void push(double X, double Y) {
    if (overflow || nv >= vcap) { overflow = true; return; }
    xy[2 * nv] = X; xy[2 * nv + 1] = Y; ++nv; ++csz[nc];
  }
  __device__ void end() { if (!overflow) ++nc; }
};

__device__ void m_push_component(MOut& o, const MRing& R, int root) {
  o.begin();
  int v = root;
  do { o.push(R.x[v], R.y[v]); v = R.nx[v]; } while (v != root);
  o.end();
}

__device__ void m_fail(const MultiArgs& a, int code) {
  raise_error(a.err, code);
  *a.status = 3;
  *a.outNC = 0;
  *a.outNV = 0;
}

// record order key for ties: (other component, other edge), larger = inserted later
__device__ __forceinline__ long long m_other_key(const MultiArgs& a, int64_t r, int side) {
  const int k = m_k(a, r);
  return side == 0 ? ((long long)(k % a.kQ) << 32) | (uint32_t)a.rq[r]
                   : ((long long)(k / a.kQ) << 32) | (uint32_t)a.rp[r];
}

__device__ void multi_clip_pair(MultiArgs& a) {
  *a.outNC = 0;
  *a.outNV = 0;
  *a.status = 0;
  for (int64_t k = 0; k < a.nPairs; ++k)
    if (a.pairStatus[k] == 1) { *a.status = 1; return; }           // P/Q counts differ
  MRing& RP = a.R[0];
  MRing& RQ = a.R[1];
  const int64_t EP = a.edgeP[a.kP], EQ = a.edgeQ[a.kQ];
  // ---- records inserting on each global edge, then sorted: ascending parameter, equal
  // parameters with the later-inserted record first (insertVertex, polygon.h:101-113)
  for (int64_t e = 0; e <= EP; ++e) a.cntP[e] = 0;
  for (int64_t e = 0; e <= EQ; ++e) a.cntQ[e] = 0;
  for (int64_t r = 0; r < a.nR; ++r) {
    const int t = a.rt[r], k = m_k(a, r), i = k / a.kQ, j = k % a.kQ;
    a.insP[r] = a.insQ[r] = -1;
    if (t == 1 || t == 3 || t == 5 || t == 7) a.cntP[a.edgeP[i] + a.rp[r] + 1]++;
    if (t == 1 || t == 2 || t == 5 || t == 6) a.cntQ[a.edgeQ[j] + a.rq[r] + 1]++;
  }
  for (int64_t e = 0; e < EP; ++e) a.cntP[e + 1] += a.cntP[e];
  for (int64_t e = 0; e < EQ; ++e) a.cntQ[e + 1] += a.cntQ[e];
  for (int64_t r = 0; r < a.nR; ++r) {                          // counts become cursors
    const int t = a.rt[r], k = m_k(a, r), i = k / a.kQ, j = k % a.kQ;
    if (t == 1 || t == 3 || t == 5 || t == 7) a.lstP[a.cntP[a.edgeP[i] + a.rp[r]]++] = (int32_t)r;
    if (t == 1 || t == 2 || t == 5 || t == 6) a.lstQ[a.cntQ[a.edgeQ[j] + a.rq[r]]++] = (int32_t)r;
  }
  for (int64_t e = EP; e > 0; --e) a.cntP[e] = a.cntP[e - 1];   // back to offsets
  for (int64_t e = EQ; e > 0; --e) a.cntQ[e] = a.cntQ[e - 1];
  a.cntP[0] = a.cntQ[0] = 0;
  for (int side = 0; side < 2; ++side) {
    const int64_t E = side == 0 ? EP : EQ;
    const int32_t* off = side == 0 ? a.cntP : a.cntQ;
    int32_t* lst = side == 0 ? a.lstP : a.lstQ;
    const double* key = side == 0 ? a.ra : a.rb;
    for (int64_t e = 0; e < E; ++e)
      for (int x = off[e] + 1; x < off[e + 1]; ++x) {
        const int32_t r = lst[x];
        const double kr = key[r];
        const long long or_ = m_other_key(a, r, side);
        int y = x - 1;
        while (y >= off[e]) {
          const int32_t s = lst[y];
          if (!(key[s] > kr || (key[s] == kr && m_other_key(a, s, side) < or_))) break;
          lst[y + 1] = s;
          --y;
        }
        lst[y + 1] = r;
      }
  }
  // ---- component rings: each ring's source vertices with their inserted vertices
  RP.used = RQ.used = 0;
  for (int side = 0; side < 2; ++side) {
    MRing& Rg = a.R[side];
    const int kc = side == 0 ? a.kP : a.kQ;
    for (int c = 0; c < kc; ++c) {
      const int first = Rg.used;
      a.root[side][c] = first;
      const int n = side == 0 ? a.sizeP[c] : a.sizeQ[c];
      const int64_t ge0 = side == 0 ? a.edgeP[c] : a.edgeQ[c];
      const double2* V = (side == 0 ? a.P + a.startP[c] : a.Q + a.startQ[c]);
      for (int e = 0; e < n; ++e) {
        const double2 A = V[e];
        const int sv = m_add(Rg, A.x, A.y);
        if (sv < 0) { m_fail(a, DEV_CAPACITY); return; }
        (side == 0 ? a.srcP : a.srcQ)[ge0 + e] = sv;
        const int32_t* off = side == 0 ? a.cntP : a.cntQ;
        const int32_t* lst = side == 0 ? a.lstP : a.lstQ;
        for (int x = off[ge0 + e]; x < off[ge0 + e + 1]; ++x) {
          const int32_t r = lst[x];
          double X, Y;
          if (side == 0) {
            if (a.rt[r] == 1) {                                  // (1-alpha) P1 + alpha P2
              const double2 P2 = V[e + 1 < n ? e + 1 : 0];
              X = (1.0 - a.ra[r]) * A.x + a.ra[r] * P2.x;
              Y = (1.0 - a.ra[r]) * A.y + a.ra[r] * P2.y;
            } else {                                             // a copy of Q1
              const int j = m_k(a, r) % a.kQ;
              const double2 Q1 = a.Q[a.startQ[j] + a.rq[r]];
              X = Q1.x; Y = Q1.y;
            }
          } else {
            if (a.rt[r] == 1) {                                  // the P-side point
              X = RP.x[a.insP[r]]; Y = RP.y[a.insP[r]];
            } else {                                             // a copy of P1
              const int i = m_k(a, r) / a.kQ;
              const double2 P1 = a.P[a.startP[i] + a.rp[r]];
              X = P1.x; Y = P1.y;
            }
          }
          const int v = m_add(Rg, X, Y);
          if (v < 0) { m_fail(a, DEV_CAPACITY); return; }
          (side == 0 ? a.insP : a.insQ)[r] = v;
        }
      }
      const int last = Rg.used;
      for (int v = first; v < last; ++v) { Rg.nx[v] = v + 1 < last ? v + 1 : first; Rg.pv[v] = v > first ? v - 1 : last - 1; }
    }
  }
  // ---- links (polyclip.h:215-267): a source vertex keeps the link of its last record in
  // the reference's loop order (P component, P edge, Q component, Q edge)
  for (int64_t e = 0; e < EP; ++e) a.winP[e] = -1;
  for (int64_t e = 0; e < EQ; ++e) a.winQ[e] = -1;
  for (int64_t r = 0; r < a.nR; ++r) {
    const int t = a.rt[r], k = m_k(a, r), i = k / a.kQ, j = k % a.kQ;
    const long long kp = m_other_key(a, r, 0), kq = m_other_key(a, r, 1);
    if (t == 2 || t == 4 || t == 5 || t == 6 || t == 8) {
      long long& w = a.winP[a.edgeP[i] + a.rp[r]];
      if (kp > w) w = kp;
    }
    if (t == 3 || t == 4 || t == 5 || t == 7 || t == 8) {
      long long& w = a.winQ[a.edgeQ[j] + a.rq[r]];
      if (kq > w) w = kq;
    }
  }
  for (int64_t r = 0; r < a.nR; ++r) {
    const int t = a.rt[r], k = m_k(a, r), i = k / a.kQ, j = k % a.kQ;
    const int64_t eP = a.edgeP[i] + a.rp[r], eQ = a.edgeQ[j] + a.rq[r];
    const int sp = a.srcP[eP], sq = a.srcQ[eQ];
    const bool wP = a.winP[eP] == m_other_key(a, r, 0), wQ = a.winQ[eQ] == m_other_key(a, r, 1);
    switch (t) {
      case 1: m_link(RP, a.insP[r], RQ, a.insQ[r]); break;
      case 2: case 6:
        RQ.nb[a.insQ[r]] = sp; RQ.it[a.insQ[r]] = 1; RP.it[sp] = 1;
        if (wP) RP.nb[sp] = a.insQ[r];
        break;
      case 3: case 7:
        RP.nb[a.insP[r]] = sq; RP.it[a.insP[r]] = 1; RQ.it[sq] = 1;
        if (wQ) RQ.nb[sq] = a.insP[r];
        break;
      case 4: case 8:
        RP.it[sp] = 1; RQ.it[sq] = 1;
        if (wP) RP.nb[sp] = sq;
        if (wQ) RQ.nb[sq] = sp;
        break;
      case 5:
        RQ.nb[a.insQ[r]] = sp; RQ.it[a.insQ[r]] = 1; RP.it[sp] = 1;
        if (wP) RP.nb[sp] = a.insQ[r];
        RP.nb[a.insP[r]] = sq; RP.it[a.insP[r]] = 1; RQ.it[sq] = 1;
        if (wQ) RQ.nb[sq] = a.insP[r];
        break;
    }
  }
  // ---- step 1 and step 2 per component of P (polyclip.h:343-451)
  long long guard = 16LL * ((long long)RP.cap + RQ.cap) + 64;
  for (int c = 0; c < a.kP; ++c) {
    if (!m_for_inter(RP, a.root[0][c], guard, [&](int I) {
          const int nb = RP.nb[I];
          if (nb < 0) return true;
          const int8_t L = m_initial_label(m_rel(a, RQ.pv[nb], RP.pv[I], I, RP.nx[I]),
                                           m_rel(a, RQ.nx[nb], RP.pv[I], I, RP.nx[I]));
          if (L != L_NONE) { RP.lb[I] = L; RQ.lb[nb] = L; }
          return true;
        })) { m_fail(a, DEV_TRACE); return; }
  }
  for (int c = 0; c < a.kP; ++c) {
    if (!m_for_inter(RP, a.root[0][c], guard, [&](int I0) {
          if (RP.lb[I0] != L_LEFT_ON && RP.lb[I0] != L_RIGHT_ON) return true;
          const int x = RP.lb[I0] == L_LEFT_ON ? R_LEFT : R_RIGHT;
          int X = I0, I = I0;
          do {
            if (--guard < 0 || RP.nb[I] < 0) return false;
            RP.lb[I] = L_NONE;
            RQ.lb[RP.nb[I]] = L_NONE;
            I = RP.nx[I];
          } while (RP.lb[I] == L_ON_ON);
          if (RP.nb[I] < 0) return false;
          const int y = RP.lb[I] == L_ON_LEFT ? R_LEFT : R_RIGHT;
          const int8_t ct = (x != y) ? L_DELAYED_CROSSING : L_DELAYED_BOUNCING;
          RP.lb[X] = ct; RP.lb[I] = ct;
          RQ.lb[RP.nb[X]] = ct; RQ.lb[RP.nb[I]] = ct;
          return true;
        })) { m_fail(a, DEV_TRACE); return; }
  }
  MOut o{a.oxy, a.ocs, a.vcap, a.ccap, 0, 0, false};
  // ---- step 3.5: components without crossing vertices (polyclip.h:474-541)
  for (int sd = 0; sd < 2; ++sd) {
    const MRing& A = a.R[sd];
    const MRing& B = a.R[1 - sd];
    const int kc = sd == 0 ? a.kP : a.kQ, kb = sd == 0 ? a.kQ : a.kP;
    for (int c = 0; c < kc; ++c) {
      const int root = a.root[sd][c];
      a.noInter[sd][c] = 0;
      a.ident[sd][c] = 0;
      if (!m_no_crossing(A, root, a.uni)) continue;
      a.noInter[sd][c] = 1;
      if (m_all_on_on(A, root)) { a.ident[sd][c] = 1; continue; }
      double px, py;
      m_non_inter_point(A, root, B, px, py);
      if (m_inside(B, a.root[1 - sd], kb, px, py, a.exact) ^ (a.uni != 0)) m_push_component(o, A, root);
    }
  }
  for (int c = 0; c < a.kP; ++c) {                       // identical components
    if (!a.ident[0][c]) continue;
    const int pr = a.root[0][c];
    const bool pHole = m_inside(RP, a.root[0], a.kP, RP.x[pr], RP.y[pr], a.exact, pr);
    for (int d = 0; d < a.kQ; ++d) {
      if (!a.ident[1][d]) continue;
      const int qr = a.root[1][d];
      bool match = false;
      int v = qr;
      do { if (v == RP.nb[pr]) { match = true; break; } v = RQ.nx[v]; } while (v != qr);
      if (!match) continue;
      const bool qHole = m_inside(RQ, a.root[1], a.kQ, RQ.x[qr], RQ.y[qr], a.exact, qr);
      if (pHole == qHole) m_push_component(o, RP, pr);
      break;
    }
  }
  // ---- step 4: entry/exit per component (polyclip.h:549-655)
  int nSplit[2] = {0, 0}, nCand[2] = {0, 0};
  for (int sd = 0; sd < 2; ++sd) {
    MRing& A = a.R[sd];
    const MRing& B = a.R[1 - sd];
    const int kc = sd == 0 ? a.kP : a.kQ, kb = sd == 0 ? a.kQ : a.kP;
    for (int c = 0; c < kc; ++c) {
      if (a.noInter[sd][c]) continue;
      const int V = m_non_inter_vertex(A, a.root[sd][c], B);
      if (V == -2) { m_fail(a, DEV_CAPACITY); return; }
      if (V < 0) continue;
      int8_t st = m_inside(B, a.root[1 - sd], kb, A.x[V], A.y[V], a.exact) ? E_EXIT : E_ENTRY;
      bool first = true;
      const bool uni = a.uni != 0;
      auto toggle = [&]() { st = (st == E_ENTRY) ? E_EXIT : E_ENTRY; };
      if (!m_for_inter(A, V, guard, [&](int I) {
            if (A.lb[I] == L_CROSSING) { A.ee[I] = st; toggle(); }
            if (A.lb[I] == L_BOUNCING && ((st == E_EXIT) ^ uni)) a.split[sd][nSplit[sd]++] = I;
            if (A.lb[I] == L_DELAYED_CROSSING) {
              A.ee[I] = st;
              if (first) { if ((st == E_EXIT) ^ uni) A.lb[I] = L_CROSSING; first = false; }
              else { if ((st == E_ENTRY) ^ uni) A.lb[I] = L_CROSSING; first = true; toggle(); }
            }
            if (A.lb[I] == L_DELAYED_BOUNCING) {
              A.ee[I] = st;
              if (first) { if ((st == E_EXIT) ^ uni) a.cand[sd][nCand[sd]++] = I; first = false; }
              else { if ((st == E_ENTRY) ^ uni) a.cand[sd][nCand[sd]++] = I; first = true; }
              toggle();
            }
            return true;
          })) { m_fail(a, DEV_TRACE); return; }
    }
  }
  // ---- step 5: split vertex pairs (polyclip.h:661-714), in the order P's components found them
  for (int v = 0; v < RQ.used; ++v) a.mark[v] = 0;
  for (int x = 0; x < nSplit[1]; ++x) a.mark[a.split[1][x]] = 1;
  for (int x = 0; x < nSplit[0]; ++x) {
    const int IP = a.split[0][x];
    const int IQ = RP.nb[IP];
    if (IQ < 0 || IQ >= RQ.used || !a.mark[IQ]) continue;
    const int VP = m_add(RP, RP.x[IP], RP.y[IP]);
    const int VQ = m_add(RQ, RQ.x[IQ], RQ.y[IQ]);
    if (VP < 0 || VQ < 0) { m_fail(a, DEV_CAPACITY); return; }
    bool same;
    if (a.exact) {
      same = orient_sign(1, RP.x[RP.pv[IP]], RP.y[RP.pv[IP]], RP.x[IP], RP.y[IP], RP.x[RP.nx[IP]], RP.y[RP.nx[IP]]) *
             orient_sign(1, RQ.x[RQ.pv[IQ]], RQ.y[RQ.pv[IQ]], RQ.x[IQ], RQ.y[IQ], RQ.x[RQ.nx[IQ]], RQ.y[RQ.nx[IQ]]) > 0;
    } else {
      const double sP = area2(RP.x[RP.pv[IP]], RP.y[RP.pv[IP]], RP.x[IP], RP.y[IP], RP.x[RP.nx[IP]], RP.y[RP.nx[IP]]);
      const double sQ = area2(RQ.x[RQ.pv[IQ]], RQ.y[RQ.pv[IQ]], RQ.x[IQ], RQ.y[IQ], RQ.x[RQ.nx[IQ]], RQ.y[RQ.nx[IQ]]);
      same = sP * sQ > 0;
    }
    if (same) { m_link(RP, IP, RQ, VQ); m_link(RP, VP, RQ, IQ); }
    else m_link(RP, VP, RQ, VQ);
    m_insert_after(RP, VP, IP);
    m_insert_after(RQ, VQ, IQ);
    const int8_t e1 = a.uni ? E_ENTRY : E_EXIT, e2 = a.uni ? E_EXIT : E_ENTRY;
    RP.ee[IP] = e1; RP.ee[VP] = e2; RQ.ee[IQ] = e1; RQ.ee[VQ] = e2;
    RP.lb[IP] = L_CROSSING; RP.lb[VP] = L_CROSSING; RQ.lb[IQ] = L_CROSSING; RQ.lb[VQ] = L_CROSSING;
  }
  // ---- step 6: crossing candidates (polyclip.h:723-734)
  for (int v = 0; v < RQ.used; ++v) a.mark[v] = 0;
  for (int x = 0; x < nCand[1]; ++x) a.mark[a.cand[1][x]] = 1;
  for (int x = 0; x < nCand[0]; ++x) {
    const int IP = a.cand[0][x];
    const int IQ = RP.nb[IP];
    if (IQ >= 0 && IQ < RQ.used && a.mark[IQ]) { RP.lb[IP] = L_CROSSING; RQ.lb[IQ] = L_CROSSING; }
  }
  // ---- tracing from every component of P (polyclip.h:743-783)
  long long budget = 4LL * (RP.used + RQ.used) + 16;
  for (int c = 0; c < a.kP; ++c) {
    const int V0 = a.root[0][c];
    auto isStart = [&](int v) { return RP.it[v] && RP.lb[v] == L_CROSSING; };
    int I = V0;
    bool have = isStart(I);
    if (!have) {
      do { I = RP.nx[I]; } while (!isStart(I) && I != V0);
      have = (I != V0);
    }
    while (have) {
      o.begin();
      int sd = 0, V = I;
      RP.it[V] = 0;
      do {
        if (--budget < 0) { m_fail(a, DEV_TRACE); return; }
        MRing& cur = a.R[sd];
        int8_t st = cur.ee[V];
        st = (st == E_ENTRY) ? E_EXIT : (st == E_EXIT ? E_ENTRY : st);
        do {
          if (--budget < 0) { m_fail(a, DEV_TRACE); return; }
          V = ((st == E_EXIT) ^ (a.uni != 0)) ? cur.nx[V] : cur.pv[V];
          cur.it[V] = 0;
          o.push(cur.x[V], cur.y[V]);
        } while (!(cur.ee[V] == st) && !(sd == 0 && V == I));
        if (!(sd == 0 && V == I)) {
          if (cur.nb[V] < 0) { m_fail(a, DEV_TRACE); return; }
          V = cur.nb[V];
          sd = 1 - sd;
          a.R[sd].it[V] = 0;
        }
      } while (!(sd == 0 && V == I));
      o.end();
      do { I = RP.nx[I]; } while (!isStart(I) && I != V0);
      have = (I != V0);
    }
  }
  if (o.overflow) { m_fail(a, DEV_CAPACITY); return; }
  // ---- clean-up (polyclip.h:791-807), component by component, compacted in place
  int64_t w = 0, rd = 0;
  int nc = 0;
  for (int c = 0; c < o.nc; ++c) {
    const int m = a.ocs[c];
    const int64_t base = rd;
    rd += m;
    if (m == 0) continue;
    for (int i = 0; i < m; ++i) { a.onx[i] = (i + 1) % m; a.opv[i] = (i + m - 1) % m; }
    const double* X = a.oxy + 2 * base;
    auto area = [&](int v) {
      return fabs(area2(X[2 * a.opv[v]], X[2 * a.opv[v] + 1], X[2 * v], X[2 * v + 1], X[2 * a.onx[v]],
                        X[2 * a.onx[v] + 1]));
    };
    int root = 0;
    auto remove = [&](int v) {
      if (root == v) { root = a.onx[v]; if (a.onx[root] == root) root = -1; }
      a.onx[a.opv[v]] = a.onx[v]; a.opv[a.onx[v]] = a.opv[v];
    };
    while (root >= 0 && area(root) < a.epsClean) remove(root);
    if (root >= 0) {
      const int start = root;
      int v = root;
      do {
        const int nxt = a.onx[v];
        if (area(v) < a.epsClean) remove(v);
        v = nxt;
      } while (v != start && root >= 0);
    }
    if (root < 0) continue;
    // the kept vertices from root, through a scratch copy (the write position w is at or
    // before the component's own start)
    int cnt = 0, v = root;
    do { a.otmp[2 * cnt] = X[2 * v]; a.otmp[2 * cnt + 1] = X[2 * v + 1]; ++cnt; v = a.onx[v]; } while (v != root);
    for (int i = 0; i < 2 * cnt; ++i) a.oxy[2 * w + i] = a.otmp[i];
    a.ocs[nc++] = cnt;
    w += cnt;
  }
  *a.outNC = nc;
  *a.outNV = w;
}

// Where one polygon pair's data sits in the batch's arrays.
struct MultiPairDesc {
  int32_t kP, kQ;          // components
  int64_t cP0, cQ0;        // first component (start, size, root and flag arrays)
  int64_t k0;              // first ring pair (pair status; the records' ring pair index)
  int64_t r0, nR;          // records
  int64_t eP0, eQ0;        // first edge (source slots, links; the count arrays at eP0 + pair)
  int64_t sP0, sQ0;        // first ring slot
  int32_t capP, capQ;      // ring slots
  int64_t v0, vcap;        // result vertices
  int64_t c0;              // result components
  int32_t ccap, pad;
};

// One thread per polygon pair: the sequential phases are a chain of dependent steps over
// linked lists, so the batch's parallelism is across pairs (as the batched clip's
// one-thread labelling kernel has it for small ring pairs).
__global__ void __launch_bounds__(32) multi_clip_batch_kernel(MultiArgs b, const MultiPairDesc* __restrict__ desc,
                                                               int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const MultiPairDesc d = desc[i];
  MultiArgs a = b;
  a.startP = b.startP + d.cP0; a.startQ = b.startQ + d.cQ0;
  a.sizeP = b.sizeP + d.cP0; a.sizeQ = b.sizeQ + d.cQ0;
  a.edgeP = b.edgeP + d.cP0 + i; a.edgeQ = b.edgeQ + d.cQ0 + i;
  a.kP = d.kP; a.kQ = d.kQ;
  a.rp = b.rp + d.r0; a.rq = b.rq + d.r0; a.ra = b.ra + d.r0; a.rb = b.rb + d.r0; a.rt = b.rt + d.r0;
  a.rk = b.rk + d.r0;
  a.nR = d.nR; a.k0 = d.k0;
  a.pairStatus = b.pairStatus + d.k0; a.nPairs = (int64_t)d.kP * d.kQ;
  a.cntP = b.cntP + d.eP0 + i; a.cntQ = b.cntQ + d.eQ0 + i;
  a.lstP = b.lstP + d.r0; a.lstQ = b.lstQ + d.r0;
  a.srcP = b.srcP + d.eP0; a.srcQ = b.srcQ + d.eQ0;
  a.insP = b.insP + d.r0; a.insQ = b.insQ + d.r0;
  a.winP = b.winP + d.eP0; a.winQ = b.winQ + d.eQ0;
  for (int sd = 0; sd < 2; ++sd) {
    MRing& R = a.R[sd];
    const int64_t o = sd == 0 ? d.sP0 : d.sQ0;
    R.x += o; R.y += o; R.nx += o; R.pv += o; R.nb += o; R.it += o; R.lb += o; R.ee += o;
    R.used = 0;
    R.cap = sd == 0 ? d.capP : d.capQ;
    const int64_t c0 = sd == 0 ? d.cP0 : d.cQ0;
    a.root[sd] = b.root[sd] + c0; a.noInter[sd] = b.noInter[sd] + c0; a.ident[sd] = b.ident[sd] + c0;
    a.split[sd] = b.split[sd] + o; a.cand[sd] = b.cand[sd] + o;
  }
  a.mark = b.mark + d.sQ0;
  a.oxy = b.oxy + 2 * d.v0; a.vcap = d.vcap; a.ocs = b.ocs + d.c0; a.ccap = d.ccap;
  a.onx = b.onx + d.v0; a.opv = b.opv + d.v0; a.otmp = b.otmp + 2 * d.v0;
  a.status = b.status + i; a.outNC = b.outNC + i; a.outNV = b.outNV + i;
  multi_clip_pair(a);
}

// per-pair result regions -> one contiguous result (a warp per pair)
__global__ void multi_compact_kernel(const MultiPairDesc* __restrict__ desc, int64_t n,
                                     const int32_t* __restrict__ ocs, const double* __restrict__ oxy,
                                     const int32_t* __restrict__ nc, const int64_t* __restrict__ nv,
                                     const int64_t* __restrict__ compOff, const int64_t* __restrict__ vertOff,
                                     int32_t* __restrict__ csz, double* __restrict__ xy) {
  const int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (i >= n) return;
  const int64_t c0 = desc[i].c0, v0 = desc[i].v0;
  for (int64_t j = lane_id(); j < nc[i]; j += 32) csz[compOff[i] + j] = ocs[c0 + j];
  for (int64_t j = lane_id(); j < 2 * nv[i]; j += 32) xy[2 * vertOff[i] + j] = oxy[2 * v0 + j];
}

}  // namespace

int run_clip_multi_batch(int64_t n, const double* hP, const int32_t* sizesP, const int32_t* ringsP,
                         const double* hQ, const int32_t* sizesQ, const int32_t* ringsQ, const ClipParams& prm,
                         Arena& A, ClipDev& C, int* d_err, int64_t* hs, cudaStream_t s) {
  C = ClipDev();
  if (n <= 0 || !hP || !hQ || !sizesP || !sizesQ || !ringsP || !ringsQ) return ST_INVALID_ARGUMENT;
  auto sync = [&]() { return cudaStreamSynchronize(s) == cudaSuccess; };
  // ---- every ring of every pair as two layers (closing vertex stored); ring pairs of
  // pair i are (P ring c, Q ring d) for its c, d, numbered i's k0 + c * kQ + d
  const int32_t* rings[2] = {ringsP, ringsQ};
  const int32_t* sz[2] = {sizesP, sizesQ};
  const double* src[2] = {hP, hQ};
  std::vector<int64_t> c0[2], e0[2], ne[2];
  std::vector<double> hxy[2];
  std::vector<int32_t> hvn[2];
  std::vector<int64_t> hvp[2], hstart[2], hedge[2];
  int64_t nring[2] = {0, 0};
  for (int sd = 0; sd < 2; ++sd) {
    c0[sd].resize(n); e0[sd].resize(n); ne[sd].resize(n);
    int64_t ring = 0, o = 0, v = 0, e = 0;
    for (int64_t i = 0; i < n; ++i) {
      if (rings[sd][i] < 1) return ST_INVALID_ARGUMENT;
      c0[sd][i] = ring;
      e0[sd][i] = e;
      int64_t le = 0;
      for (int c = 0; c < rings[sd][i]; ++c, ++ring) {
        const int m = sz[sd][ring];
        if (m < 3) return ST_INVALID_ARGUMENT;
        hstart[sd].push_back(v);
        hedge[sd].push_back(le);
        hxy[sd].insert(hxy[sd].end(), src[sd] + 2 * o, src[sd] + 2 * (o + m));
        hxy[sd].push_back(src[sd][2 * o]);
        hxy[sd].push_back(src[sd][2 * o + 1]);
        o += m;
        v += m + 1;
        le += m;
        hvn[sd].push_back(m + 1);
        hvp[sd].push_back(v);
      }
      hedge[sd].push_back(le);            // pair i's local edge offsets: rings + 1 entries
      ne[sd][i] = le;
      e += le;
    }
    nring[sd] = ring;
    if (ring > INT32_MAX) return ST_INVALID_ARGUMENT;
  }
  std::vector<int64_t> k0(n + 1);
  k0[0] = 0;
  for (int64_t i = 0; i < n; ++i) k0[i + 1] = k0[i] + (int64_t)ringsP[i] * ringsQ[i];
  const int64_t K = k0[n];
  std::vector<int32_t> hpid(K), hqid(K);
  for (int64_t i = 0; i < n; ++i)
    for (int64_t k = 0; k < k0[i + 1] - k0[i]; ++k) {
      hpid[k0[i] + k] = (int32_t)(c0[0][i] + k / ringsQ[i]);
      hqid[k0[i] + k] = (int32_t)(c0[1][i] + k % ringsQ[i]);
    }
  double* dxy[2];
  int32_t* dvn[2];
  int64_t *dvp[2], *dstart[2], *dedge[2];
  int32_t* dsz[2];
  for (int sd = 0; sd < 2; ++sd) {
    const int64_t nr = nring[sd];
    dxy[sd] = A.take_n<double>(hxy[sd].size());
    dvn[sd] = A.take_n<int32_t>(nr);
    dvp[sd] = A.take_n<int64_t>(nr);
    dstart[sd] = A.take_n<int64_t>(nr);
    dedge[sd] = A.take_n<int64_t>(nr + n);
    dsz[sd] = A.take_n<int32_t>(nr);
    if (!dxy[sd] || !dvn[sd] || !dvp[sd] || !dstart[sd] || !dedge[sd] || !dsz[sd]) return ST_OUT_OF_MEMORY;
    cudaMemcpyAsync(dxy[sd], hxy[sd].data(), hxy[sd].size() * sizeof(double), cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(dvn[sd], hvn[sd].data(), nr * sizeof(int32_t), cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(dvp[sd], hvp[sd].data(), nr * sizeof(int64_t), cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(dstart[sd], hstart[sd].data(), nr * sizeof(int64_t), cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(dedge[sd], hedge[sd].data(), (nr + n) * sizeof(int64_t), cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(dsz[sd], sz[sd], nr * sizeof(int32_t), cudaMemcpyHostToDevice, s);
  }
  int32_t* dpid = A.take_n<int32_t>(K);
  int32_t* dqid = A.take_n<int32_t>(K);
  if (!dpid || !dqid) return ST_OUT_OF_MEMORY;
  cudaMemcpyAsync(dpid, hpid.data(), K * sizeof(int32_t), cudaMemcpyHostToDevice, s);
  cudaMemcpyAsync(dqid, hqid.data(), K * sizeof(int32_t), cudaMemcpyHostToDevice, s);
  if (!sync()) return ST_CUDA_ERROR;                         // host staging vectors end here
  const LayerDev LP{dxy[0], dvn[0], dvp[0], nring[0]}, LQ{dxy[1], dvn[1], dvp[1], nring[1]};
  // ---- intersection records of every ring pair (stages G0-G3), in ring-pair order
  ClipParams p2 = prm;
  p2.no_swap = 1;
  RingExport ex;
  ex.records_only = true;
  ClipDev CR;
  int st = run_clip(LP, LQ, dpid, dqid, K, p2, A, CR, d_err, hs, s, nullptr, nullptr, &ex);
  if (st != ST_OK) return st;
  const int64_t nRall = ex.n_records;
  std::vector<int64_t> c1(K);
  cudaMemcpyAsync(c1.data(), CR.count1, K * sizeof(int64_t), cudaMemcpyDeviceToHost, s);
  if (!sync()) return ST_CUDA_ERROR;
  // ---- each pair's place in the work arrays and result regions
  std::vector<MultiPairDesc> hd(n);
  std::vector<int64_t> hcount1(n);
  int64_t r = 0, sP = 0, sQ = 0, vo = 0, co = 0;
  for (int64_t i = 0; i < n; ++i) {
    MultiPairDesc& d = hd[i];
    int64_t nR = 0;
    for (int64_t k = k0[i]; k < k0[i + 1]; ++k) nR += c1[k];
    const int64_t capP = ne[0][i] + 2 * nR + ringsP[i] + 8, capQ = ne[1][i] + 2 * nR + ringsQ[i] + 8;
    if (capP > INT32_MAX || capQ > INT32_MAX) return ST_OUT_OF_MEMORY;
    d.kP = ringsP[i]; d.kQ = ringsQ[i];
    d.cP0 = c0[0][i]; d.cQ0 = c0[1][i];
    d.k0 = k0[i];
    d.r0 = r; d.nR = nR;
    d.eP0 = e0[0][i]; d.eQ0 = e0[1][i];
    d.sP0 = sP; d.sQ0 = sQ; d.capP = (int32_t)capP; d.capQ = (int32_t)capQ;
    d.v0 = vo; d.vcap = 2 * (capP + capQ) + 16;
    d.c0 = co; d.ccap = (int32_t)std::min<int64_t>(2 * nR + ringsP[i] + ringsQ[i] + 16, INT32_MAX); d.pad = 0;
    hcount1[i] = nR;
    r += nR; sP += capP; sQ += capQ; vo += d.vcap; co += d.ccap;
  }
  if (r != nRall) return ST_CUDA_ERROR;                    // records are in ring-pair order
  const int64_t EP = e0[0][n - 1] + ne[0][n - 1], EQ = e0[1][n - 1] + ne[1][n - 1];
  MultiArgs a{};
  a.P = reinterpret_cast<const double2*>(dxy[0]); a.Q = reinterpret_cast<const double2*>(dxy[1]);
  a.startP = dstart[0]; a.startQ = dstart[1]; a.sizeP = dsz[0]; a.sizeQ = dsz[1];
  a.edgeP = dedge[0]; a.edgeQ = dedge[1];
  a.rp = ex.rec_p; a.rq = ex.rec_q; a.ra = ex.rec_a; a.rb = ex.rec_b; a.rt = ex.rec_t; a.rk = ex.rec_k;
  a.pairStatus = CR.status;
  const int64_t nR1 = std::max<int64_t>(nRall, 1);
  a.cntP = A.take_n<int32_t>(EP + n); a.cntQ = A.take_n<int32_t>(EQ + n);
  a.lstP = A.take_n<int32_t>(nR1); a.lstQ = A.take_n<int32_t>(nR1);
  a.srcP = A.take_n<int32_t>(EP); a.srcQ = A.take_n<int32_t>(EQ);
  a.insP = A.take_n<int32_t>(nR1); a.insQ = A.take_n<int32_t>(nR1);
  a.winP = A.take_n<long long>(EP); a.winQ = A.take_n<long long>(EQ);
  bool ok = a.cntP && a.cntQ && a.lstP && a.lstQ && a.srcP && a.srcQ && a.insP && a.insQ && a.winP && a.winQ;
  const int64_t cap[2] = {sP, sQ};
  for (int sd = 0; sd < 2; ++sd) {
    MRing& R = a.R[sd];
    R.x = A.take_n<double>(cap[sd]); R.y = A.take_n<double>(cap[sd]);
    R.nx = A.take_n<int32_t>(cap[sd]); R.pv = A.take_n<int32_t>(cap[sd]); R.nb = A.take_n<int32_t>(cap[sd]);
    R.it = A.take_n<uint8_t>(cap[sd]); R.lb = A.take_n<int8_t>(cap[sd]); R.ee = A.take_n<int8_t>(cap[sd]);
    a.root[sd] = A.take_n<int32_t>(nring[sd]);
    a.noInter[sd] = A.take_n<uint8_t>(nring[sd]); a.ident[sd] = A.take_n<uint8_t>(nring[sd]);
    a.split[sd] = A.take_n<int32_t>(cap[sd]); a.cand[sd] = A.take_n<int32_t>(cap[sd]);
    ok = ok && R.x && R.y && R.nx && R.pv && R.nb && R.it && R.lb && R.ee && a.root[sd] && a.noInter[sd] &&
         a.ident[sd] && a.split[sd] && a.cand[sd];
  }
  a.mark = A.take_n<uint8_t>(sQ);
  a.oxy = A.take_n<double>(2 * vo); a.ocs = A.take_n<int32_t>(co);
  a.onx = A.take_n<int32_t>(vo); a.opv = A.take_n<int32_t>(vo); a.otmp = A.take_n<double>(2 * vo);
  MultiPairDesc* dd = A.take_n<MultiPairDesc>(n);
  C.status = A.take_n<int32_t>(n);
  C.ncomp = A.take_n<int32_t>(n);
  C.comp_off = A.take_n<int64_t>(n);
  C.count1 = A.take_n<int64_t>(n);
  C.vert_off = A.take_n<int64_t>(n);
  C.swapped = A.take_n<int32_t>(n);
  int64_t* nvOut = A.take_n<int64_t>(n);
  int64_t* tot = A.take_n<int64_t>(2);
  void* stN = A.take(scan_temp_bytes(n));
  ok = ok && a.mark && a.oxy && a.ocs && a.onx && a.opv && a.otmp && dd && C.status && C.ncomp && C.comp_off &&
       C.count1 && C.vert_off && C.swapped && nvOut && tot && stN;
  if (!ok) return ST_OUT_OF_MEMORY;
  a.status = C.status; a.outNC = C.ncomp; a.outNV = nvOut;
  a.epsClean = prm.eps_clean; a.uni = prm.union_mode; a.exact = prm.exact; a.err = d_err;
  cudaMemsetAsync(C.swapped, 0, n * sizeof(int32_t), s);
  cudaMemcpyAsync(C.count1, hcount1.data(), n * sizeof(int64_t), cudaMemcpyHostToDevice, s);
  cudaMemcpyAsync(dd, hd.data(), n * sizeof(MultiPairDesc), cudaMemcpyHostToDevice, s);
  // a warp per block: a batch of a few thousand pairs then spreads over every SM
  { multi_clip_batch_kernel<<<(unsigned)((n + 31) / 32), 32, 0, s>>>(a, dd, n); note_launch(); }
  exclusive_scan_i32(C.ncomp, C.comp_off, n, tot, stN, d_err, s);
  exclusive_scan_i64(nvOut, C.vert_off, n, tot + 1, stN, d_err, s);
  cudaMemcpyAsync(hs, tot, 2 * sizeof(int64_t), cudaMemcpyDeviceToHost, s);
  if (!sync()) return ST_CUDA_ERROR;
  const int64_t nComp = hs[0], nVert = hs[1];
  C.comp_size = A.take_n<int32_t>(std::max<int64_t>(nComp, 1));
  C.xy = A.take_n<double>(2 * std::max<int64_t>(nVert, 1));
  if (!C.comp_size || !C.xy) return ST_OUT_OF_MEMORY;
  { multi_compact_kernel<<<(unsigned)((32 * n + 127) / 128), 128, 0, s>>>(dd, n, a.ocs, a.oxy, C.ncomp, nvOut,
                                                                          C.comp_off, C.vert_off, C.comp_size,
                                                                          C.xy); note_launch(); }
  if (!sync()) return ST_CUDA_ERROR;
  C.n_pairs = n;
  C.n_components = nComp;
  C.n_vertices = nVert;
  C.n_records = nRall;
  return ST_OK;
}

int run_clip_multi(const double* hP, const int32_t* sizesP, int kP, const double* hQ, const int32_t* sizesQ, int kQ,
                   const ClipParams& prm, Arena& A, ClipDev& C, int* d_err, int64_t* hs, cudaStream_t s) {
  if (kP <= 0 || kQ <= 0) return ST_INVALID_ARGUMENT;
  const int32_t rp = kP, rq = kQ;
  return run_clip_multi_batch(1, hP, sizesP, &rp, hQ, sizesQ, &rq, prm, A, C, d_err, hs, s);
}

}  // namespace gcmfgh
