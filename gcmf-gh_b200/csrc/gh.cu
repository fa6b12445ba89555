// gh.cu -- batched Greiner-Hormann clipping of polygon pairs on sm_100a.
//
// Reference path: ghcuda (GH-CUDA/ghcuda.cpp:385-425) clips one pair at a time:
// calculateIntersections on the GPU (gppolyclip_mDIV512.cu:1298-1715: CMBR edge filter,
// counts, host scans, neighbour map, intersections, per-edge alpha sort, initial labels),
// then the CPU phases of GH-CUDA/lib/polyclip.h (labelIntersections :335-735,
// createResult :743-783, cleanUpResult :791-807).  Here every phase of every pair of a
// batch runs on the device:
//
//   G0 setup        thread/pair: the swap rule (ghcuda.cpp:64-91: the polygon with more
//                   vertices is P), MBRs, common MBR (ghcuda.cpp:94-125), disjoint check
//   G1 edge filter  warp/pair: P and Q edges whose box touches the common MBR
//                   (gppolyclip_mDIV512.cu:382-415), compacted in edge order
//   G2 count        warp per 256-edge-pair chunk of each pair's filtered P x Q grid: box
//                   test (:345-371) and classification from both sides (:95-169);
//                   records = P-side hits, the P/Q totals decide validity (:1461)
//   G3 emit         same chunks; records written in (pair, P edge, Q edge) order, so no
//                   sort is needed and results do not depend on scheduling
//   G4 ring layout  per edge: 1 source vertex + inserted vertices; one device scan per
//                   side gives every vertex its slot (replaces the host scans :1431-1434)
//   G5 ring fill    thread/edge: inserted vertices ordered by exact parameter (ties: later
//                   insertion first, as polygon.h:101-113 inserts in the loop order of
//                   polyclip.h:202-205) instead of the reference GPU's 1e-7-quantised
//                   radix sort (:290-305, :1034)
//   G6 links        thread/record: neighbour links as polyclip.h:215-267 makes them; a
//                   source vertex linked by several records keeps the last one
//   G7 label+trace  thread/pair: initial labels, chains, special cases, entry/exit, split
//                   pairs, crossing candidates, tracing and clean-up
//   G8 compaction   per-pair output regions -> one contiguous result
//
// Layout in HBM: the input layers stay interleaved FP64 (16 B per vertex).  Records are
// structure-of-arrays (P edge, Q edge, alpha, beta, type, pair).  Each pair owns a ring
// region per side holding its merged vertex ring followed by room for the vertices the
// labelling may add (one temporary vertex, one duplicate per split vertex): x, y, next,
// prev, neighbour (pair-local slot on the other side), flags, label, entry/exit.
#include <algorithm>
#include "common.cuh"
#include "engine.cuh"
#include "prims.cuh"

namespace gcmfgh {

namespace {

constexpr int kThreads = 256;
constexpr int kWarpsPerBlock = kThreads / 32;
constexpr int kChunk = 256;            // edge pairs per warp work unit (8 x 32 lanes)

inline unsigned blocks_for_warps(int64_t warps) {
  return (unsigned)((warps + kWarpsPerBlock - 1) / kWarpsPerBlock);
}
inline unsigned blocks_for(int64_t n) { return (unsigned)((n + kThreads - 1) / kThreads); }

enum : int8_t { L_NONE = 0, L_CROSSING, L_BOUNCING, L_LEFT_ON, L_RIGHT_ON, L_ON_ON, L_ON_LEFT,
                L_ON_RIGHT, L_DELAYED_CROSSING, L_DELAYED_BOUNCING };
enum : int8_t { E_EXIT = 0, E_ENTRY = 1, E_NEITHER = 2 };
enum : int { R_LEFT = 0, R_RIGHT = 1, R_IS_P_M = 2, R_IS_P_P = 3 };

// ---------------------------------------------------------------- pair setup
struct PairDev {
  int64_t* pS;      // first vertex (index into P's layer)
  int64_t* qS;
  int32_t* nP;      // ring size (closing vertex excluded)
  int32_t* nQ;
  int8_t* pSide;    // 0: P is the base polygon, 1: P is the overlay polygon
  double* cmbr;     // [4 K]
  int32_t* status;  // 0 ok, 1 invalid, 2 disjoint, 3 trace error
};

__device__ __forceinline__ const double2* layer_xy(const LayerDev& Lb, const LayerDev& Lo, int side) {
  return reinterpret_cast<const double2*>(side == 0 ? Lb.xy : Lo.xy);
}

__global__ void setup_kernel(LayerDev Lb, LayerDev Lo, const int32_t* __restrict__ pid,
                             const int32_t* __restrict__ qid, int64_t K, const double* __restrict__ mb,
                             const double* __restrict__ mo, PairDev D, int32_t* __restrict__ swapped,
                             int no_swap) {
  int64_t k = (int64_t)blockIdx.x * kThreads + threadIdx.x;
  if (k >= K) return;
  int b = pid[k], o = qid[k];
  int nb = Lb.vnum[b] - 1, no = Lo.vnum[o] - 1;
  bool sw = !no_swap && nb < no;        // ghcuda.cpp:66: swap when |P| < |Q|
  int64_t sb = Lb.vps[b] - Lb.vnum[b], so = Lo.vps[o] - Lo.vnum[o];
  double4 MB = reinterpret_cast<const double4*>(mb)[b];
  double4 MO = reinterpret_cast<const double4*>(mo)[o];
  double4 MP = sw ? MO : MB, MQ = sw ? MB : MO;
  D.pS[k] = sw ? so : sb; D.qS[k] = sw ? sb : so;
  D.nP[k] = sw ? no : nb; D.nQ[k] = sw ? nb : no;
  D.pSide[k] = sw ? 1 : 0;
  swapped[k] = sw ? 1 : 0;
  int st = 0;
  if (MP.x > MQ.z || MP.z < MQ.x || MP.y > MQ.w || MP.w < MQ.y) st = 2;   // ghcuda.cpp:109-116
  if (D.nP[k] < 1 || D.nQ[k] < 1) st = 2;
  D.status[k] = st;
  reinterpret_cast<double4*>(D.cmbr)[k] = make_double4(fmax(MP.x, MQ.x), fmax(MP.y, MQ.y),
                                                       fmin(MP.z, MQ.z), fmin(MP.w, MQ.w));
}

// ---------------------------------------------------------------- G1 edge filter
template <int kMode>
__global__ void __launch_bounds__(kThreads)
edge_filter_kernel(LayerDev Lb, LayerDev Lo, PairDev D, int64_t K, int32_t* __restrict__ cP,
                   int32_t* __restrict__ cQ, const int64_t* __restrict__ offP,
                   const int64_t* __restrict__ offQ, int32_t* __restrict__ LP, int32_t* __restrict__ LQ) {
  int64_t w = ((int64_t)blockIdx.x * kThreads + threadIdx.x) >> 5;
  if (w >= K) return;
  if (D.status[w] != 0) { if (kMode == 0 && lane_id() == 0) { cP[w] = 0; cQ[w] = 0; } return; }
  double4 c = reinterpret_cast<const double4*>(D.cmbr)[w];
  const int pside = D.pSide[w];
  for (int side = 0; side < 2; ++side) {
    const double2* v = layer_xy(Lb, Lo, side == 0 ? pside : 1 - pside) + (side == 0 ? D.pS[w] : D.qS[w]);
    const int n = side == 0 ? D.nP[w] : D.nQ[w];
    int cnt = 0;
    int64_t pos = 0;
    int32_t* list = nullptr;
    if (kMode == 1) { pos = side == 0 ? offP[w] : offQ[w]; list = side == 0 ? LP : LQ; }
    for (int k0 = 0; k0 < n; k0 += 32) {
      int k = k0 + lane_id();
      bool hit = false;
      if (k < n) {
        double2 a = __ldg(v + k), b = __ldg(v + (k + 1 < n ? k + 1 : 0));
        hit = edge_touches_box(a.x, a.y, b.x, b.y, c.x, c.y, c.z, c.w);
      }
      unsigned m = __ballot_sync(0xffffffffu, hit);
      if (kMode == 1 && hit) list[pos + cnt + __popc(m & lanemask_lt())] = k;
      cnt += __popc(m);
    }
    if (kMode == 0 && lane_id() == 0) { if (side == 0) cP[w] = cnt; else cQ[w] = cnt; }
  }
}

__global__ void chunk_count_kernel(const int32_t* __restrict__ cP, const int32_t* __restrict__ cQ,
                                   int64_t K, int64_t* __restrict__ nchunk) {
  int64_t k = (int64_t)blockIdx.x * kThreads + threadIdx.x;
  if (k >= K) return;
  int64_t W = (int64_t)cP[k] * cQ[k];
  nchunk[k] = (W + kChunk - 1) / kChunk;
}

// ---------------------------------------------------------------- G2/G3 count + emit
struct Records {
  int32_t* p;       // pair-local P edge
  int32_t* q;       // pair-local Q edge
  double* a;        // alpha (on P)
  double* b;        // beta (on Q)
  int8_t* t;        // intersection type 1..8
  int32_t* k;       // pair
};

template <int kMode>
__global__ void __launch_bounds__(kThreads)
intersect_kernel(LayerDev Lb, LayerDev Lo, PairDev D, int64_t K, const int64_t* __restrict__ chunkOff,
                 int64_t nChunks, const int32_t* __restrict__ cP, const int32_t* __restrict__ cQ,
                 const int64_t* __restrict__ offP, const int64_t* __restrict__ offQ,
                 const int32_t* __restrict__ LP, const int32_t* __restrict__ LQ, double eps,
                 int32_t* __restrict__ chunkRec, int32_t* __restrict__ chunkQ,
                 const int64_t* __restrict__ chunkRecOff, Records R) {
  int64_t c = ((int64_t)blockIdx.x * kThreads + threadIdx.x) >> 5;
  if (c >= nChunks) return;
  // pair of this chunk: last k with chunkOff[k] <= c (pairs without chunks are skipped)
  int64_t k = upper_index(chunkOff, K, c);
  const int nq = cQ[k];
  const int64_t W = (int64_t)cP[k] * nq;
  const int64_t t0 = (c - chunkOff[k]) * kChunk;
  const int pside = D.pSide[k];
  const double2* pv = layer_xy(Lb, Lo, pside) + D.pS[k];
  const double2* qv = layer_xy(Lb, Lo, 1 - pside) + D.qS[k];
  const int np_ = D.nP[k], nq_ = D.nQ[k];
  const int32_t* lp = LP + offP[k];
  const int32_t* lq = LQ + offQ[k];
  int recs = 0, qhits = 0;
  int64_t pos = (kMode == 1) ? chunkRecOff[c] : 0;
  for (int it = 0; it < kChunk / 32; ++it) {
    int64_t t = t0 + it * 32 + lane_id();
    int tp = 0, tq = 0;
    int pe = 0, qe = 0;
    double alpha = 0, beta = 0;
    if (t < W) {
      pe = lp[t / nq];
      qe = lq[t % nq];
      double2 P1 = __ldg(pv + pe), P2 = __ldg(pv + (pe + 1 < np_ ? pe + 1 : 0));
      double2 Q1 = __ldg(qv + qe), Q2 = __ldg(qv + (qe + 1 < nq_ ? qe + 1 : 0));
      if (edge_boxes_touch(P1.x, P1.y, P2.x, P2.y, Q1.x, Q1.y, Q2.x, Q2.y)) {
        tp = classify_edges(P1.x, P1.y, P2.x, P2.y, Q1.x, Q1.y, Q2.x, Q2.y, eps, alpha, beta);
        if (kMode == 0) {
          double a2, b2;
          tq = classify_edges(Q1.x, Q1.y, Q2.x, Q2.y, P1.x, P1.y, P2.x, P2.y, eps, a2, b2);
        }
      }
    }
    unsigned m = __ballot_sync(0xffffffffu, tp != 0);
    if (kMode == 0) {
      recs += __popc(m);
      qhits += __popc(__ballot_sync(0xffffffffu, tq != 0));
    } else if (tp != 0) {
      int64_t r = pos + __popc(m & lanemask_lt());
      R.p[r] = pe; R.q[r] = qe; R.a[r] = alpha; R.b[r] = beta; R.t[r] = (int8_t)tp; R.k[r] = (int32_t)k;
    }
    pos += __popc(m);
  }
  if (kMode == 0 && lane_id() == 0) { chunkRec[c] = recs; chunkQ[c] = qhits; }
}

// per pair: record range, validity
__global__ void pair_records_kernel(const int64_t* __restrict__ chunkOff, const int64_t* __restrict__ nchunk,
                                    const int64_t* __restrict__ recScan, const int64_t* __restrict__ qScan,
                                    const int32_t* __restrict__ chunkRec, const int32_t* __restrict__ chunkQ,
                                    int64_t K, int64_t* __restrict__ recOff, int32_t* __restrict__ nrec,
                                    int64_t* __restrict__ count1, PairDev D) {
  int64_t k = (int64_t)blockIdx.x * kThreads + threadIdx.x;
  if (k >= K) return;
  int64_t c0 = chunkOff[k], n = nchunk[k];
  int64_t r0 = 0, r1 = 0, q0 = 0, q1 = 0;
  if (n > 0) {
    r0 = recScan[c0]; r1 = recScan[c0 + n - 1] + chunkRec[c0 + n - 1];
    q0 = qScan[c0]; q1 = qScan[c0 + n - 1] + chunkQ[c0 + n - 1];
  }
  recOff[k] = r0;
  nrec[k] = (int32_t)(r1 - r0);
  count1[k] = r1 - r0;
  if (D.status[k] == 0 && (r1 - r0) != (q1 - q0)) D.status[k] = 1;   // gppolyclip_mDIV512.cu:1461
}

// ---------------------------------------------------------------- G4 ring layout
// Per record: insertion counts per edge, and the winning (last) record for each source
// vertex that records link (P: types 2,4,5,6,8; Q: types 3,4,5,7,8).
__global__ void record_count_kernel(Records R, int64_t nR, const int64_t* __restrict__ eoffP,
                                    const int64_t* __restrict__ eoffQ, const int32_t* __restrict__ status,
                                    int32_t* __restrict__ insP, int32_t* __restrict__ insQ,
                                    int64_t* __restrict__ srcLinkP, int64_t* __restrict__ srcLinkQ) {
  int64_t r = (int64_t)blockIdx.x * kThreads + threadIdx.x;
  if (r >= nR) return;
  int k = R.k[r];
  if (status[k] != 0) return;
  int t = R.t[r];
  int64_t eP = eoffP[k] + R.p[r], eQ = eoffQ[k] + R.q[r];
  if (t == 1 || t == 3 || t == 5 || t == 7) atomicAdd(&insP[eP], 1);
  if (t == 1 || t == 2 || t == 5 || t == 6) atomicAdd(&insQ[eQ], 1);
  if (t == 2 || t == 4 || t == 5 || t == 6 || t == 8)
    atomicMax(reinterpret_cast<unsigned long long*>(&srcLinkP[eP]), (unsigned long long)(r + 1));
  if (t == 3 || t == 4 || t == 5 || t == 7 || t == 8)
    atomicMax(reinterpret_cast<unsigned long long*>(&srcLinkQ[eQ]), (unsigned long long)(r + 1));
}

__global__ void edge_slots_kernel(const int32_t* __restrict__ ins, int64_t nE, int32_t* __restrict__ sz) {
  int64_t e = (int64_t)blockIdx.x * kThreads + threadIdx.x;
  if (e < nE) sz[e] = 1 + ins[e];
}

struct RingSet {
  double* x; double* y;
  int32_t* nx; int32_t* pv; int32_t* nb;
  uint8_t* it;      // intersection flag (cleared when visited by the trace)
  int8_t* lb;       // IntersectionLabel
  int8_t* ee;       // EntryExitLabel
  uint8_t* fl;      // bit0 split candidate, bit1 crossing candidate
};

// per pair: ring size, region offset (ring + room for added vertices)
__global__ void pair_ring_kernel(const int64_t* __restrict__ eoff, const int64_t* __restrict__ vpos,
                                 const int32_t* __restrict__ n, const int32_t* __restrict__ nrec,
                                 const int32_t* __restrict__ status, int64_t K, int64_t nE, int64_t vtot,
                                 int32_t* __restrict__ m, int64_t* __restrict__ regSize) {
  int64_t k = (int64_t)blockIdx.x * kThreads + threadIdx.x;
  if (k >= K) return;
  int64_t e0 = eoff[k], e1 = e0 + (status[k] == 2 ? 0 : n[k]);
  int64_t v0 = e0 < nE ? vpos[e0] : vtot, v1 = e1 < nE ? vpos[e1] : vtot;
  int mm = status[k] == 0 ? (int)(v1 - v0) : 0;
  m[k] = mm;
  regSize[k] = status[k] == 0 ? (int64_t)mm + 2 + 2 * (int64_t)nrec[k] : 0;
}

// ---------------------------------------------------------------- G5 ring fill
// Thread per edge: the edge's source vertex, then its inserted vertices sorted by
// (parameter ascending, other edge descending).  side 0 fills P rings, side 1 Q rings.
// An edge of the smaller polygon can cross thousands of edges of a large one; edges with
// more than kLightEdge insertions are left to heavy_fill_kernel, which sorts them with a
// block-wide bitonic network.
constexpr int kLightEdge = 32;

struct EdgeFill {
  int64_t k, base;
  int s0, mm, np_;
  const double2* pvx;
  const double2* qvx;
};

template <int kSide>
__device__ __forceinline__ void write_inserted(const EdgeFill& f, const Records& R, int64_t r, int i,
                                               RingSet& S, int64_t* slotOfRec) {
  int t = R.t[r];
  double X, Y;
  if (t == 1) {
    // I = (1-alpha) P1 + alpha P2 (gppolyclip_mDIV512.cu:1029, polyclip.h:220)
    int pe = R.p[r];
    double a = R.a[r];
    double2 P1 = __ldg(f.pvx + pe), P2 = __ldg(f.pvx + (pe + 1 < f.np_ ? pe + 1 : 0));
    X = (1.0 - a) * P1.x + a * P2.x;
    Y = (1.0 - a) * P1.y + a * P2.y;
  } else if (kSide == 0) {          // types 3, 5, 7: a copy of Q1 on P
    double2 Q1 = __ldg(f.qvx + R.q[r]);
    X = Q1.x; Y = Q1.y;
  } else {                          // types 2, 5, 6: a copy of P1 on Q
    double2 P1 = __ldg(f.pvx + R.p[r]);
    X = P1.x; Y = P1.y;
  }
  int sl = f.s0 + 1 + i;
  int64_t gs = f.base + sl;
  S.x[gs] = X; S.y[gs] = Y;
  S.nx[gs] = (sl + 1) % f.mm; S.pv[gs] = (sl + f.mm - 1) % f.mm; S.nb[gs] = -1;
  S.it[gs] = 0; S.lb[gs] = L_NONE; S.ee[gs] = E_NEITHER; S.fl[gs] = 0;
  slotOfRec[r] = sl;
}

template <int kSide>
__device__ __forceinline__ bool edge_fill_info(const LayerDev& Lb, const LayerDev& Lo, const PairDev& D,
                                               const int64_t* eoff, int64_t K, const int64_t* vpos,
                                               const int64_t* regOff, const int32_t* m, int64_t e, EdgeFill& f) {
  int64_t k = upper_index(eoff, K, e);
  if (D.status[k] != 0) return false;
  const int n = kSide == 0 ? D.nP[k] : D.nQ[k];
  if ((int)(e - eoff[k]) >= n) return false;
  const int pside = D.pSide[k];
  f.k = k;
  f.mm = m[k];
  f.base = regOff[k];
  f.s0 = (int)(vpos[e] - vpos[eoff[k]]);
  f.pvx = layer_xy(Lb, Lo, pside) + D.pS[k];
  f.qvx = layer_xy(Lb, Lo, 1 - pside) + D.qS[k];
  f.np_ = D.nP[k];
  return true;
}

template <int kSide>
__global__ void ring_fill_kernel(LayerDev Lb, LayerDev Lo, PairDev D, Records R,
                                 const int64_t* __restrict__ eoff, int64_t nE, int64_t K,
                                 const int64_t* __restrict__ vpos, const int64_t* __restrict__ regOff,
                                 const int32_t* __restrict__ m, RingSet S, int64_t* __restrict__ slotOfRec,
                                 const int64_t* __restrict__ insCursorBase, int32_t* __restrict__ insCursor,
                                 const int64_t* __restrict__ insList, int64_t* __restrict__ heavy,
                                 unsigned long long* __restrict__ nHeavy) {
  int64_t e = (int64_t)blockIdx.x * kThreads + threadIdx.x;
  if (e >= nE) return;
  EdgeFill f;
  if (!edge_fill_info<kSide>(Lb, Lo, D, eoff, K, vpos, regOff, m, e, f)) return;
  const int le = (int)(e - eoff[f.k]);
  const double2 A = __ldg((kSide == 0 ? f.pvx : f.qvx) + le);
  const int64_t g = f.base + f.s0;
  S.x[g] = A.x; S.y[g] = A.y;
  S.nx[g] = (f.s0 + 1) % f.mm; S.pv[g] = (f.s0 + f.mm - 1) % f.mm; S.nb[g] = -1;
  S.it[g] = 0; S.lb[g] = L_NONE; S.ee[g] = E_NEITHER; S.fl[g] = 0;
  // inserted records of this edge, gathered by record_scatter_kernel into insList
  const int64_t l0 = insCursorBase[e];
  const int cnt = insCursor[e];
  if (cnt > kLightEdge) {
    heavy[atomicAdd(nHeavy, 1ull)] = e;
    return;
  }
  // insertion sort of the (few) records by (parameter asc, other edge desc)
  int64_t* lst = const_cast<int64_t*>(insList) + l0;
  for (int i = 1; i < cnt; ++i) {
    int64_t r = lst[i];
    double key = kSide == 0 ? R.a[r] : R.b[r];
    int oth = kSide == 0 ? R.q[r] : R.p[r];
    int j = i - 1;
    while (j >= 0) {
      int64_t rj = lst[j];
      double kj = kSide == 0 ? R.a[rj] : R.b[rj];
      int oj = kSide == 0 ? R.q[rj] : R.p[rj];
      bool after = (kj > key) || (kj == key && oj < oth);
      if (!after) break;
      lst[j + 1] = rj;
      --j;
    }
    lst[j + 1] = r;
  }
  for (int i = 0; i < cnt; ++i) write_inserted<kSide>(f, R, lst[i], i, S, slotOfRec);
}

// Block per heavy edge: bitonic sort of (parameter bits, ~other edge, list position) --
// ascending parameter, descending other edge -- in shared memory up to kHeavySmem
// elements, in a global scratch segment beyond; then the vertices are written in order.
constexpr int kHeavyThreads = 512;
constexpr int kHeavySmem = 4096;

__device__ void bitonic_sort(uint64_t* key, uint32_t* tie, uint32_t* idx, int npad) {
  for (int size = 2; size <= npad; size <<= 1) {
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int i = threadIdx.x; i < (npad >> 1); i += blockDim.x) {
        int lo = 2 * i - (i & (stride - 1));
        int hi = lo + stride;
        bool up = (lo & size) == 0;
        uint64_t ka = key[lo], kb = key[hi];
        uint32_t ta = tie[lo], tb = tie[hi];
        bool gt = (ka > kb) || (ka == kb && ta > tb);
        if (gt == up) {
          key[lo] = kb; key[hi] = ka;
          tie[lo] = tb; tie[hi] = ta;
          uint32_t x = idx[lo]; idx[lo] = idx[hi]; idx[hi] = x;
        }
      }
      __syncthreads();
    }
  }
}

template <int kSide>
__global__ void __launch_bounds__(kHeavyThreads)
heavy_fill_kernel(LayerDev Lb, LayerDev Lo, PairDev D, Records R, const int64_t* __restrict__ eoff, int64_t K,
                  const int64_t* __restrict__ vpos, const int64_t* __restrict__ regOff,
                  const int32_t* __restrict__ m, RingSet S, int64_t* __restrict__ slotOfRec,
                  const int64_t* __restrict__ insCursorBase, const int32_t* __restrict__ insCursor,
                  const int64_t* __restrict__ insList, const int64_t* __restrict__ heavy,
                  const unsigned long long* __restrict__ nHeavy, uint64_t* gkey, uint32_t* gtie, uint32_t* gidx) {
  extern __shared__ unsigned char smem[];
  uint64_t* skey = reinterpret_cast<uint64_t*>(smem);
  uint32_t* stie = reinterpret_cast<uint32_t*>(skey + kHeavySmem);
  uint32_t* sidx = stie + kHeavySmem;
  __shared__ EdgeFill f;
  const unsigned long long nh = *nHeavy;
  for (unsigned long long h = blockIdx.x; h < nh; h += gridDim.x) {
    const int64_t e = heavy[h];
    if (threadIdx.x == 0) edge_fill_info<kSide>(Lb, Lo, D, eoff, K, vpos, regOff, m, e, f);
    __syncthreads();
    const int64_t l0 = insCursorBase[e];
    const int cnt = insCursor[e];
    int npad = 1;
    while (npad < cnt) npad <<= 1;
    uint64_t* key = skey;
    uint32_t* tie = stie;
    uint32_t* idx = sidx;
    if (npad > kHeavySmem) { key = gkey + 2 * l0; tie = gtie + 2 * l0; idx = gidx + 2 * l0; }
    for (int i = threadIdx.x; i < npad; i += blockDim.x) {
      if (i < cnt) {
        int64_t r = insList[l0 + i];
        key[i] = ordered_key(kSide == 0 ? R.a[r] : R.b[r]);
        tie[i] = 0xffffffffu - (uint32_t)(kSide == 0 ? R.q[r] : R.p[r]);
        idx[i] = (uint32_t)i;
      } else {
        key[i] = ~0ull; tie[i] = 0xffffffffu; idx[i] = 0xffffffffu;
      }
    }
    __syncthreads();
    bitonic_sort(key, tie, idx, npad);
    for (int i = threadIdx.x; i < cnt; i += blockDim.x)
      write_inserted<kSide>(f, R, insList[l0 + idx[i]], i, S, slotOfRec);
    __syncthreads();
  }
}

// records inserting on an edge -> that edge's list (order fixed later by ring_fill)
__global__ void record_scatter_kernel(Records R, int64_t nR, const int64_t* __restrict__ eoffP,
                                      const int64_t* __restrict__ eoffQ, const int32_t* __restrict__ status,
                                      const int64_t* __restrict__ baseP, int32_t* __restrict__ curP,
                                      int64_t* __restrict__ listP, const int64_t* __restrict__ baseQ,
                                      int32_t* __restrict__ curQ, int64_t* __restrict__ listQ) {
  int64_t r = (int64_t)blockIdx.x * kThreads + threadIdx.x;
  if (r >= nR) return;
  int k = R.k[r];
  if (status[k] != 0) return;
  int t = R.t[r];
  int64_t eP = eoffP[k] + R.p[r], eQ = eoffQ[k] + R.q[r];
  if (t == 1 || t == 3 || t == 5 || t == 7) listP[baseP[eP] + atomicAdd(&curP[eP], 1)] = r;
  if (t == 1 || t == 2 || t == 5 || t == 6) listQ[baseQ[eQ] + atomicAdd(&curQ[eQ], 1)] = r;
}

// ---------------------------------------------------------------- G6 links
__device__ __forceinline__ void set_link(RingSet& S, int64_t base, int slot, int target) {
  S.nb[base + slot] = target;
  S.it[base + slot] = 1;
}

__global__ void link_kernel(Records R, int64_t nR, const int32_t* __restrict__ status,
                            const int64_t* __restrict__ eoffP, const int64_t* __restrict__ eoffQ,
                            const int64_t* __restrict__ vposP, const int64_t* __restrict__ vposQ,
                            const int64_t* __restrict__ regP, const int64_t* __restrict__ regQ,
                            const int64_t* __restrict__ slotP, const int64_t* __restrict__ slotQ,
                            const int64_t* __restrict__ srcLinkP, const int64_t* __restrict__ srcLinkQ,
                            RingSet SP, RingSet SQ) {
  int64_t r = (int64_t)blockIdx.x * kThreads + threadIdx.x;
  if (r >= nR) return;
  int k = R.k[r];
  if (status[k] != 0) return;
  int t = R.t[r];
  int64_t eP = eoffP[k] + R.p[r], eQ = eoffQ[k] + R.q[r];
  const int srcP = (int)(vposP[eP] - vposP[eoffP[k]]);
  const int srcQ = (int)(vposQ[eQ] - vposQ[eoffQ[k]]);
  const int64_t bP = regP[k], bQ = regQ[k];
  const bool winP = srcLinkP[eP] == r + 1, winQ = srcLinkQ[eQ] == r + 1;
  switch (t) {
    case 1: {
      int sp = (int)slotP[r], sq = (int)slotQ[r];
      set_link(SP, bP, sp, sq); set_link(SQ, bQ, sq, sp);
      break;
    }
    case 2: case 6: {
      int sq = (int)slotQ[r];
      set_link(SQ, bQ, sq, srcP);
      SP.it[bP + srcP] = 1;
      if (winP) SP.nb[bP + srcP] = sq;
      break;
    }
    case 3: case 7: {
      int sp = (int)slotP[r];
      set_link(SP, bP, sp, srcQ);
      SQ.it[bQ + srcQ] = 1;
      if (winQ) SQ.nb[bQ + srcQ] = sp;
      break;
    }
    case 4: case 8: {
      SP.it[bP + srcP] = 1; SQ.it[bQ + srcQ] = 1;
      if (winP) SP.nb[bP + srcP] = srcQ;
      if (winQ) SQ.nb[bQ + srcQ] = srcP;
      break;
    }
    case 5: {
      int sp = (int)slotP[r], sq = (int)slotQ[r];
      set_link(SQ, bQ, sq, srcP);
      SP.it[bP + srcP] = 1;
      if (winP) SP.nb[bP + srcP] = sq;
      set_link(SP, bP, sp, srcQ);
      SQ.it[bQ + srcQ] = 1;
      if (winQ) SQ.nb[bQ + srcQ] = sp;
      break;
    }
  }
}

// ---------------------------------------------------------------- G7 label + trace
struct Ring {
  double* x; double* y; int32_t* nx; int32_t* pv; int32_t* nb;
  uint8_t* it; int8_t* lb; int8_t* ee; uint8_t* fl;
  int m;        // slots in the merged ring
  int used;     // slots in use (ring + added vertices)
  int cap;      // region capacity
};

__device__ __forceinline__ Ring ring_of(const RingSet& S, int64_t base, int m, int cap) {
  Ring r;
  r.x = S.x + base; r.y = S.y + base; r.nx = S.nx + base; r.pv = S.pv + base; r.nb = S.nb + base;
  r.it = S.it + base; r.lb = S.lb + base; r.ee = S.ee + base; r.fl = S.fl + base;
  r.m = m; r.used = m; r.cap = cap;
  return r;
}

__device__ int add_vertex(Ring& R, double X, double Y) {
  if (R.used >= R.cap) return -1;
  int v = R.used++;
  R.x[v] = X; R.y[v] = Y; R.nx[v] = v; R.pv[v] = v; R.nb[v] = -1;
  R.it[v] = 0; R.lb[v] = L_NONE; R.ee[v] = E_NEITHER; R.fl[v] = 0;
  return v;
}

__device__ __forceinline__ void insert_after(Ring& R, int v, int after) {
  int c = R.nx[after];
  R.nx[R.pv[c]] = v; R.pv[v] = R.pv[c]; R.nx[v] = c; R.pv[c] = v;
}

// polygon.h:427-448 (winding parity) over the ring reached from slot 0, skipping `skip`
__device__ bool point_in_ring(const Ring& R, double Rx, double Ry, int skip) {
  int w = 0;
  int one = 0;
  int guard = R.used + 2;
  do {
    int two = R.nx[one];
    if (two == skip) two = R.nx[two];
    double P0x = R.x[one], P0y = R.y[one], P1x = R.x[two], P1y = R.y[two];
    if ((P0y < Ry) != (P1y < Ry)) {
      if (P0x >= Rx) {
        if (P1x > Rx) w = w + 2 * (P1y > P0y) - 1;
        else if ((area2(P0x, P0y, P1x, P1y, Rx, Ry) > 0) == (P1y > P0y)) w = w + 2 * (P1y > P0y) - 1;
      } else if (P1x > Rx) {
        if ((area2(P0x, P0y, P1x, P1y, Rx, Ry) > 0) == (P1y > P0y)) w = w + 2 * (P1y > P0y) - 1;
      }
    }
    one = two;
  } while (one != 0 && --guard > 0);
  return (w % 2) != 0;
}

// relative position of Q w.r.t. the chain (P1, P2, P3): polyclip.h:297-326
__device__ int rel_position(const Ring& P, const Ring& Q, int qv, int p1, int p2, int p3) {
  if (P.it[p1] && P.nb[p1] == qv) return R_IS_P_M;
  if (P.it[p3] && P.nb[p3] == qv) return R_IS_P_P;
  double s1 = area2(Q.x[qv], Q.y[qv], P.x[p1], P.y[p1], P.x[p2], P.y[p2]);
  double s2 = area2(Q.x[qv], Q.y[qv], P.x[p2], P.y[p2], P.x[p3], P.y[p3]);
  double s3 = area2(P.x[p1], P.y[p1], P.x[p2], P.y[p2], P.x[p3], P.y[p3]);
  if (s3 > 0) return (s1 > 0 && s2 > 0) ? R_LEFT : R_RIGHT;
  return (s1 < 0 && s2 < 0) ? R_RIGHT : R_LEFT;
}

// gppolyclip_mDIV512.cu:237-252
__device__ __forceinline__ int8_t initial_label(int m, int p) {
  auto is = [&](int a, int b) { return (m == a && p == b) || (m == b && p == a); };
  if (is(R_LEFT, R_RIGHT)) return L_CROSSING;
  if ((m == R_LEFT && p == R_LEFT) || (m == R_RIGHT && p == R_RIGHT)) return L_BOUNCING;
  if (is(R_IS_P_P, R_RIGHT)) return L_LEFT_ON;
  if (is(R_IS_P_P, R_LEFT)) return L_RIGHT_ON;
  if (is(R_IS_P_P, R_IS_P_M)) return L_ON_ON;
  if (is(R_IS_P_M, R_RIGHT)) return L_ON_LEFT;
  if (is(R_IS_P_M, R_LEFT)) return L_ON_RIGHT;
  return L_NONE;
}

struct OutRegion {
  double* xy;        // vertex region of the pair (2 doubles per vertex)
  int32_t* csz;      // component sizes of the pair
  int64_t vcap;
  int ccap;
  int64_t nv;
  int nc;
  bool overflow;
  __device__ void begin() { if (nc < ccap) csz[nc] = 0; else overflow = true; }
  __device__ void push(double X, double Y) {
    if (overflow) return;
    if (nv >= vcap) { overflow = true; return; }
    xy[2 * nv] = X; xy[2 * nv + 1] = Y; ++nv; ++csz[nc];
  }
  __device__ void end() { if (!overflow) ++nc; }
};

// first non-intersection vertex in ring order from slot 0, else the first vertex whose
// edge to the next vertex is not collinear with the other polygon (polygon.h:480-512)
__device__ int first_non_intersection(const Ring& A, const Ring& B, bool& midpoint) {
  midpoint = false;
  int v = 0, guard = A.used + 1;
  do { if (!A.it[v]) return v; v = A.nx[v]; } while (v != 0 && --guard > 0);
  v = 0; guard = A.used + 1;
  do {
    int nb = A.nb[v], nx = A.nx[v];
    if (nb >= 0 && A.nb[nx] != B.pv[nb] && A.nb[nx] != B.nx[nb]) { midpoint = true; return v; }
    v = A.nx[v];
  } while (v != 0 && --guard > 0);
  return -1;
}

__device__ void push_ring(OutRegion& O, const Ring& A) {
  O.begin();
  int v = 0, guard = A.used + 1;
  do { O.push(A.x[v], A.y[v]); v = A.nx[v]; } while (v != 0 && --guard > 0);
  O.end();
}

// Per-pair state of the labelling and tracing phases.
struct PairCtx {
  Ring R[2];
  OutRegion O;
  bool uni;
  double eps_clean;
  int* err;
  int32_t* status;
  bool noInter[2];
  bool ident[2];
};

__device__ __forceinline__ int8_t toggled(int8_t st) {
  return (st == E_ENTRY) ? E_EXIT : (st == E_EXIT ? E_ENTRY : st);
}

__device__ __forceinline__ void fail(PairCtx& c, int code) {
  raise_error(c.err, code);
  *c.status = 3;
}

// ================================================================ sequential phases
// One thread walks the pair exactly as polyclip.h does.  Used whole when the links are not
// one-to-one, and for the parts the warp version leaves to one lane (chain anomalies,
// split vertices, tracing through added vertices).

// step 1: initial labels (computed on P, copied to the neighbour on Q)
__device__ void seq_step1(PairCtx& c) {
  Ring& P = c.R[0];
  Ring& Q = c.R[1];
  for (int s = 0; s < P.m; ++s) {
    if (!P.it[s]) continue;
    int nb = P.nb[s];
    if (nb < 0) continue;
    int pm = P.pv[s], pp = P.nx[s];
    int a = rel_position(P, Q, Q.pv[nb], pm, s, pp);
    int b = rel_position(P, Q, Q.nx[nb], pm, s, pp);
    int8_t L = initial_label(a, b);
    if (L != L_NONE) { P.lb[s] = L; Q.lb[nb] = L; }
  }
}

// step 2: intersection chains (polyclip.h:405-451)
__device__ void seq_step2(PairCtx& c) {
  Ring& P = c.R[0];
  Ring& Q = c.R[1];
  for (int s = 0; s < P.m; ++s) {
    if (!P.it[s] || (P.lb[s] != L_LEFT_ON && P.lb[s] != L_RIGHT_ON)) continue;
    int x = P.lb[s] == L_LEFT_ON ? R_LEFT : R_RIGHT;
    int X = s, I = s, guard = P.m + 1;
    do {
      P.lb[I] = L_NONE;
      if (P.nb[I] >= 0) Q.lb[P.nb[I]] = L_NONE;
      I = P.nx[I];
    } while (P.lb[I] == L_ON_ON && --guard > 0);
    int y = P.lb[I] == L_ON_LEFT ? R_LEFT : R_RIGHT;
    int8_t ct = (x != y) ? L_DELAYED_CROSSING : L_DELAYED_BOUNCING;
    P.lb[X] = ct; P.lb[I] = ct;
    if (P.nb[X] >= 0) Q.lb[P.nb[X]] = ct;
    if (P.nb[I] >= 0) Q.lb[P.nb[I]] = ct;
  }
}

// step 3.5: components without crossings (polyclip.h:474-541)
__device__ void seq_step35(PairCtx& c) {
  for (int sd = 0; sd < 2; ++sd) {
    Ring& A = c.R[sd];
    bool none = true, allOn = true;
    for (int v = 0; v < A.m; ++v) {
      int8_t l = A.lb[v];
      if (l != L_ON_ON) allOn = false;
      if (A.it[v]) {
        if (l == L_CROSSING || l == L_DELAYED_CROSSING) none = false;
        if (c.uni && (l == L_BOUNCING || l == L_DELAYED_BOUNCING)) none = false;
      }
    }
    c.noInter[sd] = none;
    c.ident[sd] = none && allOn;
  }
  for (int sd = 0; sd < 2; ++sd) {
    if (!c.noInter[sd] || c.ident[sd]) continue;
    Ring& A = c.R[sd];
    Ring& B = c.R[1 - sd];
    bool mid;
    int v = first_non_intersection(A, B, mid);
    if (v < 0) continue;
    double px = A.x[v], py = A.y[v];
    if (mid) { int n = A.nx[v]; px = 0.5 * (A.x[v] + A.x[n]); py = 0.5 * (A.y[v] + A.y[n]); }
    bool inside = point_in_ring(B, px, py, -1);
    if (inside ^ c.uni) push_ring(c.O, A);
  }
  if (c.ident[0] && c.ident[1]) push_ring(c.O, c.R[0]);
}

// step 4: entry/exit flags (polyclip.h:549-655)
__device__ bool seq_step4(PairCtx& c) {
  for (int sd = 0; sd < 2; ++sd) {
    if (c.noInter[sd]) continue;
    Ring& A = c.R[sd];
    Ring& B = c.R[1 - sd];
    bool mid;
    int V = first_non_intersection(A, B, mid);
    if (V < 0) continue;
    if (mid) {
      int n = A.nx[V];
      int T = add_vertex(A, 0.5 * (A.x[V] + A.x[n]), 0.5 * (A.y[V] + A.y[n]));
      if (T < 0) { fail(c, DEV_CAPACITY); return false; }
      insert_after(A, T, V);
      V = T;
    }
    // the Q pass sees P's temporary vertex; P's pass cannot see Q's (not yet added)
    int8_t st = point_in_ring(B, A.x[V], A.y[V], -1) ? E_EXIT : E_ENTRY;
    bool first = true;
    int I = A.nx[V], guard = A.used + 1;
    while (I != V && --guard > 0) {
      if (A.it[I]) {
        int8_t l = A.lb[I];
        if (l == L_CROSSING) { A.ee[I] = st; st = toggled(st); }
        if (A.lb[I] == L_BOUNCING && ((st == E_EXIT) ^ c.uni)) A.fl[I] |= 1;
        if (A.lb[I] == L_DELAYED_CROSSING) {
          A.ee[I] = st;
          if (first) { if ((st == E_EXIT) ^ c.uni) A.lb[I] = L_CROSSING; first = false; }
          else {
            if ((st == E_ENTRY) ^ c.uni) A.lb[I] = L_CROSSING;
            first = true;
            st = toggled(st);
          }
        }
        if (A.lb[I] == L_DELAYED_BOUNCING) {
          A.ee[I] = st;
          if (first) { if ((st == E_EXIT) ^ c.uni) A.fl[I] |= 2; first = false; }
          else { if ((st == E_ENTRY) ^ c.uni) A.fl[I] |= 2; first = true; }
          st = toggled(st);
        }
      }
      I = A.nx[I];
    }
  }
  return true;
}

// step 5: split vertex pairs (polyclip.h:661-714)
__device__ bool seq_step5(PairCtx& c) {
  Ring& P = c.R[0];
  Ring& Q = c.R[1];
  const int pm0 = P.used;
  for (int ip = 0; ip < pm0; ++ip) {
    if (!(P.fl[ip] & 1)) continue;
    int iq = P.nb[ip];
    if (iq < 0 || !(Q.fl[iq] & 1)) continue;
    int vp = add_vertex(P, P.x[ip], P.y[ip]);
    int vq = add_vertex(Q, Q.x[iq], Q.y[iq]);
    if (vp < 0 || vq < 0) { fail(c, DEV_CAPACITY); return false; }
    double sP = area2(P.x[P.pv[ip]], P.y[P.pv[ip]], P.x[ip], P.y[ip], P.x[P.nx[ip]], P.y[P.nx[ip]]);
    double sQ = area2(Q.x[Q.pv[iq]], Q.y[Q.pv[iq]], Q.x[iq], Q.y[iq], Q.x[Q.nx[iq]], Q.y[Q.nx[iq]]);
    if (sP * sQ > 0) {
      P.nb[ip] = vq; Q.nb[vq] = ip; P.it[ip] = 1; Q.it[vq] = 1;
      Q.nb[iq] = vp; P.nb[vp] = iq; Q.it[iq] = 1; P.it[vp] = 1;
    } else {
      P.nb[vp] = vq; Q.nb[vq] = vp; P.it[vp] = 1; Q.it[vq] = 1;
    }
    insert_after(P, vp, ip);
    insert_after(Q, vq, iq);
    int8_t e1 = c.uni ? E_ENTRY : E_EXIT, e2 = c.uni ? E_EXIT : E_ENTRY;
    P.ee[ip] = e1; P.ee[vp] = e2; Q.ee[iq] = e1; Q.ee[vq] = e2;
    P.lb[ip] = L_CROSSING; P.lb[vp] = L_CROSSING; Q.lb[iq] = L_CROSSING; Q.lb[vq] = L_CROSSING;
  }
  return true;
}

// step 6: crossing candidates (polyclip.h:723-734)
__device__ void seq_step6(PairCtx& c) {
  Ring& P = c.R[0];
  Ring& Q = c.R[1];
  for (int ip = 0; ip < P.m; ++ip) {
    if (!(P.fl[ip] & 2)) continue;
    int iq = P.nb[ip];
    if (iq >= 0 && (Q.fl[iq] & 2)) { P.lb[ip] = L_CROSSING; Q.lb[iq] = L_CROSSING; }
  }
}

// tracing (polyclip.h:743-783): starts at unvisited CROSSING vertices of P in ring order
// from slot 0; visited vertices are marked by clearing their intersection flag.
__device__ bool seq_trace(PairCtx& c) {
  Ring& P = c.R[0];
  OutRegion& O = c.O;
  long long budget = 4ll * (c.R[0].used + c.R[1].used) + 16;
  int I = 0;
  bool have = P.it[I] && P.lb[I] == L_CROSSING;
  if (!have) {
    int guard = P.used + 1;
    do { I = P.nx[I]; } while (!(P.it[I] && P.lb[I] == L_CROSSING) && I != 0 && --guard > 0);
    have = I != 0 && guard > 0;
  }
  while (have) {
    O.begin();
    int side = 0, V = I;
    P.it[V] = 0;
    do {
      Ring& C = c.R[side];
      int8_t st = toggled(C.ee[V]);
      do {
        if (--budget < 0) { fail(c, DEV_TRACE); return false; }
        V = ((st == E_EXIT) ^ c.uni) ? C.nx[V] : C.pv[V];
        C.it[V] = 0;
        O.push(C.x[V], C.y[V]);
      } while (!(C.ee[V] == st) && !(side == 0 && V == I));
      if (!(side == 0 && V == I)) {
        int nb = C.nb[V];
        if (nb < 0) { fail(c, DEV_TRACE); return false; }
        V = nb;
        side = 1 - side;
        c.R[side].it[V] = 0;
      }
    } while (!(side == 0 && V == I));
    O.end();
    int guard = P.used + 1;
    do { I = P.nx[I]; } while (!(P.it[I] && P.lb[I] == L_CROSSING) && I != 0 && --guard > 0);
    have = I != 0 && guard > 0;
  }
  if (O.overflow) { fail(c, DEV_CAPACITY); return false; }
  return true;
}

// clean-up of one component (polyclip.h:791-807): drop the first vertex while it is
// collinear with its ring neighbours, then one forward pass that removes every vertex
// collinear with the last kept vertex and its original successor.  Reads n vertices at
// src, writes the kept ones at dst (dst <= src, ascending); returns how many were kept.
__device__ int seq_cleanup_component(const double* src, double* dst, int n, double eps) {
  if (n == 0) return 0;
  const double lx = src[2 * (n - 1)], ly = src[2 * (n - 1) + 1];
  int r = 0;
  while (r < n) {
    int nxt = (r + 1 < n) ? r + 1 : r;    // a lone vertex is its own neighbour
    double a = area2(lx, ly, src[2 * r], src[2 * r + 1], src[2 * nxt], src[2 * nxt + 1]);
    if (r == n - 1) a = 0.0;              // ring of the last vertex alone: A(v,v,v)
    if (fabs(a) < eps) ++r; else break;
  }
  if (r >= n) return 0;
  double kx = src[2 * r], ky = src[2 * r + 1];
  const double rx = kx, ry = ky;
  int kept = 1;
  dst[0] = kx; dst[1] = ky;
  for (int j = r + 1; j < n; ++j) {
    double vx = src[2 * j], vy = src[2 * j + 1];
    double nx = (j + 1 < n) ? src[2 * (j + 1)] : rx, ny = (j + 1 < n) ? src[2 * (j + 1) + 1] : ry;
    if (fabs(area2(kx, ky, vx, vy, nx, ny)) < eps) continue;
    dst[2 * kept] = vx; dst[2 * kept + 1] = vy;
    ++kept;
    kx = vx; ky = vy;
  }
  return kept;
}

__device__ void seq_cleanup(PairCtx& c, int32_t* outNC, int64_t* outNV) {
  OutRegion& O = c.O;
  int64_t vin = 0, vout = 0;
  int nc = 0;
  for (int k = 0; k < O.nc; ++k) {
    const int n = O.csz[k];
    int kept = seq_cleanup_component(O.xy + 2 * vin, O.xy + 2 * vout, n, c.eps_clean);
    vin += n;
    if (kept == 0) continue;
    O.csz[nc++] = kept;
    vout += kept;
  }
  *outNC = nc;
  *outNV = vout;
}

// the whole pair from `step` on (1: everything, 2: after the initial labels)
__device__ void seq_pair_from(PairCtx& c, int step, int32_t* outNC, int64_t* outNV) {
  if (step <= 1) seq_step1(c);
  seq_step2(c);
  seq_step35(c);
  if (!seq_step4(c) || !seq_step5(c)) return;
  seq_step6(c);
  if (!seq_trace(c)) return;
  seq_cleanup(c, outNC, outNV);
}

// ================================================================ warp phases
constexpr unsigned kFull = 0xffffffffu;

// winding increment of edge (P0,P1) for point R: polygon.h:433-444
__device__ __forceinline__ int wind(double P0x, double P0y, double P1x, double P1y, double Rx, double Ry) {
  if ((P0y < Ry) == (P1y < Ry)) return 0;
  int d = 2 * (P1y > P0y) - 1;
  if (P0x >= Rx) {
    if (P1x > Rx) return d;
    return ((area2(P0x, P0y, P1x, P1y, Rx, Ry) > 0) == (P1y > P0y)) ? d : 0;
  }
  if (P1x > Rx) return ((area2(P0x, P0y, P1x, P1y, Rx, Ry) > 0) == (P1y > P0y)) ? d : 0;
  return 0;
}

// polygon.h:427-448 over ring B in slot order; `after`/`T`: a temporary vertex T inserted
// after slot `after` (or -1)
__device__ bool warp_point_in_ring(const Ring& B, double Rx, double Ry, int after, int T) {
  int w = 0;
  for (int s = lane_id(); s < B.m; s += 32) {
    int n = (s + 1 < B.m) ? s + 1 : 0;
    if (s == after) {
      w += wind(B.x[s], B.y[s], B.x[T], B.y[T], Rx, Ry);
      w += wind(B.x[T], B.y[T], B.x[n], B.y[n], Rx, Ry);
    } else {
      w += wind(B.x[s], B.y[s], B.x[n], B.y[n], Rx, Ry);
    }
  }
  w = warp_sum(w);
  return (w % 2) != 0;
}

// first slot s >= from (slot order, s < n) where pred(s); n if none
template <class F>
__device__ int warp_find_first(int from, int n, F pred) {
  for (int b = from; b < n; b += 32) {
    int s = b + lane_id();
    unsigned m = __ballot_sync(kFull, s < n && pred(s));
    if (m) return b + __ffs(m) - 1;
  }
  return n;
}

__device__ bool warp_links_one_to_one(const Ring& P, const Ring& Q) {
  bool ok = true;
  for (int s = lane_id(); s < P.m; s += 32)
    if (P.it[s]) { int nb = P.nb[s]; if (nb < 0 || nb >= Q.m || Q.nb[nb] != s) ok = false; }
  for (int s = lane_id(); s < Q.m; s += 32)
    if (Q.it[s]) { int nb = Q.nb[s]; if (nb < 0 || nb >= P.m || P.nb[nb] != s) ok = false; }
  return __all_sync(kFull, ok);
}

__device__ void warp_step1(PairCtx& c) {
  Ring& P = c.R[0];
  Ring& Q = c.R[1];
  for (int s = lane_id(); s < P.m; s += 32) {
    if (!P.it[s]) continue;
    int nb = P.nb[s];
    int pm = (s > 0) ? s - 1 : P.m - 1, pp = (s + 1 < P.m) ? s + 1 : 0;
    int a = rel_position(P, Q, (nb > 0) ? nb - 1 : Q.m - 1, pm, s, pp);
    int b = rel_position(P, Q, (nb + 1 < Q.m) ? nb + 1 : 0, pm, s, pp);
    int8_t L = initial_label(a, b);
    if (L != L_NONE) { P.lb[s] = L; Q.lb[nb] = L; }
  }
  __syncwarp();
}

// Chains run from a LEFT_ON/RIGHT_ON vertex over ON_ON vertices to an ON_LEFT/ON_RIGHT
// vertex.  When every chain ends so, chains are disjoint and can be resolved in parallel
// with the sequential result; otherwise returns false and nothing is changed.
__device__ bool warp_step2(PairCtx& c) {
  Ring& P = c.R[0];
  Ring& Q = c.R[1];
  const int m = P.m;
  bool ok = true;
  for (int s = lane_id(); s < m; s += 32) {
    if (!P.it[s] || (P.lb[s] != L_LEFT_ON && P.lb[s] != L_RIGHT_ON)) continue;
    int I = (s + 1 < m) ? s + 1 : 0, guard = m;
    while (P.lb[I] == L_ON_ON && --guard > 0) I = (I + 1 < m) ? I + 1 : 0;
    if ((P.lb[I] != L_ON_LEFT && P.lb[I] != L_ON_RIGHT) || !P.it[I]) ok = false;
  }
  if (!__all_sync(kFull, ok)) return false;
  for (int s = lane_id(); s < m; s += 32) {
    int8_t l0 = P.lb[s];
    if (!P.it[s] || (l0 != L_LEFT_ON && l0 != L_RIGHT_ON)) continue;
    int x = l0 == L_LEFT_ON ? R_LEFT : R_RIGHT;
    int I = (s + 1 < m) ? s + 1 : 0;
    Q.lb[P.nb[s]] = L_NONE;
    while (P.lb[I] == L_ON_ON) {
      P.lb[I] = L_NONE;
      Q.lb[P.nb[I]] = L_NONE;
      I = (I + 1 < m) ? I + 1 : 0;
    }
    int y = P.lb[I] == L_ON_LEFT ? R_LEFT : R_RIGHT;
    int8_t ct = (x != y) ? L_DELAYED_CROSSING : L_DELAYED_BOUNCING;
    P.lb[s] = ct; P.lb[I] = ct;
    Q.lb[P.nb[s]] = ct; Q.lb[P.nb[I]] = ct;
  }
  __syncwarp();
  return true;
}

// copies ring A (slot order, no added vertices) as one output component
__device__ void warp_push_ring(OutRegion& O, const Ring& A) {
  O.begin();
  if (O.overflow) return;
  if (O.nv + A.m > O.vcap) { O.overflow = true; return; }
  for (int s = lane_id(); s < A.m; s += 32) { O.xy[2 * (O.nv + s)] = A.x[s]; O.xy[2 * (O.nv + s) + 1] = A.y[s]; }
  if (lane_id() == 0) O.csz[O.nc] = A.m;
  O.nv += A.m;
  O.end();
  __syncwarp();
}

// first non-intersection slot (slot order = ring order before any insertion), else the
// first vertex whose edge to the next one is not collinear with the other polygon
// (polygon.h:480-512); returns -1 if none
__device__ int warp_first_non_intersection(const Ring& A, const Ring& B, bool& mid) {
  mid = false;
  int v = warp_find_first(0, A.m, [&](int s) { return !A.it[s]; });
  if (v < A.m) return v;
  // B's own links: B may already hold its temporary vertex when A is Q
  v = warp_find_first(0, A.m, [&](int s) {
    int nb = A.nb[s], nx = A.nx[s];
    return nb >= 0 && A.nb[nx] != B.pv[nb] && A.nb[nx] != B.nx[nb];
  });
  if (v < A.m) { mid = true; return v; }
  return -1;
}

__device__ void warp_step35(PairCtx& c) {
  for (int sd = 0; sd < 2; ++sd) {
    Ring& A = c.R[sd];
    bool none = true, allOn = true;
    for (int v = lane_id(); v < A.m; v += 32) {
      int8_t l = A.lb[v];
      if (l != L_ON_ON) allOn = false;
      if (A.it[v]) {
        if (l == L_CROSSING || l == L_DELAYED_CROSSING) none = false;
        if (c.uni && (l == L_BOUNCING || l == L_DELAYED_BOUNCING)) none = false;
      }
    }
    none = __all_sync(kFull, none);
    allOn = __all_sync(kFull, allOn);
    c.noInter[sd] = none;
    c.ident[sd] = none && allOn;
  }
  for (int sd = 0; sd < 2; ++sd) {
    if (!c.noInter[sd] || c.ident[sd]) continue;
    Ring& A = c.R[sd];
    Ring& B = c.R[1 - sd];
    bool mid;
    int v = warp_first_non_intersection(A, B, mid);
    if (v < 0) continue;
    double px = A.x[v], py = A.y[v];
    if (mid) { int n = (v + 1 < A.m) ? v + 1 : 0; px = 0.5 * (A.x[v] + A.x[n]); py = 0.5 * (A.y[v] + A.y[n]); }
    bool inside = warp_point_in_ring(B, px, py, -1, -1);
    if (inside ^ c.uni) warp_push_ring(c.O, A);
  }
  if (c.ident[0] && c.ident[1]) warp_push_ring(c.O, c.R[0]);
}

// Entry/exit flags as a warp prefix scan over the ring from the start vertex: the status
// at a vertex is the start status toggled once per earlier CROSSING, DELAYED_BOUNCING and
// second-of-a-chain DELAYED_CROSSING; "first chain vertex" alternates over the DELAYED
// vertices met (polyclip.h:582-653).
__device__ bool warp_step4(PairCtx& c, int tempAfter[2], int tempSlot[2]) {
  for (int sd = 0; sd < 2; ++sd) {
    tempAfter[sd] = -1;
    tempSlot[sd] = -1;
  }
  for (int sd = 0; sd < 2; ++sd) {
    if (c.noInter[sd]) continue;
    Ring& A = c.R[sd];
    Ring& B = c.R[1 - sd];
    bool mid;
    int V0 = warp_first_non_intersection(A, B, mid);
    if (V0 < 0) continue;
    double qx = A.x[V0], qy = A.y[V0];
    if (mid) {
      int T = -1;
      if (lane_id() == 0) {
        T = add_vertex(A, 0.5 * (A.x[V0] + A.x[(V0 + 1 < A.m) ? V0 + 1 : 0]),
                       0.5 * (A.y[V0] + A.y[(V0 + 1 < A.m) ? V0 + 1 : 0]));
        if (T >= 0) insert_after(A, T, V0);
      }
      T = __shfl_sync(kFull, T, 0);
      A.used = __shfl_sync(kFull, A.used, 0);
      __syncwarp();
      if (T < 0) { if (lane_id() == 0) fail(c, DEV_CAPACITY); return false; }
      tempAfter[sd] = V0;
      tempSlot[sd] = T;
      qx = A.x[T];
      qy = A.y[T];
    }
    // the Q pass tests against P's ring including P's temporary vertex
    int8_t st0 = (sd == 1 ? warp_point_in_ring(B, qx, qy, tempAfter[0], tempSlot[0])
                          : warp_point_in_ring(B, qx, qy, -1, -1)) ? E_EXIT : E_ENTRY;
    int carryD = 0, carryT = 0;
    const int m = A.m;
    for (int b = 0; b < m; b += 32) {
      int j = b + lane_id();
      int s = -1;
      int8_t L = L_NONE;
      bool inter = false;
      if (j < m) {
        s = V0 + 1 + j;
        if (s >= m) s -= m;
        inter = A.it[s];
        L = inter ? A.lb[s] : L_NONE;
      }
      int d = inter && (L == L_DELAYED_CROSSING || L == L_DELAYED_BOUNCING);
      int dIncl = warp_incl_scan(d);
      bool first = ((carryD + dIncl - d) & 1) == 0;
      int t = inter && (L == L_CROSSING || L == L_DELAYED_BOUNCING || (L == L_DELAYED_CROSSING && !first));
      int tIncl = warp_incl_scan(t);
      int8_t st = ((carryT + tIncl - t) & 1) ? toggled(st0) : st0;
      if (inter) {
        if (L == L_CROSSING) A.ee[s] = st;
        else if (L == L_BOUNCING) { if ((st == E_EXIT) ^ c.uni) A.fl[s] |= 1; }
        else if (L == L_DELAYED_CROSSING) {
          A.ee[s] = st;
          if (first) { if ((st == E_EXIT) ^ c.uni) A.lb[s] = L_CROSSING; }
          else if ((st == E_ENTRY) ^ c.uni) A.lb[s] = L_CROSSING;
        } else if (L == L_DELAYED_BOUNCING) {
          A.ee[s] = st;
          if (first) { if ((st == E_EXIT) ^ c.uni) A.fl[s] |= 2; }
          else if ((st == E_ENTRY) ^ c.uni) A.fl[s] |= 2;
        }
      }
      carryD += __shfl_sync(kFull, dIncl, 31);
      carryT += __shfl_sync(kFull, tIncl, 31);
    }
    __syncwarp();
  }
  return true;
}

__device__ bool warp_any_split(const Ring& P, const Ring& Q) {
  bool any = false;
  for (int s = lane_id(); s < P.m; s += 32)
    if (P.fl[s] & 1) { int nb = P.nb[s]; if (nb >= 0 && (Q.fl[nb] & 1)) any = true; }
  return __any_sync(kFull, any);
}

__device__ void warp_step6(PairCtx& c) {
  Ring& P = c.R[0];
  Ring& Q = c.R[1];
  for (int ip = lane_id(); ip < P.m; ip += 32) {
    if (!(P.fl[ip] & 2)) continue;
    int iq = P.nb[ip];
    if (iq >= 0 && (Q.fl[iq] & 2)) { P.lb[ip] = L_CROSSING; Q.lb[iq] = L_CROSSING; }
  }
  __syncwarp();
}

// Tracing when neither ring has added vertices (rings in slot order): each run from V to
// the next vertex with the target entry/exit flag (or back at the start) is found with a
// warp ballot and copied with coalesced stores.
__device__ bool warp_trace(PairCtx& c) {
  Ring& P = c.R[0];
  OutRegion& O = c.O;
  long long budget = 4ll * (c.R[0].used + c.R[1].used) + 16;
  int from = 0;
  for (;;) {
    int I = warp_find_first(from, P.m, [&](int s) { return P.it[s] && P.lb[s] == L_CROSSING; });
    if (I >= P.m) break;
    O.begin();
    if (O.overflow) { if (lane_id() == 0) fail(c, DEV_CAPACITY); return false; }
    int side = 0, V = I;
    if (lane_id() == 0) P.it[V] = 0;
    __syncwarp();
    do {
      Ring& C = c.R[side];
      const int m = C.m;
      int8_t st = toggled(C.ee[V]);
      const int dir = ((st == E_EXIT) ^ c.uni) ? 1 : -1;
      int L = -1;
      for (int j0 = 1; j0 <= m && L < 0; j0 += 32) {
        int j = j0 + lane_id();
        bool hit = false;
        if (j <= m) {
          int w = V + dir * (j % m);
          w = (w % m + m) % m;
          hit = (C.ee[w] == st) || (side == 0 && w == I);
        }
        unsigned msk = __ballot_sync(kFull, hit);
        if (msk) L = j0 + __ffs(msk) - 1;
      }
      if (L < 0) { if (lane_id() == 0) fail(c, DEV_TRACE); return false; }
      budget -= L;
      if (budget < 0) { if (lane_id() == 0) fail(c, DEV_TRACE); return false; }
      if (O.nv + L > O.vcap) { if (lane_id() == 0) fail(c, DEV_CAPACITY); return false; }
      for (int j0 = 1; j0 <= L; j0 += 32) {
        int j = j0 + lane_id();
        if (j <= L) {
          int w = V + dir * (j % m);
          w = (w % m + m) % m;
          C.it[w] = 0;
          O.xy[2 * (O.nv + j - 1)] = C.x[w];
          O.xy[2 * (O.nv + j - 1) + 1] = C.y[w];
        }
      }
      O.nv += L;
      if (lane_id() == 0) O.csz[O.nc] += L;
      int W = V + dir * (L % m);
      V = (W % m + m) % m;
      __syncwarp();
      if (!(side == 0 && V == I)) {
        int nb = C.nb[V];
        if (nb < 0) { if (lane_id() == 0) fail(c, DEV_TRACE); return false; }
        V = nb;
        side = 1 - side;
        if (lane_id() == 0) c.R[side].it[V] = 0;
        __syncwarp();
      }
    } while (!(side == 0 && V == I));
    O.end();
    from = I + 1;
  }
  return true;
}

// Clean-up: a component where no vertex is collinear with its two ring neighbours keeps
// every vertex (the sequential pass would remove nothing), so it is only moved into place;
// any other component is cleaned by one lane with the sequential pass.
__device__ void warp_cleanup(PairCtx& c, int32_t* outNC, int64_t* outNV) {
  OutRegion& O = c.O;
  int64_t vin = 0, vout = 0;
  int nc = 0;
  for (int k = 0; k < O.nc; ++k) {
    const int n = O.csz[k];
    const double* src = O.xy + 2 * vin;
    double* dst = O.xy + 2 * vout;
    bool flag = false;
    for (int j = lane_id(); j < n; j += 32) {
      int p = (j > 0) ? j - 1 : n - 1, q = (j + 1 < n) ? j + 1 : 0;
      if (fabs(area2(src[2 * p], src[2 * p + 1], src[2 * j], src[2 * j + 1], src[2 * q], src[2 * q + 1])) <
          c.eps_clean)
        flag = true;
    }
    flag = __any_sync(kFull, flag);
    int kept;
    if (!flag) {
      if (dst != src) {
        for (int b = 0; b < 2 * n; b += 32) {
          int i = b + lane_id();
          double v = (i < 2 * n) ? src[i] : 0.0;
          __syncwarp();
          if (i < 2 * n) dst[i] = v;
        }
      }
      kept = n;
    } else {
      kept = 0;
      if (lane_id() == 0) kept = seq_cleanup_component(src, dst, n, c.eps_clean);
      kept = __shfl_sync(kFull, kept, 0);
    }
    __syncwarp();
    vin += n;
    if (kept == 0) continue;
    if (lane_id() == 0) O.csz[nc] = kept;
    ++nc;
    vout += kept;
    __syncwarp();
  }
  if (lane_id() == 0) { *outNC = nc; *outNV = vout; }
}

// One warp per pair.  The warp phases give the sequential result whenever neighbour links
// are one-to-one (then labels written through a link never collide) and chains are well
// formed; otherwise lane 0 runs the sequential phases from the first one that could differ.
__global__ void __launch_bounds__(128)
label_trace_kernel(PairDev D, int64_t K, const int32_t* __restrict__ mP, const int32_t* __restrict__ mQ,
                   const int64_t* __restrict__ regP, const int64_t* __restrict__ regQ,
                   const int64_t* __restrict__ regSizeP, const int64_t* __restrict__ regSizeQ,
                   RingSet SP, RingSet SQ, double* __restrict__ outXY, const int64_t* __restrict__ outVOff,
                   const int64_t* __restrict__ outVCap, int32_t* __restrict__ outCsz,
                   const int64_t* __restrict__ outCOff, const int32_t* __restrict__ outCCap,
                   int32_t* __restrict__ outNC, int64_t* __restrict__ outNV, ClipParams prm, int* err) {
  int64_t k = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (k >= K) return;
  const bool lane0 = lane_id() == 0;
  if (lane0) { outNC[k] = 0; outNV[k] = 0; }
  if (D.status[k] != 0) return;
  PairCtx c;
  c.R[0] = ring_of(SP, regP[k], mP[k], (int)regSizeP[k]);
  c.R[1] = ring_of(SQ, regQ[k], mQ[k], (int)regSizeQ[k]);
  c.O.xy = outXY + 2 * outVOff[k]; c.O.csz = outCsz + outCOff[k]; c.O.vcap = outVCap[k]; c.O.ccap = outCCap[k];
  c.O.nv = 0; c.O.nc = 0; c.O.overflow = false;
  c.uni = prm.union_mode != 0;
  c.eps_clean = prm.eps_clean;
  c.err = err;
  c.status = D.status + k;
  c.noInter[0] = c.noInter[1] = c.ident[0] = c.ident[1] = false;

  if (!warp_links_one_to_one(c.R[0], c.R[1])) {
    if (lane0) seq_pair_from(c, 1, outNC + k, outNV + k);
    return;
  }
  warp_step1(c);
  if (!warp_step2(c)) {
    if (lane0) seq_pair_from(c, 2, outNC + k, outNV + k);
    return;
  }
  warp_step35(c);
  int tempAfter[2], tempSlot[2];
  if (!warp_step4(c, tempAfter, tempSlot)) return;
  if (warp_any_split(c.R[0], c.R[1])) {
    bool ok = true;
    if (lane0) ok = seq_step5(c);
    ok = __shfl_sync(kFull, (int)ok, 0);
    c.R[0].used = __shfl_sync(kFull, c.R[0].used, 0);
    c.R[1].used = __shfl_sync(kFull, c.R[1].used, 0);
    __syncwarp();
    if (!ok) return;
  }
  warp_step6(c);
  const bool added = c.R[0].used != c.R[0].m || c.R[1].used != c.R[1].m;
  if (added) {
    // vertices were added to a ring: trace through the next/prev links on one lane
    int ok = 1;
    if (lane0) ok = seq_trace(c) ? 1 : 0;
    ok = __shfl_sync(kFull, ok, 0);
    c.O.nv = __shfl_sync(kFull, (long long)c.O.nv, 0);
    c.O.nc = __shfl_sync(kFull, c.O.nc, 0);
    __syncwarp();
    if (!ok) return;
  } else if (!warp_trace(c)) {
    return;
  }
  if (c.O.overflow) {
    if (lane0) fail(c, DEV_CAPACITY);
    return;
  }
  warp_cleanup(c, outNC + k, outNV + k);
}

// ---------------------------------------------------------------- G8 compaction
__global__ void out_sizes_kernel(const int32_t* __restrict__ mP, const int32_t* __restrict__ mQ,
                                 const int32_t* __restrict__ nrec, const int32_t* __restrict__ status,
                                 int64_t K, int64_t* __restrict__ vcap, int32_t* __restrict__ ccap) {
  int64_t k = (int64_t)blockIdx.x * kThreads + threadIdx.x;
  if (k >= K) return;
  if (status[k] != 0) { vcap[k] = 0; ccap[k] = 0; return; }
  int64_t ext = (int64_t)mP[k] + mQ[k] + 4 * ((int64_t)nrec[k] + 1);
  vcap[k] = 2 * ext + 16;
  ccap[k] = mP[k] + 2 * nrec[k] + 8;
}

__global__ void __launch_bounds__(kThreads)
out_compact_kernel(int64_t K, const double* __restrict__ xy, const int64_t* __restrict__ vOff,
                   const int32_t* __restrict__ csz, const int64_t* __restrict__ cOff,
                   const int32_t* __restrict__ nc, const int64_t* __restrict__ nv,
                   const int64_t* __restrict__ fVOff, const int64_t* __restrict__ fCOff,
                   double* __restrict__ oxy, int32_t* __restrict__ ocsz) {
  int64_t w = ((int64_t)blockIdx.x * kThreads + threadIdx.x) >> 5;
  if (w >= K) return;
  const double* s = xy + 2 * vOff[w];
  double* d = oxy + 2 * fVOff[w];
  for (int64_t i = lane_id(); i < 2 * nv[w]; i += 32) d[i] = s[i];
  for (int i = lane_id(); i < nc[w]; i += 32) ocsz[fCOff[w] + i] = csz[cOff[w] + i];
}

}  // namespace

int run_clip(const LayerDev& Lb, const LayerDev& Lo, const int32_t* d_pid, const int32_t* d_qid,
             int64_t K, const ClipParams& prm, Arena& A, ClipDev& C, int* d_err, int64_t* hs,
             cudaStream_t s, Marks* mk) {
  Marks dummy;
  if (!mk) mk = &dummy;
  C = ClipDev();
  mk->mark("clip:start", s);
  C.n_pairs = K;
  if (K <= 0) return ST_OK;
  auto sync = [&]() { return cudaStreamSynchronize(s) == cudaSuccess; };
  // layer MBRs (same definition as the join's)
  double* mb = A.take_n<double>(4 * Lb.n);
  double* mo = A.take_n<double>(4 * Lo.n);
  if (!mb || !mo) return ST_OUT_OF_MEMORY;
  layer_mbrs(Lb, mb, s);
  layer_mbrs(Lo, mo, s);
  // ---- G0 setup
  PairDev D;
  D.pS = A.take_n<int64_t>(K); D.qS = A.take_n<int64_t>(K);
  D.nP = A.take_n<int32_t>(K); D.nQ = A.take_n<int32_t>(K);
  D.pSide = A.take_n<int8_t>(K); D.cmbr = A.take_n<double>(4 * K);
  C.status = D.status = A.take_n<int32_t>(K);
  C.swapped = A.take_n<int32_t>(K);
  C.count1 = A.take_n<int64_t>(K);
  int32_t* cP = A.take_n<int32_t>(K);
  int32_t* cQ = A.take_n<int32_t>(K);
  int64_t* offP = A.take_n<int64_t>(K);
  int64_t* offQ = A.take_n<int64_t>(K);
  int64_t* nchunk = A.take_n<int64_t>(K);
  int64_t* chunkOff = A.take_n<int64_t>(K);
  int64_t* eoffP = A.take_n<int64_t>(K);
  int64_t* eoffQ = A.take_n<int64_t>(K);
  int64_t* tot = A.take_n<int64_t>(16);
  void* stK = A.take(scan_temp_bytes(K));
  if (!D.pS || !D.qS || !D.nP || !D.nQ || !D.pSide || !D.cmbr || !D.status || !C.swapped || !C.count1 ||
      !cP || !cQ || !offP || !offQ || !nchunk || !chunkOff || !eoffP || !eoffQ || !tot || !stK)
    return ST_OUT_OF_MEMORY;
  { setup_kernel<<<blocks_for(K), kThreads, 0, s>>>(Lb, Lo, d_pid, d_qid, K, mb, mo, D, C.swapped, prm.no_swap); note_launch(); }
  // ---- G1 edge filter
  { edge_filter_kernel<0><<<blocks_for_warps(K), kThreads, 0, s>>>(Lb, Lo, D, K, cP, cQ, nullptr, nullptr,
                                                                 nullptr, nullptr); note_launch(); }
  exclusive_scan_i32(cP, offP, K, tot + 0, stK, d_err, s);
  exclusive_scan_i32(cQ, offQ, K, tot + 1, stK, d_err, s);
  exclusive_scan_i32(D.nP, eoffP, K, tot + 2, stK, d_err, s);
  exclusive_scan_i32(D.nQ, eoffQ, K, tot + 3, stK, d_err, s);
  { chunk_count_kernel<<<blocks_for(K), kThreads, 0, s>>>(cP, cQ, K, nchunk); note_launch(); }
  exclusive_scan_i64(nchunk, chunkOff, K, tot + 4, stK, d_err, s);
  mk->mark("clip:setup+filter", s);
  cudaMemcpyAsync(hs, tot, 5 * sizeof(int64_t), cudaMemcpyDeviceToHost, s);
  if (!sync()) return ST_CUDA_ERROR;
  const int64_t nLP = hs[0], nLQ = hs[1], nEP = hs[2], nEQ = hs[3], nCh = hs[4];
  int32_t* LP = A.take_n<int32_t>(nLP);
  int32_t* LQ = A.take_n<int32_t>(nLQ);
  int32_t* chunkRec = A.take_n<int32_t>(nCh);
  int32_t* chunkQ = A.take_n<int32_t>(nCh);
  int64_t* recScan = A.take_n<int64_t>(nCh);
  int64_t* qScan = A.take_n<int64_t>(nCh);
  void* stC = A.take(scan_temp_bytes(std::max<int64_t>(nCh, 1)));
  if (!LP || !LQ || !chunkRec || !chunkQ || !recScan || !qScan || !stC) return ST_OUT_OF_MEMORY;
  { edge_filter_kernel<1><<<blocks_for_warps(K), kThreads, 0, s>>>(Lb, Lo, D, K, cP, cQ, offP, offQ, LP, LQ); note_launch(); }
  // ---- G2 count
  Records R{};
  if (nCh > 0) {
    { intersect_kernel<0><<<blocks_for_warps(nCh), kThreads, 0, s>>>(
        Lb, Lo, D, K, chunkOff, nCh, cP, cQ, offP, offQ, LP, LQ, prm.eps, chunkRec, chunkQ, nullptr, R); note_launch(); }
    exclusive_scan_i32(chunkRec, recScan, nCh, tot + 5, stC, d_err, s);
    exclusive_scan_i32(chunkQ, qScan, nCh, tot + 6, stC, d_err, s);
  } else {
    cudaMemsetAsync(tot + 5, 0, 2 * sizeof(int64_t), s);
  }
  int64_t* recOff = A.take_n<int64_t>(K);
  int32_t* nrec = A.take_n<int32_t>(K);
  if (!recOff || !nrec) return ST_OUT_OF_MEMORY;
  { pair_records_kernel<<<blocks_for(K), kThreads, 0, s>>>(chunkOff, nchunk, recScan, qScan, chunkRec, chunkQ,
                                                         K, recOff, nrec, C.count1, D); note_launch(); }
  mk->mark("clip:count", s);
  cudaMemcpyAsync(hs, tot + 5, sizeof(int64_t), cudaMemcpyDeviceToHost, s);
  if (!sync()) return ST_CUDA_ERROR;
  const int64_t nR = hs[0];
  // ---- G3 emit
  R.p = A.take_n<int32_t>(nR); R.q = A.take_n<int32_t>(nR);
  R.a = A.take_n<double>(nR); R.b = A.take_n<double>(nR);
  R.t = A.take_n<int8_t>(nR); R.k = A.take_n<int32_t>(nR);
  if (!R.p || !R.q || !R.a || !R.b || !R.t || !R.k) return ST_OUT_OF_MEMORY;
  if (nCh > 0)
    { intersect_kernel<1><<<blocks_for_warps(nCh), kThreads, 0, s>>>(
        Lb, Lo, D, K, chunkOff, nCh, cP, cQ, offP, offQ, LP, LQ, prm.eps, nullptr, nullptr, recScan, R); note_launch(); }
  mk->mark("clip:emit", s);
  // ---- G4 ring layout
  int32_t* insP = A.take_n<int32_t>(nEP);
  int32_t* insQ = A.take_n<int32_t>(nEQ);
  int64_t* srcLinkP = A.take_n<int64_t>(nEP);
  int64_t* srcLinkQ = A.take_n<int64_t>(nEQ);
  int32_t* szP = A.take_n<int32_t>(nEP);
  int32_t* szQ = A.take_n<int32_t>(nEQ);
  int64_t* vposP = A.take_n<int64_t>(nEP);
  int64_t* vposQ = A.take_n<int64_t>(nEQ);
  int64_t* insBaseP = A.take_n<int64_t>(nEP);
  int64_t* insBaseQ = A.take_n<int64_t>(nEQ);
  int32_t* curP = A.take_n<int32_t>(nEP);
  int32_t* curQ = A.take_n<int32_t>(nEQ);
  int64_t* slotP = A.take_n<int64_t>(nR);
  int64_t* slotQ = A.take_n<int64_t>(nR);
  void* stE = A.take(scan_temp_bytes(std::max<int64_t>(std::max(nEP, nEQ), 1)));
  if (!insP || !insQ || !srcLinkP || !srcLinkQ || !szP || !szQ || !vposP || !vposQ || !insBaseP ||
      !insBaseQ || !curP || !curQ || !slotP || !slotQ || !stE)
    return ST_OUT_OF_MEMORY;
  cudaMemsetAsync(insP, 0, nEP * sizeof(int32_t), s);
  cudaMemsetAsync(insQ, 0, nEQ * sizeof(int32_t), s);
  cudaMemsetAsync(srcLinkP, 0, nEP * sizeof(int64_t), s);
  cudaMemsetAsync(srcLinkQ, 0, nEQ * sizeof(int64_t), s);
  cudaMemsetAsync(curP, 0, nEP * sizeof(int32_t), s);
  cudaMemsetAsync(curQ, 0, nEQ * sizeof(int32_t), s);
  if (nR > 0)
    { record_count_kernel<<<blocks_for(nR), kThreads, 0, s>>>(R, nR, eoffP, eoffQ, D.status, insP, insQ,
                                                            srcLinkP, srcLinkQ); note_launch(); }
  { edge_slots_kernel<<<blocks_for(nEP), kThreads, 0, s>>>(insP, nEP, szP); note_launch(); }
  { edge_slots_kernel<<<blocks_for(nEQ), kThreads, 0, s>>>(insQ, nEQ, szQ); note_launch(); }
  exclusive_scan_i32(szP, vposP, nEP, tot + 7, stE, d_err, s);
  exclusive_scan_i32(szQ, vposQ, nEQ, tot + 8, stE, d_err, s);
  exclusive_scan_i32(insP, insBaseP, nEP, tot + 9, stE, d_err, s);
  exclusive_scan_i32(insQ, insBaseQ, nEQ, tot + 10, stE, d_err, s);
  cudaMemcpyAsync(hs, tot + 7, 4 * sizeof(int64_t), cudaMemcpyDeviceToHost, s);
  if (!sync()) return ST_CUDA_ERROR;
  const int64_t vtotP = hs[0], vtotQ = hs[1], nInsP = hs[2], nInsQ = hs[3];
  int64_t* insListP = A.take_n<int64_t>(nInsP);
  int64_t* insListQ = A.take_n<int64_t>(nInsQ);
  int32_t* mP = A.take_n<int32_t>(K);
  int32_t* mQ = A.take_n<int32_t>(K);
  int64_t* regSizeP = A.take_n<int64_t>(K);
  int64_t* regSizeQ = A.take_n<int64_t>(K);
  int64_t* regP = A.take_n<int64_t>(K);
  int64_t* regQ = A.take_n<int64_t>(K);
  if (!insListP || !insListQ || !mP || !mQ || !regSizeP || !regSizeQ || !regP || !regQ) return ST_OUT_OF_MEMORY;
  if (nR > 0)
    { record_scatter_kernel<<<blocks_for(nR), kThreads, 0, s>>>(R, nR, eoffP, eoffQ, D.status, insBaseP, curP,
                                                              insListP, insBaseQ, curQ, insListQ); note_launch(); }
  { pair_ring_kernel<<<blocks_for(K), kThreads, 0, s>>>(eoffP, vposP, D.nP, nrec, D.status, K, nEP, vtotP, mP,
                                                      regSizeP); note_launch(); }
  { pair_ring_kernel<<<blocks_for(K), kThreads, 0, s>>>(eoffQ, vposQ, D.nQ, nrec, D.status, K, nEQ, vtotQ, mQ,
                                                      regSizeQ); note_launch(); }
  exclusive_scan_i64(regSizeP, regP, K, tot + 11, stK, d_err, s);
  exclusive_scan_i64(regSizeQ, regQ, K, tot + 12, stK, d_err, s);
  {
    int64_t* junk = A.take_n<int64_t>(K);
    if (!junk) return ST_OUT_OF_MEMORY;
    exclusive_scan_i32(mP, junk, K, tot + 13, stK, d_err, s);
    exclusive_scan_i32(mQ, junk, K, tot + 14, stK, d_err, s);
  }
  cudaMemcpyAsync(hs, tot + 11, 4 * sizeof(int64_t), cudaMemcpyDeviceToHost, s);
  if (!sync()) return ST_CUDA_ERROR;
  const int64_t regTotP = hs[0], regTotQ = hs[1];
  C.n_ring_vertices = hs[2] + hs[3];
  C.n_records = nR;
  auto take_ring = [&](int64_t n, RingSet& S) {
    S.x = A.take_n<double>(n); S.y = A.take_n<double>(n);
    S.nx = A.take_n<int32_t>(n); S.pv = A.take_n<int32_t>(n); S.nb = A.take_n<int32_t>(n);
    S.it = A.take_n<uint8_t>(n); S.lb = A.take_n<int8_t>(n); S.ee = A.take_n<int8_t>(n);
    S.fl = A.take_n<uint8_t>(n);
    return S.x && S.y && S.nx && S.pv && S.nb && S.it && S.lb && S.ee && S.fl;
  };
  RingSet SP, SQ;
  if (!take_ring(regTotP, SP) || !take_ring(regTotQ, SQ)) return ST_OUT_OF_MEMORY;
  mk->mark("clip:layout", s);
  // ---- G5 ring fill (light edges per thread, heavy edges per block)
  {
    int64_t* heavy = A.take_n<int64_t>(std::max(nEP, nEQ));
    unsigned long long* nHeavy = A.take_n<unsigned long long>(2);
    const int64_t nIns = std::max(nInsP, nInsQ);
    uint64_t* gkey = A.take_n<uint64_t>(2 * nIns);
    uint32_t* gtie = A.take_n<uint32_t>(2 * nIns);
    uint32_t* gidx = A.take_n<uint32_t>(2 * nIns);
    if (!heavy || !nHeavy || !gkey || !gtie || !gidx) return ST_OUT_OF_MEMORY;
    const size_t smem = (size_t)kHeavySmem * (sizeof(uint64_t) + 2 * sizeof(uint32_t));
    cudaFuncSetAttribute(heavy_fill_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaFuncSetAttribute(heavy_fill_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if (nEP > 0) {
      cudaMemsetAsync(nHeavy, 0, sizeof(unsigned long long), s);
      { ring_fill_kernel<0><<<blocks_for(nEP), kThreads, 0, s>>>(Lb, Lo, D, R, eoffP, nEP, K, vposP, regP, mP, SP,
                                                               slotP, insBaseP, curP, insListP, heavy, nHeavy); note_launch(); }
      { heavy_fill_kernel<0><<<2 * nsm, kHeavyThreads, smem, s>>>(Lb, Lo, D, R, eoffP, K, vposP, regP, mP, SP, slotP,
                                                                  insBaseP, curP, insListP, heavy, nHeavy, gkey, gtie,
                                                                  gidx); note_launch(); }
    }
    if (nEQ > 0) {
      cudaMemsetAsync(nHeavy + 1, 0, sizeof(unsigned long long), s);
      { ring_fill_kernel<1><<<blocks_for(nEQ), kThreads, 0, s>>>(Lb, Lo, D, R, eoffQ, nEQ, K, vposQ, regQ, mQ, SQ,
                                                               slotQ, insBaseQ, curQ, insListQ, heavy, nHeavy + 1); note_launch(); }
      { heavy_fill_kernel<1><<<2 * nsm, kHeavyThreads, smem, s>>>(Lb, Lo, D, R, eoffQ, K, vposQ, regQ, mQ, SQ, slotQ,
                                                                  insBaseQ, curQ, insListQ, heavy, nHeavy + 1, gkey, gtie,
                                                                  gidx); note_launch(); }
    }
  }
  // ---- G6 links
  if (nR > 0)
    { link_kernel<<<blocks_for(nR), kThreads, 0, s>>>(R, nR, D.status, eoffP, eoffQ, vposP, vposQ, regP, regQ,
                                                    slotP, slotQ, srcLinkP, srcLinkQ, SP, SQ); note_launch(); }
  // ---- G7 label + trace into per-pair output regions
  int64_t* vcap = A.take_n<int64_t>(K);
  int32_t* ccap = A.take_n<int32_t>(K);
  int64_t* vOff = A.take_n<int64_t>(K);
  int64_t* cOff = A.take_n<int64_t>(K);
  int32_t* nc = A.take_n<int32_t>(K);
  int64_t* nv = A.take_n<int64_t>(K);
  if (!vcap || !ccap || !vOff || !cOff || !nc || !nv) return ST_OUT_OF_MEMORY;
  { out_sizes_kernel<<<blocks_for(K), kThreads, 0, s>>>(mP, mQ, nrec, D.status, K, vcap, ccap); note_launch(); }
  exclusive_scan_i64(vcap, vOff, K, tot + 13, stK, d_err, s);
  exclusive_scan_i32(ccap, cOff, K, tot + 14, stK, d_err, s);
  cudaMemcpyAsync(hs, tot + 13, 2 * sizeof(int64_t), cudaMemcpyDeviceToHost, s);
  if (!sync()) return ST_CUDA_ERROR;
  double* oxy = A.take_n<double>(2 * hs[0]);
  int32_t* ocsz = A.take_n<int32_t>(hs[1]);
  if (!oxy || !ocsz) return ST_OUT_OF_MEMORY;
  mk->mark("clip:fill+link", s);
  { label_trace_kernel<<<(unsigned)((K + 3) / 4), 128, 0, s>>>(D, K, mP, mQ, regP, regQ, regSizeP, regSizeQ,
                                                                  SP, SQ, oxy, vOff, vcap, ocsz, cOff, ccap, nc,
                                                                  nv, prm, d_err); note_launch(); }
  mk->mark("clip:label+trace", s);
  // ---- G8 compaction
  C.ncomp = nc;
  C.comp_off = A.take_n<int64_t>(K);
  int64_t* fVOff = A.take_n<int64_t>(K);
  if (!C.comp_off || !fVOff) return ST_OUT_OF_MEMORY;
  exclusive_scan_i32(nc, C.comp_off, K, tot + 0, stK, d_err, s);
  exclusive_scan_i64(nv, fVOff, K, tot + 1, stK, d_err, s);
  cudaMemcpyAsync(hs, tot, 2 * sizeof(int64_t), cudaMemcpyDeviceToHost, s);
  if (!sync()) return ST_CUDA_ERROR;
  C.n_components = hs[0];
  C.n_vertices = hs[1];
  C.xy = A.take_n<double>(2 * C.n_vertices);
  C.comp_size = A.take_n<int32_t>(C.n_components);
  if (!C.xy || !C.comp_size) return ST_OUT_OF_MEMORY;
  { out_compact_kernel<<<blocks_for_warps(K), kThreads, 0, s>>>(K, oxy, vOff, ocsz, cOff, nc, nv, fVOff,
                                                              C.comp_off, C.xy, C.comp_size); note_launch(); }
  C.vert_off = fVOff;
  mk->mark("clip:compact", s);
  return ST_OK;
}

}  // namespace gcmfgh
