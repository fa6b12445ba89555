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
#include <climits>
#include <cmath>
#include <vector>
#include "common.cuh"
#include "engine.cuh"
#include "prims.cuh"

namespace gcmfgh {

namespace {

constexpr int kThreads = 256;
constexpr int kWarpsPerBlock = kThreads / 32;
constexpr int kChunk = 32;             // edge pairs per warp work unit (one per lane; 64 and 128 measured slower)
constexpr int64_t kFirstRecordCap = 1 << 22;   // records held by a fused count + emit without a hint
constexpr int kFilterTile = 4;         // lanes per small pair in the edge filter
constexpr int64_t kFilterTileMax = 64; // ring size up to which the narrow tiles take a pair

inline unsigned blocks_for_warps(int64_t warps) {
  return (unsigned)((warps + kWarpsPerBlock - 1) / kWarpsPerBlock);
}
inline unsigned blocks_for(int64_t n) { return (unsigned)((n + kThreads - 1) / kThreads); }


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
// W lanes per pair (W = 32: a warp).  Two passes split the pairs by ring size: narrow
// tiles for small pairs (they also zero the counts of pairs with nothing to test), whole
// warps for the rest.
// A pair of a join's clip set whose candidate has the join's common-MBR edge lists (the
// same boxes, the same test) takes them from there: the join tests every stored edge
// including the zero-length one from the stored closing vertex back to the first
// (GPU_Join.h:576-577), which the clip's open ring does not have, so that entry (the last,
// index n) is dropped; and both rings must be closed (stored closing vertex equal to the
// first), so that the join's last real edge is the clip's.
__device__ __forceinline__ bool ring_closed(const double2* v, int n) {
  const double2 a = __ldg(v), b = __ldg(v + n);
  return a.x == b.x && a.y == b.y;
}

template <int kMode, int W>
__global__ void __launch_bounds__(kThreads, 6)
edge_filter_kernel(LayerDev Lb, LayerDev Lo, PairDev D, int64_t K, int32_t* __restrict__ cP,
                   int32_t* __restrict__ cQ, const int64_t* __restrict__ offP,
                   const int64_t* __restrict__ offQ, int32_t* __restrict__ LP, int32_t* __restrict__ LQ,
                   int64_t lo, int64_t hi, JoinEdges je) {
  constexpr unsigned kBits = (W == 32) ? 0xffffffffu : ((1u << (W & 31)) - 1u);
  const int64_t w = ((int64_t)blockIdx.x * kThreads + threadIdx.x) / W;
  const int tl = (int)(threadIdx.x & (W - 1));
  const int tbase = (int)(lane_id() & ~(unsigned)(W - 1));
  const unsigned tmask = kBits << tbase;
  if (w >= K) return;
  if (D.status[w] != 0) { if (kMode == 0 && W != 32 && tl == 0) { cP[w] = 0; cQ[w] = 0; } return; }
  {
    const int64_t size = (int64_t)D.nP[w] + D.nQ[w];
    if (size <= lo || size > hi) return;             // the other pass takes this pair
  }
  const int pside = D.pSide[w];
  if (je.cand) {
    const int64_t cd = je.cand[w];
    if (je.flag[cd] && ring_closed(layer_xy(Lb, Lo, pside) + D.pS[w], D.nP[w]) &&
        ring_closed(layer_xy(Lb, Lo, 1 - pside) + D.qS[w], D.nQ[w])) {
      for (int side = 0; side < 2; ++side) {
        const bool base = (side == 0 ? pside : 1 - pside) == 0;
        const int n = side == 0 ? D.nP[w] : D.nQ[w];
        const int E = (base ? je.bE : je.oE)[cd];
        const int32_t* src = base ? je.bList + je.bOff[cd] : je.oList + je.oOff[cd];
        const int cnt = E - ((E > 0 && src[E - 1] == n) ? 1 : 0);
        if (kMode == 0) {
          if (tl == 0) (side == 0 ? cP : cQ)[w] = cnt;
        } else {
          int32_t* dst = side == 0 ? LP + offP[w] : LQ + offQ[w];
          for (int j = tl; j < cnt; j += W) dst[j] = src[j];
        }
      }
      return;
    }
  }
  double4 c = reinterpret_cast<const double4*>(D.cmbr)[w];
  for (int side = 0; side < 2; ++side) {
    const double2* v = layer_xy(Lb, Lo, side == 0 ? pside : 1 - pside) + (side == 0 ? D.pS[w] : D.qS[w]);
    const int n = side == 0 ? D.nP[w] : D.nQ[w];
    int cnt = 0;
    int64_t pos = 0;
    int32_t* list = nullptr;
    if (kMode == 1) { pos = side == 0 ? offP[w] : offQ[w]; list = side == 0 ? LP : LQ; }
    // whole warps take kUnroll groups of W edges per step: every group's loads are issued
    // before the first ballot
    constexpr int kUnroll = (W == 32) ? 4 : 1;
    for (int k0 = 0; k0 < n; k0 += W * kUnroll) {
      bool hit[kUnroll];
#pragma unroll
      for (int u = 0; u < kUnroll; ++u) {
        const int k = k0 + u * W + tl;
        hit[u] = false;
        if (k < n) {
          double2 a = __ldg(v + k), b = __ldg(v + (k + 1 < n ? k + 1 : 0));
          hit[u] = edge_touches_box(a.x, a.y, b.x, b.y, c.x, c.y, c.z, c.w);
        }
      }
#pragma unroll
      for (int u = 0; u < kUnroll; ++u) {
        unsigned m = __ballot_sync(tmask, hit[u]);
        if (W != 32) m = (m >> tbase) & kBits;
        if (kMode == 1 && hit[u]) list[pos + cnt + __popc(m & ((1u << tl) - 1u))] = k0 + u * W + tl;
        cnt += __popc(m);
      }
    }
    if (kMode == 0 && tl == 0) { if (side == 0) cP[w] = cnt; else cQ[w] = cnt; }
  }
}

// Pairs whose filtered edge grid exceeds ClipParams::bin_grid edge pairs are not
// enumerated pair by pair: their edges are binned on a uniform grid (bin_* kernels).

// edge -> pair: a warp per pair fills the entries of its cnt[k] edges starting at off[k]
__global__ void range_owner_kernel(const int64_t* __restrict__ off, const int32_t* __restrict__ cnt, int64_t K,
                                   int32_t* __restrict__ owner) {
  const int64_t k = ((int64_t)blockIdx.x * kThreads + threadIdx.x) >> 5;
  if (k >= K) return;
  const int64_t o = off[k];
  const int n = cnt[k];
  for (int j = lane_id(); j < n; j += 32) owner[o + j] = (int32_t)k;
}

// chunk -> pair: a warp per pair fills its chunks' entries
__global__ void chunk_pair_kernel(const int64_t* __restrict__ chunkOff, const int64_t* __restrict__ nchunk, int64_t K,
                                  int32_t* __restrict__ chunkPair) {
  const int64_t k = ((int64_t)blockIdx.x * kThreads + threadIdx.x) >> 5;
  if (k >= K) return;
  const int64_t o = chunkOff[k], n = nchunk[k];
  for (int64_t j = lane_id(); j < n; j += 32) chunkPair[o + j] = (int32_t)k;
}

__global__ void chunk_count_kernel(const int32_t* __restrict__ cP, const int32_t* __restrict__ cQ,
                                   int64_t K, int64_t* __restrict__ nchunk, int64_t* __restrict__ bigList,
                                   unsigned long long* __restrict__ nBig, int64_t binGrid) {
  int64_t k = (int64_t)blockIdx.x * kThreads + threadIdx.x;
  if (k >= K) return;
  int64_t W = (int64_t)cP[k] * cQ[k];
  if (W > binGrid) {
    nchunk[k] = 0;
    bigList[atomicAdd(nBig, 1ull)] = k;
  } else {
    nchunk[k] = (W + kChunk - 1) / kChunk;
  }
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

// Occupancy over registers: the count pass at most 64 registers (4 blocks per SM; count
// stage 1.29 -> 0.81 ms), the emit pass 40 (6 blocks; 0.55 -> 0.39 ms).  The
// exact-predicate instances keep 128 registers (their expansions would spill).
template <int kMode, int kExact>
__global__ void __launch_bounds__(kThreads, kExact ? 2 : (kMode == 1 ? 6 : 4))
intersect_kernel(LayerDev Lb, LayerDev Lo, PairDev D, int64_t K, const int64_t* __restrict__ chunkOff,
                 int64_t nChunks, const int32_t* __restrict__ cP, const int32_t* __restrict__ cQ,
                 const int64_t* __restrict__ offP, const int64_t* __restrict__ offQ,
                 const int32_t* __restrict__ LP, const int32_t* __restrict__ LQ, double eps,
                 int32_t* __restrict__ chunkRec, int32_t* __restrict__ chunkQ,
                 const int64_t* __restrict__ chunkRecOff, const int64_t* __restrict__ recOff, Records R,
                 const int32_t* __restrict__ chunkPair) {
  int64_t c = ((int64_t)blockIdx.x * kThreads + threadIdx.x) >> 5;
  if (c >= nChunks) return;
  const int64_t k = chunkPair[c];                  // the pair this chunk belongs to
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
  int64_t pos = (kMode == 1) ? recOff[k] + chunkRecOff[c] - chunkRecOff[chunkOff[k]] : 0;
  for (int it = 0; it < kChunk / 32; ++it) {
    int64_t t = t0 + it * 32 + lane_id();
    int tp = 0, tq = 0;
    int pe = 0, qe = 0;
    double alpha = 0, beta = 0;
    if (t < W) {
      if (W <= INT32_MAX) {                         // 32-bit division when it suffices
        const int tt = (int)t, r = tt / nq;
        pe = lp[r];
        qe = lq[tt - r * nq];
      } else {
        pe = lp[t / nq];
        qe = lq[t % nq];
      }
      double2 P1 = __ldg(pv + pe), P2 = __ldg(pv + (pe + 1 < np_ ? pe + 1 : 0));
      double2 Q1 = __ldg(qv + qe), Q2 = __ldg(qv + (qe + 1 < nq_ ? qe + 1 : 0));
      if (edge_boxes_touch(P1.x, P1.y, P2.x, P2.y, Q1.x, Q1.y, Q2.x, Q2.y)) {
        if (kMode == 0 && !kExact) {
          bool qhit;
          tp = classify_edges_both(P1.x, P1.y, P2.x, P2.y, Q1.x, Q1.y, Q2.x, Q2.y, eps, alpha, beta, qhit);
          tq = qhit ? 1 : 0;
        } else {
          tp = classify_mode(kExact, P1.x, P1.y, P2.x, P2.y, Q1.x, Q1.y, Q2.x, Q2.y, eps, alpha, beta);
          if (kMode == 0) {
            double a2, b2;
            tq = classify_mode(kExact, Q1.x, Q1.y, Q2.x, Q2.y, P1.x, P1.y, P2.x, P2.y, eps, a2, b2);
          }
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

// Count and emit in one pass over the chunks.  Each warp classifies its chunk's edge pairs
// from both sides as the count pass does and stages its P-side records in shared memory;
// the block then takes one range of a global counter and copies its records there.  The
// records end up in block order, which nothing downstream depends on (the ring fill orders
// a ring's insertions by parameter and other edge; a link keeps the largest other edge).
// Per pair, the P-side records and the Q-side hits are added into pairRec / pairQ (skipped
// when pairRec is null: a re-run after an overflow).  Records at or past cap are counted
// and not written; the host then re-runs with arrays of the counted size.
struct FusedRecords {
  unsigned long long* total;   // records taken so far (all blocks)
  int64_t cap;                 // records the arrays hold
  int32_t* pairRec;            // per pair: P-side records
  int32_t* pairQ;              // per pair: Q-side hits
};

template <int kExact, int kWarpAppend>
__global__ void __launch_bounds__(kThreads, kExact ? 2 : 4)
intersect_fused_kernel(LayerDev Lb, LayerDev Lo, PairDev D, const int64_t* __restrict__ chunkOff, int64_t nChunks,
                       const int32_t* __restrict__ cP, const int32_t* __restrict__ cQ,
                       const int64_t* __restrict__ offP, const int64_t* __restrict__ offQ,
                       const int32_t* __restrict__ LP, const int32_t* __restrict__ LQ, double eps, Records R,
                       const int32_t* __restrict__ chunkPair, FusedRecords F) {
  constexpr int kWarps = kThreads / 32;
  constexpr int kStage = kWarps * kChunk;           // at most one record per edge pair
  __shared__ double sA[kStage], sB[kStage];
  __shared__ int32_t sP[kStage], sQ[kStage];
  __shared__ int8_t sT[kStage];
  __shared__ int sOff[kWarps + 1];
  __shared__ int32_t sK[kWarps];
  __shared__ unsigned long long sBase;
  const int wib = (int)(threadIdx.x >> 5);
  const int64_t c = (int64_t)blockIdx.x * kWarps + wib;
  int recs = 0, qhits = 0;
  int64_t k = -1;
  if (c < nChunks) {
    k = chunkPair[c];
    const int nq = cQ[k];
    const int64_t W = (int64_t)cP[k] * nq;
    const int64_t t0 = (c - chunkOff[k]) * kChunk;
    const int pside = D.pSide[k];
    const double2* pv = layer_xy(Lb, Lo, pside) + D.pS[k];
    const double2* qv = layer_xy(Lb, Lo, 1 - pside) + D.qS[k];
    const int np_ = D.nP[k], nq_ = D.nQ[k];
    const int32_t* lp = LP + offP[k];
    const int32_t* lq = LQ + offQ[k];
    for (int it = 0; it < kChunk / 32; ++it) {
      const int64_t t = t0 + it * 32 + lane_id();
      int tp = 0, tq = 0, pe = 0, qe = 0;
      double alpha = 0, beta = 0;
      if (t < W) {
        if (W <= INT32_MAX) {
          const int tt = (int)t, r = tt / nq;
          pe = lp[r];
          qe = lq[tt - r * nq];
        } else {
          pe = lp[t / nq];
          qe = lq[t % nq];
        }
        double2 P1 = __ldg(pv + pe), P2 = __ldg(pv + (pe + 1 < np_ ? pe + 1 : 0));
        double2 Q1 = __ldg(qv + qe), Q2 = __ldg(qv + (qe + 1 < nq_ ? qe + 1 : 0));
        if (edge_boxes_touch(P1.x, P1.y, P2.x, P2.y, Q1.x, Q1.y, Q2.x, Q2.y)) {
          if (!kExact) {
            bool qhit;
            tp = classify_edges_both(P1.x, P1.y, P2.x, P2.y, Q1.x, Q1.y, Q2.x, Q2.y, eps, alpha, beta, qhit);
            tq = qhit ? 1 : 0;
          } else {
            double a2, b2;
            tp = classify_mode(kExact, P1.x, P1.y, P2.x, P2.y, Q1.x, Q1.y, Q2.x, Q2.y, eps, alpha, beta);
            tq = classify_mode(kExact, Q1.x, Q1.y, Q2.x, Q2.y, P1.x, P1.y, P2.x, P2.y, eps, a2, b2);
          }
        }
      }
      const unsigned m = __ballot_sync(0xffffffffu, tp != 0);
      if (tp != 0) {
        const int i = wib * kChunk + recs + __popc(m & lanemask_lt());
        sP[i] = pe; sQ[i] = qe; sA[i] = alpha; sB[i] = beta; sT[i] = (int8_t)tp;
      }
      recs += __popc(m);
      qhits += __popc(__ballot_sync(0xffffffffu, tq != 0));
    }
  }
  if (lane_id() == 0 && k >= 0 && F.pairRec) {
    if (recs) atomicAdd(&F.pairRec[k], recs);
    if (qhits) atomicAdd(&F.pairQ[k], qhits);
  }
  if (kWarpAppend) {                                // each warp takes its own range
    unsigned long long b = 0;
    if (lane_id() == 0 && recs) b = atomicAdd(F.total, (unsigned long long)recs);
    const int64_t base = (int64_t)__shfl_sync(0xffffffffu, b, 0);
    __syncwarp();
    for (int j = lane_id(); j < recs; j += 32) {
      const int i = wib * kChunk + j;
      const int64_t r = base + j;
      if (r < F.cap) { R.p[r] = sP[i]; R.q[r] = sQ[i]; R.a[r] = sA[i]; R.b[r] = sB[i]; R.t[r] = sT[i]; R.k[r] = (int32_t)k; }
    }
    return;
  }
  if (lane_id() == 0) { sOff[wib] = recs; sK[wib] = (int32_t)k; }
  __syncthreads();
  if (threadIdx.x == 0) {
    int run = 0;
    for (int w = 0; w < kWarps; ++w) { const int n = sOff[w]; sOff[w] = run; run += n; }
    sOff[kWarps] = run;
    sBase = run ? atomicAdd(F.total, (unsigned long long)run) : 0ull;
  }
  __syncthreads();
  const int n = sOff[kWarps];
  const int64_t base = (int64_t)sBase;
  for (int j = threadIdx.x; j < n; j += kThreads) {
    int w = 0;
    while (w + 1 < kWarps && sOff[w + 1] <= j) ++w;
    const int i = w * kChunk + (j - sOff[w]);
    const int64_t r = base + j;
    if (r < F.cap) { R.p[r] = sP[i]; R.q[r] = sQ[i]; R.a[r] = sA[i]; R.b[r] = sB[i]; R.t[r] = sT[i]; R.k[r] = sK[w]; }
  }
}

// per pair: record count (chunked + binned), validity
__global__ void pair_records_kernel(const int64_t* __restrict__ chunkOff, const int64_t* __restrict__ nchunk,
                                    const int64_t* __restrict__ recScan, const int64_t* __restrict__ qScan,
                                    const int32_t* __restrict__ chunkRec, const int32_t* __restrict__ chunkQ,
                                    const int64_t* __restrict__ binRec, const int64_t* __restrict__ binQ,
                                    int64_t K, int64_t* __restrict__ nrec64, int32_t* __restrict__ nrec,
                                    int64_t* __restrict__ count1, PairDev D,
                                    const int32_t* __restrict__ pairRec, const int32_t* __restrict__ pairQ) {
  int64_t k = (int64_t)blockIdx.x * kThreads + threadIdx.x;
  if (k >= K) return;
  int64_t c0 = chunkOff[k], n = nchunk[k];
  int64_t r = binRec[k], q = binQ[k];
  if (pairRec) {                                   // the fused pass counted per pair
    r += pairRec[k];
    q += pairQ[k];
  } else if (n > 0) {
    r += recScan[c0 + n - 1] + chunkRec[c0 + n - 1] - recScan[c0];
    q += qScan[c0 + n - 1] + chunkQ[c0 + n - 1] - qScan[c0];
  }
  nrec64[k] = r;
  nrec[k] = (int32_t)r;
  count1[k] = r;
  if (D.status[k] == 0 && r != q) D.status[k] = 1;   // gppolyclip_mDIV512.cu:1461
}

// ---------------------------------------------------------------- G2/G3 binned
// Pairs whose filtered edge grid exceeds ClipParams::bin_grid edge pairs are not
// enumerated edge pair by edge pair.  Each gets a uniform grid over its common MBR
// (about one Q edge per cell); its Q edges are listed in every cell their box covers;
// each P edge visits the cells its box covers and tests a Q edge only in the cell holding
// the lower-left corner of the two boxes' overlap, so every edge pair whose boxes touch
// is tested exactly once (cell indices are monotone in the coordinate).  All binned pairs
// go through the same launches: their P and Q edges are numbered consecutively (pair by
// pair) and each edge finds its pair through an owner table.
struct BinGrid { double x0, y0, cw, ch; int gx, gy; };

__device__ __forceinline__ int cell_1d(double v, double c0, double cs, int g) {
  double t = (v - c0) / cs;
  if (!(t > 0)) return 0;             // also NaN
  if (t >= (double)g) return g - 1;
  return (int)t;
}

// The binned pairs, i = 0..B-1 (pair k = list[i]).
struct BinSet {
  const int64_t* list;
  int32_t* cp; int32_t* cq;           // filtered edges per side
  int64_t* pBase; int64_t* qBase;     // first binned P / Q edge of pair i
  int32_t* ownP; int32_t* ownQ;       // binned edge -> i
  double* ext;                        // per pair: sums of the Q edges' box widths, heights
  BinGrid* grid;
  int64_t* cellBase;                  // first cell of pair i (cells of all pairs in one array)
  int32_t* ncell;
};

__global__ void bin_sizes_kernel(BinSet S, int n, const int32_t* __restrict__ cP, const int32_t* __restrict__ cQ) {
  int i = blockIdx.x * kThreads + threadIdx.x;
  if (i >= n) return;
  const int64_t k = S.list[i];
  S.cp[i] = cP[k];
  S.cq[i] = cQ[k];
}

// the pair-local Q (P) edge of binned edge j
__device__ __forceinline__ int binned_q(const BinSet& S, int64_t j, int i, const int64_t* offQ, const int32_t* LQ) {
  return LQ[offQ[S.list[i]] + (j - S.qBase[i])];
}
__device__ __forceinline__ int binned_p(const BinSet& S, int64_t j, int i, const int64_t* offP, const int32_t* LP) {
  return LP[offP[S.list[i]] + (j - S.pBase[i])];
}

// Sums of the Q edges' box widths and heights per pair (they size the cells).  Edges of
// one pair are consecutive, so a warp reduces each run of equal owners and one lane per
// run adds it.
__global__ void bin_extent_kernel(LayerDev Lb, LayerDev Lo, PairDev D, BinSet S, int64_t nq,
                                  const int64_t* __restrict__ offQ, const int32_t* __restrict__ LQ) {
  const int64_t j = (int64_t)blockIdx.x * kThreads + threadIdx.x;
  int i = -1;
  double w = 0, h = 0;
  if (j < nq) {
    i = S.ownQ[j];
    const int64_t k = S.list[i];
    const double2* qv = layer_xy(Lb, Lo, 1 - D.pSide[k]) + D.qS[k];
    const int n = D.nQ[k];
    const int q = binned_q(S, j, i, offQ, LQ);
    const double2 a = __ldg(qv + q), b = __ldg(qv + (q + 1 < n ? q + 1 : 0));
    w = fabs(b.x - a.x);
    h = fabs(b.y - a.y);
  }
  const int lane = (int)lane_id();
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {          // segmented inclusive scan over equal owners
    const double uw = __shfl_up_sync(0xffffffffu, w, d), uh = __shfl_up_sync(0xffffffffu, h, d);
    const int ui = __shfl_up_sync(0xffffffffu, i, d);
    if (lane >= d && ui == i) { w += uw; h += uh; }
  }
  const int ni = __shfl_down_sync(0xffffffffu, i, 1);
  if (i >= 0 && (lane == 31 || ni != i)) {
    atomicAdd(S.ext + 2 * i, w);
    atomicAdd(S.ext + 2 * i + 1, h);
  }
}

// Grid of each binned pair: about one Q edge per cell, but never cells smaller than the
// Q edges' mean box (long edges would otherwise be listed in many cells and each P edge
// would scan them all again); at most 4096 cells per axis.
__global__ void bin_grid_kernel(PairDev D, BinSet S, int n) {
  int i = blockIdx.x * kThreads + threadIdx.x;
  if (i >= n) return;
  const double4 c = reinterpret_cast<const double4*>(D.cmbr)[S.list[i]];
  const double w = c.z - c.x, h = c.w - c.y;
  const double target = (double)max(1, S.cq[i]);
  const double mw = S.ext[2 * i] / target, mh = S.ext[2 * i + 1] / target;
  double gx = 1, gy = 1;
  if (w > 0 && h > 0) {
    gx = ceil(sqrt(target * w / h));
    gx = fmin(fmax(gx, 1.0), 4096.0);
    gy = ceil(target / gx);
    if (mw > 0) gx = fmin(gx, ceil(w / mw));
    if (mh > 0) gy = fmin(gy, ceil(h / mh));
    gx = fmin(fmax(gx, 1.0), 4096.0);
    gy = fmin(fmax(gy, 1.0), 4096.0);
  } else if (w > 0) {
    gx = fmin(target, 4096.0);
  } else if (h > 0) {
    gy = fmin(target, 4096.0);
  }
  BinGrid G{c.x, c.y, w > 0 ? w / gx : 1.0, h > 0 ? h / gy : 1.0, (int)gx, (int)gy};
  S.grid[i] = G;
  S.ncell[i] = G.gx * G.gy;
}

// kMode 0: count the listings per cell; kMode 1: list every Q edge in the cells its box covers
template <int kMode>
__global__ void bin_cells_kernel(LayerDev Lb, LayerDev Lo, PairDev D, BinSet S, int64_t nq,
                                 const int64_t* __restrict__ offQ, const int32_t* __restrict__ LQ,
                                 int32_t* __restrict__ cellCnt, const int64_t* __restrict__ cellOff,
                                 int32_t* __restrict__ cursor, int32_t* __restrict__ cellList) {
  const int64_t j = (int64_t)blockIdx.x * kThreads + threadIdx.x;
  if (j >= nq) return;
  const int i = S.ownQ[j];
  const int64_t k = S.list[i];
  const double2* qv = layer_xy(Lb, Lo, 1 - D.pSide[k]) + D.qS[k];
  const int n = D.nQ[k];
  const int q = binned_q(S, j, i, offQ, LQ);
  const double2 a = __ldg(qv + q), b = __ldg(qv + (q + 1 < n ? q + 1 : 0));
  const BinGrid G = S.grid[i];
  const int64_t cb = S.cellBase[i];
  const int x0 = cell_1d(fmin(a.x, b.x), G.x0, G.cw, G.gx), x1 = cell_1d(fmax(a.x, b.x), G.x0, G.cw, G.gx);
  const int y0 = cell_1d(fmin(a.y, b.y), G.y0, G.ch, G.gy), y1 = cell_1d(fmax(a.y, b.y), G.y0, G.ch, G.gy);
  for (int y = y0; y <= y1; ++y)
    for (int x = x0; x <= x1; ++x) {
      const int64_t c = cb + (int64_t)y * G.gx + x;
      if (kMode == 0) atomicAdd(&cellCnt[c], 1);
      else cellList[cellOff[c] + atomicAdd(&cursor[c], 1)] = q;
    }
}

// kMode 0: per binned P edge, its records (P side) into recCnt, and the pair's Q-side
// count into binQ; kMode 1: write the records of each P edge at its offset (in cell
// order: nothing downstream depends on record order).  The offset is the pair's recOff
// plus the edge's place in the pair, or, with recOff null (after the fused count + emit
// of the chunked pairs), *recBase plus the edge's place among all binned edges; records
// at or past cap are not written.
template <int kMode, int kExact>
__global__ void __launch_bounds__(kThreads, kExact ? 2 : 4)
bin_pairs_kernel(LayerDev Lb, LayerDev Lo, PairDev D, BinSet S, int64_t np,
                 const int64_t* __restrict__ offP, const int32_t* __restrict__ LP,
                 const int64_t* __restrict__ cellOff, const int32_t* __restrict__ cellList, double eps,
                 int32_t* __restrict__ recCnt, int64_t* __restrict__ binQ,
                 const int64_t* __restrict__ recPos, const int64_t* __restrict__ recOff, Records R,
                 const unsigned long long* __restrict__ recBase, int64_t cap) {
  const int64_t j = (int64_t)blockIdx.x * kThreads + threadIdx.x;
  if (j >= np) return;
  const int i = S.ownP[j];
  const int64_t k = S.list[i];
  const int pside = D.pSide[k];
  const double2* pv = layer_xy(Lb, Lo, pside) + D.pS[k];
  const double2* qv = layer_xy(Lb, Lo, 1 - pside) + D.qS[k];
  const int np_ = D.nP[k], nq = D.nQ[k];
  const int p = binned_p(S, j, i, offP, LP);
  const double2 P1 = __ldg(pv + p), P2 = __ldg(pv + (p + 1 < np_ ? p + 1 : 0));
  const double pminx = fmin(P1.x, P2.x), pmaxx = fmax(P1.x, P2.x);
  const double pminy = fmin(P1.y, P2.y), pmaxy = fmax(P1.y, P2.y);
  const BinGrid G = S.grid[i];
  const int64_t cb = S.cellBase[i];
  const int x0 = cell_1d(pminx, G.x0, G.cw, G.gx), x1 = cell_1d(pmaxx, G.x0, G.cw, G.gx);
  const int y0 = cell_1d(pminy, G.y0, G.ch, G.gy), y1 = cell_1d(pmaxy, G.y0, G.ch, G.gy);
  int recs = 0, qhits = 0;
  const int64_t base = (kMode == 0) ? 0
                       : recOff ? recOff[k] + recPos[j] - recPos[S.pBase[i]]
                                : (int64_t)*recBase + recPos[j];
  for (int y = y0; y <= y1; ++y)
    for (int x = x0; x <= x1; ++x) {
      const int64_t c = cb + (int64_t)y * G.gx + x;
      for (int64_t e = cellOff[c]; e < cellOff[c + 1]; ++e) {
        const int q = cellList[e];
        const double2 Q1 = __ldg(qv + q), Q2 = __ldg(qv + (q + 1 < nq ? q + 1 : 0));
        if (!edge_boxes_touch(P1.x, P1.y, P2.x, P2.y, Q1.x, Q1.y, Q2.x, Q2.y)) continue;
        const double cx = fmax(pminx, fmin(Q1.x, Q2.x)), cy = fmax(pminy, fmin(Q1.y, Q2.y));
        if (cell_1d(cx, G.x0, G.cw, G.gx) != x || cell_1d(cy, G.y0, G.ch, G.gy) != y) continue;
        double alpha = 0, beta = 0;
        const int tp = classify_mode(kExact, P1.x, P1.y, P2.x, P2.y, Q1.x, Q1.y, Q2.x, Q2.y, eps, alpha, beta);
        if (kMode == 0) {
          double a2, b2;
          if (classify_mode(kExact, Q1.x, Q1.y, Q2.x, Q2.y, P1.x, P1.y, P2.x, P2.y, eps, a2, b2)) ++qhits;
          if (tp) ++recs;
        } else if (tp) {
          const int64_t r = base + recs++;
          if (r < cap) {
            R.p[r] = p; R.q[r] = q; R.a[r] = alpha; R.b[r] = beta; R.t[r] = (int8_t)tp; R.k[r] = (int32_t)k;
          }
        }
      }
    }
  if (kMode == 0) {
    recCnt[j] = recs;
    if (qhits) atomicAdd(reinterpret_cast<unsigned long long*>(binQ + k), (unsigned long long)qhits);
  }
}

// per binned pair: its records (the P edges' counts summed through their scan)
__global__ void bin_rec_total_kernel(BinSet S, int n, const int64_t* __restrict__ recPos,
                                     int64_t* __restrict__ binRec) {
  int i = blockIdx.x * kThreads + threadIdx.x;
  if (i >= n) return;
  const int64_t b = S.pBase[i];
  binRec[S.list[i]] = recPos[b + S.cp[i]] - recPos[b];
}

// ---------------------------------------------------------------- G4 ring layout
// Per record: insertion counts per edge, and the winning (last) record for each source
// vertex that records link (P: types 2,4,5,6,8; Q: types 3,4,5,7,8).
// "Last record wins" in the reference's loop order (P edge outer, Q edge inner) is the
// record with the largest other-side edge, so the winner is the maximum of
// (other edge, record index): independent of the order records were emitted in.
constexpr int kLinkKeyShift = 33;             // record indices below 2^33
__device__ __forceinline__ unsigned long long link_key(int other, int64_t r) {
  return (((unsigned long long)other << kLinkKeyShift) | (unsigned long long)r) + 1ull;
}

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
    atomicMax(reinterpret_cast<unsigned long long*>(&srcLinkP[eP]), link_key(R.q[r], r));
  if (t == 3 || t == 4 || t == 5 || t == 7 || t == 8)
    atomicMax(reinterpret_cast<unsigned long long*>(&srcLinkQ[eQ]), link_key(R.p[r], r));
}

// slot of each edge's source vertex in the concatenated merged rings: the exclusive scan
// of (1 + insertions) over the edges, i.e. the edge index plus the scan of the insertions
__global__ void edge_slots_kernel(const int64_t* __restrict__ insBase, int64_t nE, int64_t* __restrict__ vpos) {
  int64_t e = (int64_t)blockIdx.x * kThreads + threadIdx.x;
  if (e < nE) vpos[e] = e + insBase[e];
}

// The merged rings of one side live in one buffer of n slots, column by column:
//   xy (double2) | nx pv nb (int32) | tn tl to ls (int32) | it lb ee fl (byte)
// 48 bytes per slot.  A ring is then the buffer, n and its first slot: a thread that
// walks a pair keeps three words per ring instead of a pointer per column, and each
// column stays dense for the scans over one field.
//   nx, pv, nb  next, previous, neighbour (slot on the other ring, -1 none)
//   tn tl to ls tracing scratch: next run start (other ring), run length, output offset,
//               and (by list index) the slots of the flagged vertices
//   it          intersection flag (cleared when visited by the trace)
//   lb, ee      IntersectionLabel, EntryExitLabel
//   fl          bit0 split candidate, bit1 crossing candidate
#define GCMFGH_RING_COLUMNS(IDX)                                                                   \
  __device__ __forceinline__ double2& xy(int64_t i) const { return reinterpret_cast<double2*>(b)[IDX]; } \
  __device__ __forceinline__ double& x(int64_t i) const { return xy(i).x; }                         \
  __device__ __forceinline__ double& y(int64_t i) const { return xy(i).y; }                         \
  __device__ __forceinline__ int32_t& nx(int64_t i) const { return reinterpret_cast<int32_t*>(b + 16 * n)[IDX]; } \
  __device__ __forceinline__ int32_t& pv(int64_t i) const { return reinterpret_cast<int32_t*>(b + 20 * n)[IDX]; } \
  __device__ __forceinline__ int32_t& nb(int64_t i) const { return reinterpret_cast<int32_t*>(b + 24 * n)[IDX]; } \
  __device__ __forceinline__ int32_t& tn(int64_t i) const { return reinterpret_cast<int32_t*>(b + 28 * n)[IDX]; } \
  __device__ __forceinline__ int32_t& tl(int64_t i) const { return reinterpret_cast<int32_t*>(b + 32 * n)[IDX]; } \
  __device__ __forceinline__ int32_t& to(int64_t i) const { return reinterpret_cast<int32_t*>(b + 36 * n)[IDX]; } \
  __device__ __forceinline__ int32_t& ls(int64_t i) const { return reinterpret_cast<int32_t*>(b + 40 * n)[IDX]; } \
  __device__ __forceinline__ uint8_t& it(int64_t i) const { return reinterpret_cast<uint8_t*>(b + 44 * n)[IDX]; } \
  __device__ __forceinline__ int8_t& lb(int64_t i) const { return reinterpret_cast<int8_t*>(b + 45 * n)[IDX]; } \
  __device__ __forceinline__ int8_t& ee(int64_t i) const { return reinterpret_cast<int8_t*>(b + 46 * n)[IDX]; } \
  __device__ __forceinline__ uint8_t& fl(int64_t i) const { return reinterpret_cast<uint8_t*>(b + 47 * n)[IDX]; }

constexpr int64_t kRingSlotBytes = 48;

// Kernels that take a RingSet by value keep its column pointers in the parameter space,
// so the side-wide kernels (fill, links, export, grid path) index columns directly.
struct RingSet {
  char* b;          // column buffer
  int64_t n;        // slots per column (a multiple of 16, so every column stays aligned)
  int exact;        // orientation signs exact (ClipParams::exact)
  double2* cxy; int32_t* cnx; int32_t* cpv; int32_t* cnb;
  uint8_t* cit; int8_t* clb; int8_t* cee; uint8_t* cfl;
  void set(char* buf, int64_t slots) {
    b = buf; n = slots;
    cxy = reinterpret_cast<double2*>(b);
    cnx = reinterpret_cast<int32_t*>(b + 16 * n); cpv = reinterpret_cast<int32_t*>(b + 20 * n);
    cnb = reinterpret_cast<int32_t*>(b + 24 * n); cit = reinterpret_cast<uint8_t*>(b + 44 * n);
    clb = reinterpret_cast<int8_t*>(b + 45 * n); cee = reinterpret_cast<int8_t*>(b + 46 * n);
    cfl = reinterpret_cast<uint8_t*>(b + 47 * n);
  }
  __device__ __forceinline__ double2& xy(int64_t i) const { return cxy[i]; }
  __device__ __forceinline__ double& x(int64_t i) const { return cxy[i].x; }
  __device__ __forceinline__ double& y(int64_t i) const { return cxy[i].y; }
  __device__ __forceinline__ int32_t& nx(int64_t i) const { return cnx[i]; }
  __device__ __forceinline__ int32_t& pv(int64_t i) const { return cpv[i]; }
  __device__ __forceinline__ int32_t& nb(int64_t i) const { return cnb[i]; }
  __device__ __forceinline__ uint8_t& it(int64_t i) const { return cit[i]; }
  __device__ __forceinline__ int8_t& lb(int64_t i) const { return clb[i]; }
  __device__ __forceinline__ int8_t& ee(int64_t i) const { return cee[i]; }
  __device__ __forceinline__ uint8_t& fl(int64_t i) const { return cfl[i]; }
};

// per pair: ring size, region offset (ring + room for added vertices)
__global__ void pair_ring_kernel(const int64_t* __restrict__ eoff, const int64_t* __restrict__ vpos,
                                 const int32_t* __restrict__ n, const int32_t* __restrict__ nrec,
                                 const int32_t* __restrict__ status, int64_t K, int64_t nE,
                                 const int64_t* __restrict__ insTot,
                                 int32_t* __restrict__ m, int64_t* __restrict__ regSize,
                                 unsigned long long* __restrict__ ringTot) {
  int64_t k = (int64_t)blockIdx.x * kThreads + threadIdx.x;
  unsigned long long mm = 0;
  if (k < K) {
    const int64_t vtot = nE + *insTot;                      // slots of the side's merged rings
    int64_t e0 = eoff[k], e1 = e0 + (status[k] == 2 ? 0 : n[k]);
    int64_t v0 = e0 < nE ? vpos[e0] : vtot, v1 = e1 < nE ? vpos[e1] : vtot;
    mm = status[k] == 0 ? (unsigned long long)(v1 - v0) : 0ull;
    m[k] = (int)mm;
    regSize[k] = status[k] == 0 ? (int64_t)mm + 2 + 2 * (int64_t)nrec[k] : 0;
  }
  mm = warp_sum(mm);                                        // merged-ring vertices, all pairs
  if (lane_id() == 0 && mm) atomicAdd(ringTot, mm);
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
  S.x(gs) = X; S.y(gs) = Y;
  S.nx(gs) = (sl + 1) % f.mm; S.pv(gs) = (sl + f.mm - 1) % f.mm; S.nb(gs) = -1;
  S.it(gs) = 0; S.lb(gs) = L_NONE; S.ee(gs) = E_NEITHER; S.fl(gs) = 0;
  slotOfRec[r] = sl;
}

template <int kSide>
__device__ __forceinline__ bool edge_fill_info(const LayerDev& Lb, const LayerDev& Lo, const PairDev& D,
                                               const int64_t* eoff, const int32_t* edgePair, const int64_t* vpos,
                                               const int64_t* regOff, const int32_t* m, int64_t e, EdgeFill& f) {
  const int64_t k = edgePair[e];
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

// At most 64 registers (4 blocks per SM): the kernel is latency-bound and the extra
// occupancy outweighs a few spilled values (measured 1.35 -> 1.03 ms for the fill stage).
template <int kSide>
__global__ void __launch_bounds__(kThreads, 4) ring_fill_kernel(LayerDev Lb, LayerDev Lo, PairDev D, Records R,
                                 const int64_t* __restrict__ eoff, int64_t nE, const int32_t* __restrict__ edgePair,
                                 const int64_t* __restrict__ vpos, const int64_t* __restrict__ regOff,
                                 const int32_t* __restrict__ m, RingSet S, int64_t* __restrict__ slotOfRec,
                                 const int64_t* __restrict__ insCursorBase, int32_t* __restrict__ insCursor,
                                 const int64_t* __restrict__ insList, int64_t* __restrict__ heavy,
                                 unsigned long long* __restrict__ nHeavy) {
  int64_t e = (int64_t)blockIdx.x * kThreads + threadIdx.x;
  if (e >= nE) return;
  EdgeFill f;
  if (!edge_fill_info<kSide>(Lb, Lo, D, eoff, edgePair, vpos, regOff, m, e, f)) return;
  const int le = (int)(e - eoff[f.k]);
  const double2 A = __ldg((kSide == 0 ? f.pvx : f.qvx) + le);
  const int64_t g = f.base + f.s0;
  S.x(g) = A.x; S.y(g) = A.y;
  S.nx(g) = (f.s0 + 1) % f.mm; S.pv(g) = (f.s0 + f.mm - 1) % f.mm; S.nb(g) = -1;
  S.it(g) = 0; S.lb(g) = L_NONE; S.ee(g) = E_NEITHER; S.fl(g) = 0;
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
heavy_fill_kernel(LayerDev Lb, LayerDev Lo, PairDev D, Records R, const int64_t* __restrict__ eoff,
                  const int32_t* __restrict__ edgePair,
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
    if (threadIdx.x == 0) edge_fill_info<kSide>(Lb, Lo, D, eoff, edgePair, vpos, regOff, m, e, f);
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
  S.nb(base + slot) = target;
  S.it(base + slot) = 1;
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
  const bool winP = (unsigned long long)srcLinkP[eP] == link_key(R.q[r], r);
  const bool winQ = (unsigned long long)srcLinkQ[eQ] == link_key(R.p[r], r);
  switch (t) {
    case 1: {
      int sp = (int)slotP[r], sq = (int)slotQ[r];
      set_link(SP, bP, sp, sq); set_link(SQ, bQ, sq, sp);
      break;
    }
    case 2: case 6: {
      int sq = (int)slotQ[r];
      set_link(SQ, bQ, sq, srcP);
      SP.it(bP + srcP) = 1;
      if (winP) SP.nb(bP + srcP) = sq;
      break;
    }
    case 3: case 7: {
      int sp = (int)slotP[r];
      set_link(SP, bP, sp, srcQ);
      SQ.it(bQ + srcQ) = 1;
      if (winQ) SQ.nb(bQ + srcQ) = sp;
      break;
    }
    case 4: case 8: {
      SP.it(bP + srcP) = 1; SQ.it(bQ + srcQ) = 1;
      if (winP) SP.nb(bP + srcP) = srcQ;
      if (winQ) SQ.nb(bQ + srcQ) = srcP;
      break;
    }
    case 5: {
      int sp = (int)slotP[r], sq = (int)slotQ[r];
      set_link(SQ, bQ, sq, srcP);
      SP.it(bP + srcP) = 1;
      if (winP) SP.nb(bP + srcP) = sq;
      set_link(SP, bP, sp, srcQ);
      SQ.it(bQ + srcQ) = 1;
      if (winQ) SQ.nb(bQ + srcQ) = sp;
      break;
    }
  }
}

// ---------------------------------------------------------------- ring export
// The reference's calculateIntersections (gppolyclip_mDIV512.cu:1298-1640) returns the
// merged rings with an integer parameter key per vertex: (int)(1e7 * alpha) where the
// vertex carries an intersection, -100 at plain vertices (:926).  Inserted vertices get
// the key of their one record (:997-1053).  The source vertex of an edge gets the key of
// its degenerate records (P: types 2/4/6/8, Q: types 3/4/7/8).  The P side is written by
// the P edge's loop over ascending Q edges, so the largest Q edge wins.  The Q side is
// written by concurrent P-edge threads (a race in the reference); here the largest P edge
// wins.  Keys are packed as (other edge + 1) << 32 | key and combined with atomicMax.
// Per pair it also counts the records that insert a vertex on each ring.
__device__ __forceinline__ uint32_t alpha_key(double a) {
  return (uint32_t)(int32_t)(10000000.0 * a);      // (int)pow(10, EPSILON_POSITIONS)*alpha
}

__global__ void export_key_kernel(Records R, int64_t nR, const int32_t* __restrict__ status,
                                  const int64_t* __restrict__ eoffP, const int64_t* __restrict__ eoffQ,
                                  const int64_t* __restrict__ vposP, const int64_t* __restrict__ vposQ,
                                  const int64_t* __restrict__ regP, const int64_t* __restrict__ regQ,
                                  const int64_t* __restrict__ slotP, const int64_t* __restrict__ slotQ,
                                  unsigned long long* __restrict__ keyP, unsigned long long* __restrict__ keyQ,
                                  int32_t* __restrict__ cntP, int32_t* __restrict__ cntQ) {
  int64_t r = (int64_t)blockIdx.x * kThreads + threadIdx.x;
  if (r >= nR) return;
  const int k = R.k[r];
  const int t = R.t[r];
  const bool insOnP = t == 1 || t == 3 || t == 5 || t == 7;
  const bool insOnQ = t == 1 || t == 2 || t == 5 || t == 6;
  if (insOnP) atomicAdd(&cntP[k], 1);
  if (insOnQ) atomicAdd(&cntQ[k], 1);
  if (status[k] != 0) return;
  const int64_t eP = eoffP[k] + R.p[r], eQ = eoffQ[k] + R.q[r];
  const uint32_t kp = alpha_key(R.a[r]), kq = alpha_key(R.b[r]);
  if (insOnP) {
    keyP[regP[k] + slotP[r]] = (1ull << 32) | kp;
  } else {
    const int64_t src = vposP[eP] - vposP[eoffP[k]];
    atomicMax(&keyP[regP[k] + src], ((unsigned long long)(R.q[r] + 1) << 32) | kp);
  }
  if (insOnQ) {
    keyQ[regQ[k] + slotQ[r]] = (1ull << 32) | kq;
  } else {
    const int64_t src = vposQ[eQ] - vposQ[eoffQ[k]];
    atomicMax(&keyQ[regQ[k] + src], ((unsigned long long)(R.p[r] + 1) << 32) | kq);
  }
}

__device__ __forceinline__ int32_t unpack_key(unsigned long long v) {
  return v == 0 ? -100 : (int32_t)(uint32_t)v;
}

// oracle() of gppolyclip_mDIV512.cu:195-215: Q's position relative to the chain
// (P1, P2, P3), or which of P1 / P3 it is linked to
__device__ int export_rel(int exact, int pMN, int pPN, int qId, const RingSet& SQ, int64_t bQ,
                          const RingSet& SP, int64_t bP, int p1, int p2, int p3) {
  if (pMN != -100 && pMN == qId) return R_IS_P_M;
  if (pPN != -100 && pPN == qId) return R_IS_P_P;
  const double qx = SQ.x(bQ + qId), qy = SQ.y(bQ + qId);
  const double x1 = SP.x(bP + p1), y1 = SP.y(bP + p1), x2 = SP.x(bP + p2), y2 = SP.y(bP + p2);
  const double x3 = SP.x(bP + p3), y3 = SP.y(bP + p3);
  const int s1 = orient_sign(exact, qx, qy, x1, y1, x2, y2);
  const int s2 = orient_sign(exact, qx, qy, x2, y2, x3, y3);
  const int s3 = orient_sign(exact, x1, y1, x2, y2, x3, y3);
  if (s3 > 0) return (s1 > 0 && s2 > 0) ? R_LEFT : R_RIGHT;
  return (s1 < 0 && s2 < 0) ? R_RIGHT : R_LEFT;
}

// getInitialLabel of gppolyclip_mDIV512.cu:237-252, including its -102 for combinations
// that name no label
__device__ int32_t export_label(int m, int p) {
  auto is = [&](int a, int b) { return (m == a && p == b) || (m == b && p == a); };
  if (is(R_LEFT, R_RIGHT)) return L_CROSSING;
  if ((m == R_LEFT && p == R_LEFT) || (m == R_RIGHT && p == R_RIGHT)) return L_BOUNCING;
  if (is(R_IS_P_P, R_RIGHT)) return L_LEFT_ON;
  if (is(R_IS_P_P, R_LEFT)) return L_RIGHT_ON;
  if (is(R_IS_P_P, R_IS_P_M)) return L_ON_ON;
  if (is(R_IS_P_M, R_RIGHT)) return L_ON_LEFT;
  if (is(R_IS_P_M, R_LEFT)) return L_ON_RIGHT;
  return -102;
}

// Block per pair: the merged rings in ring order (slot order before any labelling), their
// keys and 1-based neighbours; then the initial labels of gpuCalculateInitLabel
// (gppolyclip_mDIV512.cu:1171-1223), computed at the P vertices that carry a key and
// copied to their Q neighbours.  Output arrays are indexed like the ring regions.
__global__ void export_ring_kernel(int64_t K, const int32_t* __restrict__ status, const int32_t* __restrict__ mP,
                                   const int32_t* __restrict__ mQ, const int64_t* __restrict__ regP,
                                   const int64_t* __restrict__ regQ, RingSet SP, RingSet SQ,
                                   const unsigned long long* __restrict__ keyP,
                                   const unsigned long long* __restrict__ keyQ, double* __restrict__ xyP,
                                   double* __restrict__ xyQ, int32_t* __restrict__ alP, int32_t* __restrict__ alQ,
                                   int32_t* __restrict__ lbP, int32_t* __restrict__ lbQ, int32_t* __restrict__ nbP,
                                   int32_t* __restrict__ nbQ) {
  const int64_t k = blockIdx.x;
  if (k >= K || status[k] != 0) return;
  const int np = mP[k], nq = mQ[k];
  const int64_t bP = regP[k], bQ = regQ[k];
  for (int s = threadIdx.x; s < np; s += blockDim.x) {
    const int64_t g = bP + s;
    xyP[2 * g] = SP.x(g); xyP[2 * g + 1] = SP.y(g);
    alP[g] = unpack_key(keyP[g]);
    lbP[g] = -100;
    nbP[g] = SP.nb(g) + 1;
  }
  for (int s = threadIdx.x; s < nq; s += blockDim.x) {
    const int64_t g = bQ + s;
    xyQ[2 * g] = SQ.x(g); xyQ[2 * g + 1] = SQ.y(g);
    alQ[g] = unpack_key(keyQ[g]);
    lbQ[g] = -100;
    nbQ[g] = SQ.nb(g) + 1;
  }
  __syncthreads();
  for (int s = threadIdx.x; s < np; s += blockDim.x) {
    if (keyP[bP + s] == 0) continue;
    const int nId = SP.nb(bP + s);
    if (nId < 0 || nId >= nq) continue;
    const int pm = s > 0 ? s - 1 : np - 1, pp = s + 1 < np ? s + 1 : 0;
    const int pMN = keyP[bP + pm] != 0 ? SP.nb(bP + pm) : -100;
    const int pPN = keyP[bP + pp] != 0 ? SP.nb(bP + pp) : -100;
    const int qm = nId > 0 ? nId - 1 : nq - 1, qp = nId + 1 < nq ? nId + 1 : 0;
    const int a = export_rel(SP.exact, pMN, pPN, qm, SQ, bQ, SP, bP, pm, s, pp);
    const int b = export_rel(SP.exact, pMN, pPN, qp, SQ, bQ, SP, bP, pm, s, pp);
    const int32_t L = export_label(a, b);
    lbP[bP + s] = L;
    lbQ[bQ + nId] = L;
  }
}

// ---------------------------------------------------------------- G7 label + trace
struct Ring {
  char* b; int64_t n;   // the side's column buffer (RingSet)
  int64_t o;            // first slot of this ring
  int m;        // slots in the merged ring
  int used;     // slots in use (ring + added vertices)
  int cap;      // region capacity
  int exact;    // orientation signs exact
  GCMFGH_RING_COLUMNS(o + i)
};

__device__ __forceinline__ Ring ring_of(const RingSet& S, int64_t base, int m, int cap) {
  Ring r;
  r.b = S.b; r.n = S.n; r.o = base;
  r.m = m; r.used = m; r.cap = cap; r.exact = S.exact;
  return r;
}

__device__ int add_vertex(Ring& R, double X, double Y) {
  if (R.used >= R.cap) return -1;
  int v = R.used++;
  R.x(v) = X; R.y(v) = Y; R.nx(v) = v; R.pv(v) = v; R.nb(v) = -1;
  R.it(v) = 0; R.lb(v) = L_NONE; R.ee(v) = E_NEITHER; R.fl(v) = 0;
  return v;
}

__device__ __forceinline__ void insert_after(Ring& R, int v, int after) {
  int c = R.nx(after);
  R.nx(R.pv(c)) = v; R.pv(v) = R.pv(c); R.nx(v) = c; R.pv(c) = v;
}

// polygon.h:427-448 (winding parity) over the ring reached from slot 0, skipping `skip`
template <int EX>
__device__ bool point_in_ring(const Ring& R, double Rx, double Ry, int skip) {
  int w = 0;
  int one = 0;
  int guard = R.used + 2;
  do {
    int two = R.nx(one);
    if (two == skip) two = R.nx(two);
    double P0x = R.x(one), P0y = R.y(one), P1x = R.x(two), P1y = R.y(two);
    if ((P0y < Ry) != (P1y < Ry)) {
      if (P0x >= Rx) {
        if (P1x > Rx) w = w + 2 * (P1y > P0y) - 1;
        else if ((orient_sign(EX, P0x, P0y, P1x, P1y, Rx, Ry) > 0) == (P1y > P0y)) w = w + 2 * (P1y > P0y) - 1;
      } else if (P1x > Rx) {
        if ((orient_sign(EX, P0x, P0y, P1x, P1y, Rx, Ry) > 0) == (P1y > P0y)) w = w + 2 * (P1y > P0y) - 1;
      }
    }
    one = two;
  } while (one != 0 && --guard > 0);
  return (w % 2) != 0;
}

// relative position of Q w.r.t. the chain (P1, P2, P3): polyclip.h:297-326
template <int EX>
__device__ int rel_position(const Ring& P, const Ring& Q, int qv, int p1, int p2, int p3) {
  if (P.it(p1) && P.nb(p1) == qv) return R_IS_P_M;
  if (P.it(p3) && P.nb(p3) == qv) return R_IS_P_P;
  const int ex = EX;
  int s1 = orient_sign(ex, Q.x(qv), Q.y(qv), P.x(p1), P.y(p1), P.x(p2), P.y(p2));
  int s2 = orient_sign(ex, Q.x(qv), Q.y(qv), P.x(p2), P.y(p2), P.x(p3), P.y(p3));
  int s3 = orient_sign(ex, P.x(p1), P.y(p1), P.x(p2), P.y(p2), P.x(p3), P.y(p3));
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
  do { if (!A.it(v)) return v; v = A.nx(v); } while (v != 0 && --guard > 0);
  v = 0; guard = A.used + 1;
  do {
    int nb = A.nb(v), nx = A.nx(v);
    if (nb >= 0 && A.nb(nx) != B.pv(nb) && A.nb(nx) != B.nx(nb)) { midpoint = true; return v; }
    v = A.nx(v);
  } while (v != 0 && --guard > 0);
  return -1;
}

__device__ void push_ring(OutRegion& O, const Ring& A) {
  O.begin();
  int v = 0, guard = A.used + 1;
  do { O.push(A.x(v), A.y(v)); v = A.nx(v); } while (v != 0 && --guard > 0);
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
template <int EX>
__device__ void seq_step1(PairCtx& c) {
  Ring& P = c.R[0];
  Ring& Q = c.R[1];
  for (int s = 0; s < P.m; ++s) {
    if (!P.it(s)) continue;
    int nb = P.nb(s);
    if (nb < 0) continue;
    int pm = P.pv(s), pp = P.nx(s);
    int a = rel_position<EX>(P, Q, Q.pv(nb), pm, s, pp);
    int b = rel_position<EX>(P, Q, Q.nx(nb), pm, s, pp);
    int8_t L = initial_label(a, b);
    if (L != L_NONE) { P.lb(s) = L; Q.lb(nb) = L; }
  }
}

// step 2: intersection chains (polyclip.h:405-451)
__device__ void seq_step2(PairCtx& c) {
  Ring& P = c.R[0];
  Ring& Q = c.R[1];
  for (int s = 0; s < P.m; ++s) {
    if (!P.it(s) || (P.lb(s) != L_LEFT_ON && P.lb(s) != L_RIGHT_ON)) continue;
    int x = P.lb(s) == L_LEFT_ON ? R_LEFT : R_RIGHT;
    int X = s, I = s, guard = P.m + 1;
    do {
      P.lb(I) = L_NONE;
      if (P.nb(I) >= 0) Q.lb(P.nb(I)) = L_NONE;
      I = P.nx(I);
    } while (P.lb(I) == L_ON_ON && --guard > 0);
    int y = P.lb(I) == L_ON_LEFT ? R_LEFT : R_RIGHT;
    int8_t ct = (x != y) ? L_DELAYED_CROSSING : L_DELAYED_BOUNCING;
    P.lb(X) = ct; P.lb(I) = ct;
    if (P.nb(X) >= 0) Q.lb(P.nb(X)) = ct;
    if (P.nb(I) >= 0) Q.lb(P.nb(I)) = ct;
  }
}

// step 3.5: components without crossings (polyclip.h:474-541)
template <int EX>
__device__ void seq_step35(PairCtx& c) {
  for (int sd = 0; sd < 2; ++sd) {
    Ring& A = c.R[sd];
    bool none = true, allOn = true;
    for (int v = 0; v < A.m; ++v) {
      int8_t l = A.lb(v);
      if (l != L_ON_ON) allOn = false;
      if (A.it(v)) {
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
    double px = A.x(v), py = A.y(v);
    if (mid) { int n = A.nx(v); px = 0.5 * (A.x(v) + A.x(n)); py = 0.5 * (A.y(v) + A.y(n)); }
    bool inside = point_in_ring<EX>(B, px, py, -1);
    if (inside ^ c.uni) push_ring(c.O, A);
  }
  if (c.ident[0] && c.ident[1]) push_ring(c.O, c.R[0]);
}

// step 4: entry/exit flags (polyclip.h:549-655)
template <int EX>
__device__ bool seq_step4(PairCtx& c) {
  for (int sd = 0; sd < 2; ++sd) {
    if (c.noInter[sd]) continue;
    Ring& A = c.R[sd];
    Ring& B = c.R[1 - sd];
    bool mid;
    int V = first_non_intersection(A, B, mid);
    if (V < 0) continue;
    if (mid) {
      int n = A.nx(V);
      int T = add_vertex(A, 0.5 * (A.x(V) + A.x(n)), 0.5 * (A.y(V) + A.y(n)));
      if (T < 0) { fail(c, DEV_CAPACITY); return false; }
      insert_after(A, T, V);
      V = T;
    }
    // the Q pass sees P's temporary vertex; P's pass cannot see Q's (not yet added)
    int8_t st = point_in_ring<EX>(B, A.x(V), A.y(V), -1) ? E_EXIT : E_ENTRY;
    bool first = true;
    int I = A.nx(V), guard = A.used + 1;
    while (I != V && --guard > 0) {
      if (A.it(I)) {
        int8_t l = A.lb(I);
        if (l == L_CROSSING) { A.ee(I) = st; st = toggled(st); }
        if (A.lb(I) == L_BOUNCING && ((st == E_EXIT) ^ c.uni)) A.fl(I) |= 1;
        if (A.lb(I) == L_DELAYED_CROSSING) {
          A.ee(I) = st;
          if (first) { if ((st == E_EXIT) ^ c.uni) A.lb(I) = L_CROSSING; first = false; }
          else {
            if ((st == E_ENTRY) ^ c.uni) A.lb(I) = L_CROSSING;
            first = true;
            st = toggled(st);
          }
        }
        if (A.lb(I) == L_DELAYED_BOUNCING) {
          A.ee(I) = st;
          if (first) { if ((st == E_EXIT) ^ c.uni) A.fl(I) |= 2; first = false; }
          else { if ((st == E_ENTRY) ^ c.uni) A.fl(I) |= 2; first = true; }
          st = toggled(st);
        }
      }
      I = A.nx(I);
    }
  }
  return true;
}

// step 5: split vertex pairs (polyclip.h:661-714)
template <int EX>
__device__ bool seq_step5(PairCtx& c) {
  Ring& P = c.R[0];
  Ring& Q = c.R[1];
  const int pm0 = P.used;
  for (int ip = 0; ip < pm0; ++ip) {
    if (!(P.fl(ip) & 1)) continue;
    int iq = P.nb(ip);
    if (iq < 0 || !(Q.fl(iq) & 1)) continue;
    int vp = add_vertex(P, P.x(ip), P.y(ip));
    int vq = add_vertex(Q, Q.x(iq), Q.y(iq));
    if (vp < 0 || vq < 0) { fail(c, DEV_CAPACITY); return false; }
    bool same;
    if (EX) {
      same = orient_exact_call(P.x(P.pv(ip)), P.y(P.pv(ip)), P.x(ip), P.y(ip), P.x(P.nx(ip)), P.y(P.nx(ip))) *
             orient_exact_call(Q.x(Q.pv(iq)), Q.y(Q.pv(iq)), Q.x(iq), Q.y(iq), Q.x(Q.nx(iq)), Q.y(Q.nx(iq))) > 0;
    } else {
      double sP = area2(P.x(P.pv(ip)), P.y(P.pv(ip)), P.x(ip), P.y(ip), P.x(P.nx(ip)), P.y(P.nx(ip)));
      double sQ = area2(Q.x(Q.pv(iq)), Q.y(Q.pv(iq)), Q.x(iq), Q.y(iq), Q.x(Q.nx(iq)), Q.y(Q.nx(iq)));
      same = sP * sQ > 0;
    }
    if (same) {
      P.nb(ip) = vq; Q.nb(vq) = ip; P.it(ip) = 1; Q.it(vq) = 1;
      Q.nb(iq) = vp; P.nb(vp) = iq; Q.it(iq) = 1; P.it(vp) = 1;
    } else {
      P.nb(vp) = vq; Q.nb(vq) = vp; P.it(vp) = 1; Q.it(vq) = 1;
    }
    insert_after(P, vp, ip);
    insert_after(Q, vq, iq);
    int8_t e1 = c.uni ? E_ENTRY : E_EXIT, e2 = c.uni ? E_EXIT : E_ENTRY;
    P.ee(ip) = e1; P.ee(vp) = e2; Q.ee(iq) = e1; Q.ee(vq) = e2;
    P.lb(ip) = L_CROSSING; P.lb(vp) = L_CROSSING; Q.lb(iq) = L_CROSSING; Q.lb(vq) = L_CROSSING;
  }
  return true;
}

// step 6: crossing candidates (polyclip.h:723-734)
__device__ void seq_step6(PairCtx& c) {
  Ring& P = c.R[0];
  Ring& Q = c.R[1];
  for (int ip = 0; ip < P.m; ++ip) {
    if (!(P.fl(ip) & 2)) continue;
    int iq = P.nb(ip);
    if (iq >= 0 && (Q.fl(iq) & 2)) { P.lb(ip) = L_CROSSING; Q.lb(iq) = L_CROSSING; }
  }
}

// tracing (polyclip.h:743-783): starts at unvisited CROSSING vertices of P in ring order
// from slot 0; visited vertices are marked by clearing their intersection flag.
__device__ bool seq_trace(PairCtx& c) {
  Ring& P = c.R[0];
  OutRegion& O = c.O;
  long long budget = 4ll * (c.R[0].used + c.R[1].used) + 16;
  int I = 0;
  bool have = P.it(I) && P.lb(I) == L_CROSSING;
  if (!have) {
    int guard = P.used + 1;
    do { I = P.nx(I); } while (!(P.it(I) && P.lb(I) == L_CROSSING) && I != 0 && --guard > 0);
    have = I != 0 && guard > 0;
  }
  while (have) {
    O.begin();
    int side = 0, V = I;
    P.it(V) = 0;
    do {
      Ring& C = c.R[side];
      int8_t st = toggled(C.ee(V));
      do {
        if (--budget < 0) { fail(c, DEV_TRACE); return false; }
        V = ((st == E_EXIT) ^ c.uni) ? C.nx(V) : C.pv(V);
        C.it(V) = 0;
        O.push(C.x(V), C.y(V));
      } while (!(C.ee(V) == st) && !(side == 0 && V == I));
      if (!(side == 0 && V == I)) {
        int nb = C.nb(V);
        if (nb < 0) { fail(c, DEV_TRACE); return false; }
        V = nb;
        side = 1 - side;
        c.R[side].it(V) = 0;
      }
    } while (!(side == 0 && V == I));
    O.end();
    int guard = P.used + 1;
    do { I = P.nx(I); } while (!(P.it(I) && P.lb(I) == L_CROSSING) && I != 0 && --guard > 0);
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
template <int EX>
__device__ void seq_pair_from(PairCtx& c, int step, int32_t* outNC, int64_t* outNV) {
  if (step <= 1) seq_step1<EX>(c);
  seq_step2(c);
  seq_step35<EX>(c);
  if (!seq_step4<EX>(c) || !seq_step5<EX>(c)) return;
  seq_step6(c);
  if (!seq_trace(c)) return;
  seq_cleanup(c, outNC, outNV);
}

// ================================================================ warp phases
constexpr unsigned kFull = 0xffffffffu;

// winding increment of edge (P0,P1) for point R: polygon.h:433-444
__device__ __forceinline__ int wind(double P0x, double P0y, double P1x, double P1y, double Rx, double Ry,
                                    int ex) {
  if ((P0y < Ry) == (P1y < Ry)) return 0;
  int d = 2 * (P1y > P0y) - 1;
  if (P0x >= Rx) {
    if (P1x > Rx) return d;
    return ((orient_sign(ex, P0x, P0y, P1x, P1y, Rx, Ry) > 0) == (P1y > P0y)) ? d : 0;
  }
  if (P1x > Rx) return ((orient_sign(ex, P0x, P0y, P1x, P1y, Rx, Ry) > 0) == (P1y > P0y)) ? d : 0;
  return 0;
}

// ---- cooperative groups for the parallel labelling and tracing of one pair.  The same
// code runs with a warp per pair (WarpGroup) or, for pairs with long rings, a whole block
// per pair (BlockGroup); every member executes every group call (uniform control flow).
struct WarpGroup {
  static constexpr bool kBlock = false;
  static constexpr bool kSolo = false;
  __device__ __forceinline__ int rank() const { return (int)lane_id(); }
  __device__ __forceinline__ int size() const { return 32; }
  __device__ __forceinline__ void sync() const { __syncwarp(); }
  __device__ __forceinline__ bool all(bool v) const { return __all_sync(kFull, v); }
  __device__ __forceinline__ bool any(bool v) const { return __any_sync(kFull, v); }
  __device__ __forceinline__ int sum(int v) const { return warp_sum(v); }
  template <class T>
  __device__ __forceinline__ T bcast0(T v) const { return __shfl_sync(kFull, v, 0); }
  // smallest member index whose flag is set, -1 if none
  __device__ __forceinline__ int first(bool hit) const {
    unsigned m = __ballot_sync(kFull, hit);
    return m ? __ffs(m) - 1 : -1;
  }
  __device__ __forceinline__ int incl_scan(int v, int& total) const {
    int x = warp_incl_scan(v);
    total = __shfl_sync(kFull, x, 31);
    return x;
  }
};

// A tile of W lanes (a power of two below 32) of one warp: the tiles work on different pairs
// side by side, each with its own lane mask.
template <int W>
struct TileGroup {
  static constexpr bool kBlock = false;
  static constexpr bool kSolo = false;
  unsigned mask;
  int base;
  __device__ __forceinline__ TileGroup() {
    base = (int)(lane_id() & ~(unsigned)(W - 1));
    mask = ((1u << W) - 1u) << base;
  }
  __device__ __forceinline__ int rank() const { return (int)lane_id() - base; }
  __device__ __forceinline__ int size() const { return W; }
  __device__ __forceinline__ void sync() const { __syncwarp(mask); }
  __device__ __forceinline__ bool all(bool v) const { return (__ballot_sync(mask, v) & mask) == mask; }
  __device__ __forceinline__ bool any(bool v) const { return (__ballot_sync(mask, v) & mask) != 0u; }
  __device__ __forceinline__ int sum(int v) const {
#pragma unroll
    for (int o = W / 2; o > 0; o >>= 1) v += __shfl_xor_sync(mask, v, o, W);
    return v;
  }
  template <class T>
  __device__ __forceinline__ T bcast0(T v) const { return __shfl_sync(mask, v, 0, W); }
  __device__ __forceinline__ int first(bool hit) const {
    const unsigned m = (__ballot_sync(mask, hit) & mask) >> base;
    return m ? __ffs(m) - 1 : -1;
  }
  __device__ __forceinline__ int incl_scan(int v, int& total) const {
#pragma unroll
    for (int o = 1; o < W; o <<= 1) {
      const int w = __shfl_up_sync(mask, v, o, W);
      if (rank() >= o) v += w;
    }
    total = __shfl_sync(mask, v, W - 1, W);
    return v;
  }
};

// One thread per pair: every collective is the identity, nothing synchronises.
struct SoloGroup {
  static constexpr bool kBlock = false;
  static constexpr bool kSolo = true;
  __device__ __forceinline__ int rank() const { return 0; }
  __device__ __forceinline__ int size() const { return 1; }
  __device__ __forceinline__ void sync() const {}
  __device__ __forceinline__ bool all(bool v) const { return v; }
  __device__ __forceinline__ bool any(bool v) const { return v; }
  __device__ __forceinline__ int sum(int v) const { return v; }
  template <class T>
  __device__ __forceinline__ T bcast0(T v) const { return v; }
  __device__ __forceinline__ int first(bool hit) const { return hit ? 0 : -1; }
  __device__ __forceinline__ int incl_scan(int v, int& total) const { total = v; return v; }
};

template <int W> struct TileOf { using type = TileGroup<W>; };
template <> struct TileOf<1> { using type = SoloGroup; };

// Block-wide versions over shared scratch (kBlockLabelThreads / 32 warps); each call
// begins with a barrier so the scratch of the previous call is free.
constexpr int kBlockLabelThreads = 512;
// Dynamic shared memory of the block labelling kernel: the trace's run table of pairs with
// up to 8,192 runs (two blocks per SM at its register budget).
constexpr int kBlockRunTableBytes = 96 * 1024;
struct BlockGroup {
  static constexpr bool kBlock = true;
  static constexpr bool kSolo = false;
  long long* sm;        // kBlockLabelThreads / 32 + 1 entries
  int32_t* runs;        // shared memory for the trace's run table (3 words per run)
  int runsCap;          // runs that fit
  __device__ __forceinline__ int rank() const { return (int)threadIdx.x; }
  __device__ __forceinline__ int size() const { return kBlockLabelThreads; }
  __device__ __forceinline__ void sync() const { __syncthreads(); }
  __device__ __forceinline__ bool all(bool v) const { return __syncthreads_and(v) != 0; }
  __device__ __forceinline__ bool any(bool v) const { return __syncthreads_or(v) != 0; }
  __device__ __forceinline__ int sum(int v) const {
    v = warp_sum(v);
    __syncthreads();
    if (lane_id() == 0) sm[threadIdx.x >> 5] = v;
    __syncthreads();
    long long t = 0;
    for (int w = 0; w < kBlockLabelThreads / 32; ++w) t += sm[w];
    return (int)t;
  }
  template <class T>
  __device__ __forceinline__ T bcast0(T v) const {
    static_assert(sizeof(T) <= sizeof(long long), "bcast0: scalar types only");
    __syncthreads();
    if (threadIdx.x == 0) { long long x = 0; memcpy(&x, &v, sizeof(T)); sm[kBlockLabelThreads / 32] = x; }
    __syncthreads();
    long long x = sm[kBlockLabelThreads / 32];
    T r;
    memcpy(&r, &x, sizeof(T));
    return r;
  }
  __device__ __forceinline__ int first(bool hit) const {
    unsigned m = __ballot_sync(kFull, hit);
    __syncthreads();
    if (lane_id() == 0) sm[threadIdx.x >> 5] = m ? (long long)((threadIdx.x & ~31u) + __ffs(m) - 1) : -1;
    __syncthreads();
    for (int w = 0; w < kBlockLabelThreads / 32; ++w)
      if (sm[w] >= 0) return (int)sm[w];
    return -1;
  }
  __device__ __forceinline__ int incl_scan(int v, int& total) const {
    int x = warp_incl_scan(v);
    __syncthreads();
    if (lane_id() == 31) sm[threadIdx.x >> 5] = x;
    __syncthreads();
    long long before = 0, all = 0;
    const int me = (int)(threadIdx.x >> 5);
    for (int w = 0; w < kBlockLabelThreads / 32; ++w) { if (w < me) before += sm[w]; all += sm[w]; }
    total = (int)all;
    return (int)(before + x);
  }
};

// polygon.h:427-448 over ring B in slot order; `after`/`T`: a temporary vertex T inserted
// after slot `after` (or -1)
template <int EX, class G>
__device__ bool grp_point_in_ring(const G& g, const Ring& B, double Rx, double Ry, int after, int T) {
  int w = 0;
  for (int s = g.rank(); s < B.m; s += g.size()) {
    int n = (s + 1 < B.m) ? s + 1 : 0;
    if (s == after) {
      w += wind(B.x(s), B.y(s), B.x(T), B.y(T), Rx, Ry, EX);
      w += wind(B.x(T), B.y(T), B.x(n), B.y(n), Rx, Ry, EX);
    } else {
      w += wind(B.x(s), B.y(s), B.x(n), B.y(n), Rx, Ry, EX);
    }
  }
  w = g.sum(w);
  return (w % 2) != 0;
}

// first slot s >= from (slot order, s < n) where pred(s); n if none
template <class G, class F>
__device__ int grp_find_first(const G& g, int from, int n, F pred) {
  for (int b = from; b < n; b += g.size()) {
    int s = b + g.rank();
    int f = g.first(s < n && pred(s));
    if (f >= 0) return b + f;
  }
  return n;
}

template <class G>
__device__ bool grp_links_one_to_one(const G& g, const Ring& P, const Ring& Q) {
  bool ok = true;
  for (int s = g.rank(); s < P.m; s += g.size())
    if (P.it(s)) { int nb = P.nb(s); if (nb < 0 || nb >= Q.m || Q.nb(nb) != s) ok = false; }
  for (int s = g.rank(); s < Q.m; s += g.size())
    if (Q.it(s)) { int nb = Q.nb(s); if (nb < 0 || nb >= P.m || P.nb(nb) != s) ok = false; }
  return g.all(ok);
}

template <int EX, class G>
__device__ void grp_step1(const G& g, PairCtx& c) {
  Ring& P = c.R[0];
  Ring& Q = c.R[1];
  for (int s = g.rank(); s < P.m; s += g.size()) {
    if (!P.it(s)) continue;
    int nb = P.nb(s);
    int pm = (s > 0) ? s - 1 : P.m - 1, pp = (s + 1 < P.m) ? s + 1 : 0;
    int a = rel_position<EX>(P, Q, (nb > 0) ? nb - 1 : Q.m - 1, pm, s, pp);
    int b = rel_position<EX>(P, Q, (nb + 1 < Q.m) ? nb + 1 : 0, pm, s, pp);
    int8_t L = initial_label(a, b);
    if (L != L_NONE) { P.lb(s) = L; Q.lb(nb) = L; }
  }
  g.sync();
}

// Chains run from a LEFT_ON/RIGHT_ON vertex over ON_ON vertices to an ON_LEFT/ON_RIGHT
// vertex.  When every chain ends so, chains are disjoint and can be resolved in parallel
// with the sequential result; otherwise returns false and nothing is changed.
template <class G>
__device__ bool grp_step2(const G& g, PairCtx& c) {
  Ring& P = c.R[0];
  Ring& Q = c.R[1];
  const int m = P.m;
  bool ok = true;
  for (int s = g.rank(); s < m; s += g.size()) {
    if (!P.it(s) || (P.lb(s) != L_LEFT_ON && P.lb(s) != L_RIGHT_ON)) continue;
    int I = (s + 1 < m) ? s + 1 : 0, guard = m;
    while (P.lb(I) == L_ON_ON && --guard > 0) I = (I + 1 < m) ? I + 1 : 0;
    if ((P.lb(I) != L_ON_LEFT && P.lb(I) != L_ON_RIGHT) || !P.it(I)) ok = false;
  }
  if (!g.all(ok)) return false;
  for (int s = g.rank(); s < m; s += g.size()) {
    int8_t l0 = P.lb(s);
    if (!P.it(s) || (l0 != L_LEFT_ON && l0 != L_RIGHT_ON)) continue;
    int x = l0 == L_LEFT_ON ? R_LEFT : R_RIGHT;
    int I = (s + 1 < m) ? s + 1 : 0;
    Q.lb(P.nb(s)) = L_NONE;
    while (P.lb(I) == L_ON_ON) {
      P.lb(I) = L_NONE;
      Q.lb(P.nb(I)) = L_NONE;
      I = (I + 1 < m) ? I + 1 : 0;
    }
    int y = P.lb(I) == L_ON_LEFT ? R_LEFT : R_RIGHT;
    int8_t ct = (x != y) ? L_DELAYED_CROSSING : L_DELAYED_BOUNCING;
    P.lb(s) = ct; P.lb(I) = ct;
    Q.lb(P.nb(s)) = ct; Q.lb(P.nb(I)) = ct;
  }
  g.sync();
  return true;
}

// copies ring A (slot order, no added vertices) as one output component
template <class G>
__device__ void grp_push_ring(const G& g, OutRegion& O, const Ring& A) {
  O.begin();
  if (O.overflow) return;
  if (O.nv + A.m > O.vcap) { O.overflow = true; return; }
  for (int s = g.rank(); s < A.m; s += g.size()) { O.xy[2 * (O.nv + s)] = A.x(s); O.xy[2 * (O.nv + s) + 1] = A.y(s); }
  if (g.rank() == 0) O.csz[O.nc] = A.m;
  O.nv += A.m;
  O.end();
  g.sync();
}

// first non-intersection slot (slot order = ring order before any insertion), else the
// first vertex whose edge to the next one is not collinear with the other polygon
// (polygon.h:480-512); returns -1 if none
template <class G>
__device__ int grp_first_non_intersection(const G& g, const Ring& A, const Ring& B, bool& mid) {
  mid = false;
  int v = grp_find_first(g, 0, A.m, [&](int s) { return !A.it(s); });
  if (v < A.m) return v;
  // B's own links: B may already hold its temporary vertex when A is Q
  v = grp_find_first(g, 0, A.m, [&](int s) {
    int nb = A.nb(s), nx = A.nx(s);
    return nb >= 0 && A.nb(nx) != B.pv(nb) && A.nb(nx) != B.nx(nb);
  });
  if (v < A.m) { mid = true; return v; }
  return -1;
}

template <int EX, class G>
__device__ void grp_step35(const G& g, PairCtx& c) {
  for (int sd = 0; sd < 2; ++sd) {
    Ring& A = c.R[sd];
    bool none = true, allOn = true;
    for (int v = g.rank(); v < A.m; v += g.size()) {
      int8_t l = A.lb(v);
      if (l != L_ON_ON) allOn = false;
      if (A.it(v)) {
        if (l == L_CROSSING || l == L_DELAYED_CROSSING) none = false;
        if (c.uni && (l == L_BOUNCING || l == L_DELAYED_BOUNCING)) none = false;
      }
    }
    none = g.all(none);
    allOn = g.all(allOn);
    c.noInter[sd] = none;
    c.ident[sd] = none && allOn;
  }
  for (int sd = 0; sd < 2; ++sd) {
    if (!c.noInter[sd] || c.ident[sd]) continue;
    Ring& A = c.R[sd];
    Ring& B = c.R[1 - sd];
    bool mid;
    int v = grp_first_non_intersection(g, A, B, mid);
    if (v < 0) continue;
    double px = A.x(v), py = A.y(v);
    if (mid) { int n = (v + 1 < A.m) ? v + 1 : 0; px = 0.5 * (A.x(v) + A.x(n)); py = 0.5 * (A.y(v) + A.y(n)); }
    bool inside = grp_point_in_ring<EX>(g, B, px, py, -1, -1);
    if (inside ^ c.uni) grp_push_ring(g, c.O, A);
  }
  if (c.ident[0] && c.ident[1]) grp_push_ring(g, c.O, c.R[0]);
}

// Entry/exit flags as a warp prefix scan over the ring from the start vertex: the status
// at a vertex is the start status toggled once per earlier CROSSING, DELAYED_BOUNCING and
// second-of-a-chain DELAYED_CROSSING; "first chain vertex" alternates over the DELAYED
// vertices met (polyclip.h:582-653).
template <int EX, class G>
__device__ bool grp_step4(const G& g, PairCtx& c, int tempAfter[2], int tempSlot[2]) {
  for (int sd = 0; sd < 2; ++sd) {
    tempAfter[sd] = -1;
    tempSlot[sd] = -1;
  }
  for (int sd = 0; sd < 2; ++sd) {
    if (c.noInter[sd]) continue;
    Ring& A = c.R[sd];
    Ring& B = c.R[1 - sd];
    bool mid;
    int V0 = grp_first_non_intersection(g, A, B, mid);
    if (V0 < 0) continue;
    double qx = A.x(V0), qy = A.y(V0);
    if (mid) {
      int T = -1;
      if (g.rank() == 0) {
        T = add_vertex(A, 0.5 * (A.x(V0) + A.x((V0 + 1 < A.m) ? V0 + 1 : 0)),
                       0.5 * (A.y(V0) + A.y((V0 + 1 < A.m) ? V0 + 1 : 0)));
        if (T >= 0) insert_after(A, T, V0);
      }
      T = g.bcast0(T);
      A.used = g.bcast0(A.used);
      g.sync();
      if (T < 0) { if (g.rank() == 0) fail(c, DEV_CAPACITY); return false; }
      tempAfter[sd] = V0;
      tempSlot[sd] = T;
      qx = A.x(T);
      qy = A.y(T);
    }
    // the Q pass tests against P's ring including P's temporary vertex
    int8_t st0 = (sd == 1 ? grp_point_in_ring<EX>(g, B, qx, qy, tempAfter[0], tempSlot[0])
                          : grp_point_in_ring<EX>(g, B, qx, qy, -1, -1)) ? E_EXIT : E_ENTRY;
    int carryD = 0, carryT = 0;
    const int m = A.m;
    for (int b = 0; b < m; b += g.size()) {
      int j = b + g.rank();
      int s = -1;
      int8_t L = L_NONE;
      bool inter = false;
      if (j < m) {
        s = V0 + 1 + j;
        if (s >= m) s -= m;
        inter = A.it(s);
        L = inter ? A.lb(s) : L_NONE;
      }
      int d = inter && (L == L_DELAYED_CROSSING || L == L_DELAYED_BOUNCING);
      int dTot, tTot;
      int dIncl = g.incl_scan(d, dTot);
      bool first = ((carryD + dIncl - d) & 1) == 0;
      int t = inter && (L == L_CROSSING || L == L_DELAYED_BOUNCING || (L == L_DELAYED_CROSSING && !first));
      int tIncl = g.incl_scan(t, tTot);
      int8_t st = ((carryT + tIncl - t) & 1) ? toggled(st0) : st0;
      if (inter) {
        if (L == L_CROSSING) A.ee(s) = st;
        else if (L == L_BOUNCING) { if ((st == E_EXIT) ^ c.uni) A.fl(s) |= 1; }
        else if (L == L_DELAYED_CROSSING) {
          A.ee(s) = st;
          if (first) { if ((st == E_EXIT) ^ c.uni) A.lb(s) = L_CROSSING; }
          else if ((st == E_ENTRY) ^ c.uni) A.lb(s) = L_CROSSING;
        } else if (L == L_DELAYED_BOUNCING) {
          A.ee(s) = st;
          if (first) { if ((st == E_EXIT) ^ c.uni) A.fl(s) |= 2; }
          else if ((st == E_ENTRY) ^ c.uni) A.fl(s) |= 2;
        }
      }
      carryD += dTot;
      carryT += tTot;
    }
    g.sync();
  }
  return true;
}

template <class G>
__device__ bool grp_any_split(const G& g, const Ring& P, const Ring& Q) {
  bool any = false;
  for (int s = g.rank(); s < P.m; s += g.size())
    if (P.fl(s) & 1) { int nb = P.nb(s); if (nb >= 0 && (Q.fl(nb) & 1)) any = true; }
  return g.any(any);
}

template <class G>
__device__ void grp_step6(const G& g, PairCtx& c) {
  Ring& P = c.R[0];
  Ring& Q = c.R[1];
  for (int ip = g.rank(); ip < P.m; ip += g.size()) {
    if (!(P.fl(ip) & 2)) continue;
    int iq = P.nb(ip);
    if (iq >= 0 && (Q.fl(iq) & 2)) { P.lb(ip) = L_CROSSING; Q.lb(iq) = L_CROSSING; }
  }
  g.sync();
}

// Run-table tracing for warp-sized pairs: the table is kept per ring slot (tl, tn, to),
// which saves the slot-to-index translation of the indexed variant below; the walk marks
// visited vertices in the rings' intersection flags.  Same phases and results.
template <class G>
__device__ int grp_trace_runs_slots(const G& g, PairCtx& c) {
  int nF[2];
  bool mismatch = false;     // a flagged vertex that is not a crossing, or the reverse
  for (int sd = 0; sd < 2; ++sd) {
    Ring& A = c.R[sd];
    int carry = 0;
    for (int b = 0; b < A.m; b += g.size()) {
      const int s = b + g.rank();
      const int f = (s < A.m && (A.ee(s) == E_ENTRY || A.ee(s) == E_EXIT)) ? 1 : 0;
      if (s < A.m && (f != 0) != (A.it(s) && A.lb(s) == L_CROSSING)) mismatch = true;
      int tot;
      const int incl = g.incl_scan(f, tot);
      if (f) A.ls(carry + incl - 1) = s;
      carry += tot;
    }
    nF[sd] = carry;
  }
  if (g.any(mismatch)) return 1;
  if (nF[0] == 0 && nF[1] == 0) return 0;
  bool bad = nF[0] < 2 || nF[1] < 2;
  bool longRun = false;
  for (int sd = 0; sd < 2 && !bad; ++sd) {
    Ring& A = c.R[sd];
    const Ring& B = c.R[1 - sd];
    const int n = nF[sd], m = A.m;
    for (int i = g.rank(); i < n; i += g.size()) {
      const int s = A.ls(i);
      const int8_t e = A.ee(s);
      if (!A.it(s) || A.lb(s) != L_CROSSING) { bad = true; continue; }
      if (A.ee(A.ls((i + 1 < n) ? i + 1 : 0)) == e) { bad = true; continue; }   // alternation
      const int nb = A.nb(s);
      if (nb < 0 || nb >= B.m || B.ee(nb) != toggled(e)) { bad = true; continue; }
      const int8_t st = toggled(e);
      const int dir = ((st == E_EXIT) ^ c.uni) ? 1 : -1;
      const int W = A.ls((i + dir + n) % n);
      int L = dir > 0 ? W - s : s - W;
      if (L <= 0) L += m;
      const int nbW = A.nb(W);
      if (nbW < 0 || nbW >= B.m) { bad = true; continue; }
      A.tl(s) = dir * L;
      A.tn(s) = nbW;
      A.to(s) = -1;
      if (L > 32) longRun = true;
    }
  }
  if (g.any(bad)) return 1;
  const bool anyLong = g.any(longRun);
  // ---- phase 2: the walk over the run table, one member
  OutRegion& O = c.O;
  int status = 0;
  int64_t nv = O.nv;
  int nc = O.nc;
  if (g.rank() == 0) {
    Ring& P = c.R[0];
    const int64_t nv0 = O.nv;
    long long budget = (long long)nF[0] + nF[1] + 4;
    for (int i = 0; i < nF[0] && status == 0; ++i) {
      const int I = P.ls(i);
      if (!P.it(I)) continue;
      if (nc >= O.ccap) { status = -1; fail(c, DEV_CAPACITY); break; }
      P.it(I) = 0;
      int side = 0, V = I;
      int64_t csz = 0;
      for (;;) {
        Ring& C = c.R[side];
        const int t = C.tl(V), L = t < 0 ? -t : t, m = C.m;
        int W = V + t % m;
        W = (W % m + m) % m;
        C.to(V) = (int32_t)(nv - nv0);
        nv += L;
        csz += L;
        C.it(W) = 0;
        if (side == 0 && W == I) break;
        const int V2 = C.tn(V);
        side ^= 1;
        if (side == 0 && V2 == I) break;
        c.R[side].it(V2) = 0;
        V = V2;
        if (--budget < 0) { status = -1; fail(c, DEV_TRACE); break; }
      }
      if (status == 0) {
        if (nv > O.vcap) { status = -1; fail(c, DEV_CAPACITY); break; }
        O.csz[nc++] = (int32_t)csz;
      }
    }
  }
  status = g.bcast0(status);
  if (status != 0) return -1;
  const int64_t nv0 = O.nv;
  O.nv = g.bcast0((long long)nv);
  O.nc = g.bcast0(nc);
  // ---- phase 3: copy every run to its place; short runs one member each, long runs by
  // the whole group (no barrier between runs: runs write disjoint ranges)
  constexpr int kShortRun = 32;      // the run-length threshold of phase 1's longRun
  for (int sd = 0; sd < 2; ++sd) {
    const Ring& A = c.R[sd];
    const int m = A.m;
    for (int i = g.rank(); i < nF[sd]; i += g.size()) {
      const int s = A.ls(i);
      const int off = A.to(s);
      if (off < 0) continue;
      const int t = A.tl(s), L = t < 0 ? -t : t, dir = t < 0 ? -1 : 1;
      if (anyLong && L > kShortRun) continue;
      double* dst = O.xy + 2 * (nv0 + off);
      int w = s;
      for (int j = 0; j < L; ++j) {
        w += dir;
        if (w >= m) w -= m;
        if (w < 0) w += m;
        dst[2 * j] = A.x(w);
        dst[2 * j + 1] = A.y(w);
      }
    }
    for (int i = 0; anyLong && i < nF[sd]; ++i) {
      const int s = A.ls(i);
      const int off = A.to(s);
      const int t = A.tl(s), L = t < 0 ? -t : t;
      if (off < 0 || L <= kShortRun) continue;
      const int dir = t < 0 ? -1 : 1;
      double* dst = O.xy + 2 * (nv0 + off);
      for (int j = g.rank(); j < L; j += g.size()) {
        int w = s + dir * (j + 1);
        w %= m;
        if (w < 0) w += m;
        dst[2 * j] = A.x(w);
        dst[2 * j + 1] = A.y(w);
      }
    }
  }
  g.sync();
  return 0;
}

// Tracing from a run table.  With entry/exit flags alternating along both rings (checked
// here), every run of the sequential walk goes from a flagged vertex to the adjacent
// flagged vertex in its direction, and the next run starts at that vertex's neighbour.
// Phase 1 (parallel) lists the flagged slots of each ring and gives each flagged vertex
// (by its index in that list) its run: the length, signed by direction, and the index of
// the next run's start on the other ring.  Phase 2 (one member) follows the runs in the
// order of the sequential walk -- components from the first unvisited crossing of P, in
// P's slot order -- and assigns each run its output offset.  Phase 3 (parallel) copies
// the runs.  Indexing the table by flagged vertex keeps the walk's visited marks in the
// table itself, so the walk touches no ring array.  Returns 0 when done, 1
// when the flags do not alternate (the caller then runs the general walk), -1 on a
// capacity or trace error.
template <class G>
__device__ int grp_trace_runs(const G& g, PairCtx& c) {
  int nF[2];
  bool mismatch = false;     // a flagged vertex that is not a crossing, or the reverse
  for (int sd = 0; sd < 2; ++sd) {
    Ring& A = c.R[sd];
    int carry = 0;
    for (int b = 0; b < A.m; b += g.size()) {
      const int s = b + g.rank();
      const int f = (s < A.m && (A.ee(s) == E_ENTRY || A.ee(s) == E_EXIT)) ? 1 : 0;
      if (s < A.m && (f != 0) != (A.it(s) && A.lb(s) == L_CROSSING)) mismatch = true;
      int tot;
      const int incl = g.incl_scan(f, tot);
      if (f) { A.ls(carry + incl - 1) = s; A.to(s) = carry + incl - 1; }   // slot -> index
      carry += tot;
    }
    nF[sd] = carry;
  }
  if (g.any(mismatch)) return 1;
  if (nF[0] == 0 && nF[1] == 0) return 0;
  // run table by list index, in the rings' scratch arrays: length RL, next start RN (sign
  // bit = visited), output offset RO.  The slot -> index map in `to` is read until phase 1
  // ends; the offsets take its place then.  (Pointers are selected per side in registers.)
  int32_t* RL0 = &c.R[0].tl(0); int32_t* RL1 = &c.R[1].tl(0);
  int32_t* RN0 = &c.R[0].tn(0); int32_t* RN1 = &c.R[1].tn(0);
  int32_t* RO0 = &c.R[0].to(0); int32_t* RO1 = &c.R[1].to(0);
#define RL_(sd) ((sd) ? RL1 : RL0)
#define RN_(sd) ((sd) ? RN1 : RN0)
#define RO_(sd) ((sd) ? RO1 : RO0)
  bool bad = nF[0] < 2 || nF[1] < 2;
  bool longRun = false;
  for (int sd = 0; sd < 2 && !bad; ++sd) {
    Ring& A = c.R[sd];
    const Ring& B = c.R[1 - sd];
    const int n = nF[sd], m = A.m;
    for (int i = g.rank(); i < n; i += g.size()) {
      const int s = A.ls(i);
      const int8_t e = A.ee(s);
      if (A.ee(A.ls((i + 1 < n) ? i + 1 : 0)) == e) { bad = true; continue; }   // alternation
      const int nb = A.nb(s);
      if (nb < 0 || nb >= B.m || B.ee(nb) != toggled(e)) { bad = true; continue; }
      const int8_t st = toggled(e);
      const int dir = ((st == E_EXIT) ^ c.uni) ? 1 : -1;
      const int W = A.ls((i + dir + n) % n);
      int L = dir > 0 ? W - s : s - W;
      if (L <= 0) L += m;
      const int nbW = A.nb(W);
      if (nbW < 0 || nbW >= B.m) { bad = true; continue; }
      RL_(sd)[i] = dir * L;
      RN_(sd)[i] = B.to(nbW);          // a flagged twin (checked): its index in B's list
      if (L > 32) longRun = true;
    }
  }
  if (g.any(bad)) return 1;
  if constexpr (G::kBlock) {
    // The walk below is one long chain of dependent loads: with the table in shared
    // memory each step costs tens of cycles instead of an L2 round trip.
    if (nF[0] + nF[1] <= g.runsCap) {
      int32_t* sh = g.runs;
      int32_t* dst[6] = {sh, sh + nF[0], sh + 2 * nF[0], sh + 3 * nF[0], sh + 3 * nF[0] + nF[1],
                         sh + 3 * nF[0] + 2 * nF[1]};
      for (int sd = 0; sd < 2; ++sd)
        for (int i = g.rank(); i < nF[sd]; i += g.size()) {
          dst[3 * sd][i] = RL_(sd)[i];
          dst[3 * sd + 1][i] = RN_(sd)[i];
        }
      RL0 = dst[0]; RN0 = dst[1]; RO0 = dst[2];
      RL1 = dst[3]; RN1 = dst[4]; RO1 = dst[5];
    }
  }
  for (int sd = 0; sd < 2; ++sd)
    for (int i = g.rank(); i < nF[sd]; i += g.size()) RO_(sd)[i] = -1;
  const bool anyLong = g.any(longRun);
  // ---- phase 2: the walk over the run table, one member
  constexpr int32_t kSeen = (int32_t)0x80000000u;
  OutRegion& O = c.O;
  int status = 0;
  int64_t nv = O.nv;
  int nc = O.nc;
  if (g.rank() == 0) {
    const int64_t nv0 = O.nv;
    const int nFP = nF[0], nFQ = nF[1];
    long long budget = (long long)nFP + nFQ + 4;
    for (int I = 0; I < nFP && status == 0; ++I) {
      if (RN_(0)[I] < 0) continue;                       // visited
      if (nc >= O.ccap) { status = -1; fail(c, DEV_CAPACITY); break; }
      RN_(0)[I] |= kSeen;
      int side = 0, V = I;
      int64_t csz = 0;
      for (;;) {
        const int t = RL_(side)[V], L = t < 0 ? -t : t, n = side ? nFQ : nFP;
        int W = V + (t < 0 ? -1 : 1);
        if (W >= n) W -= n;
        if (W < 0) W += n;
        RO_(side)[V] = (int32_t)(nv - nv0);
        nv += L;
        csz += L;
        const int V2 = RN_(side)[V] & 0x7fffffff;
        RN_(side)[W] |= kSeen;
        if (side == 0 && W == I) break;
        side ^= 1;
        if (side == 0 && V2 == I) break;
        RN_(side)[V2] |= kSeen;
        V = V2;
        if (--budget < 0) { status = -1; fail(c, DEV_TRACE); break; }
      }
      if (status == 0) {
        if (nv > O.vcap) { status = -1; fail(c, DEV_CAPACITY); break; }
        O.csz[nc++] = (int32_t)csz;
      }
    }
  }
  status = g.bcast0(status);
  if (status != 0) return -1;
  const int64_t nv0 = O.nv;
  O.nv = g.bcast0((long long)nv);
  O.nc = g.bcast0(nc);
  // ---- phase 3: copy every run to its place; short runs one member each, long runs by
  // the whole group (no barrier between runs: runs write disjoint ranges)
  constexpr int kShortRun = 32;      // the run-length threshold of phase 1's longRun
  for (int sd = 0; sd < 2; ++sd) {
    const Ring& A = c.R[sd];
    const int m = A.m;
    for (int i = g.rank(); i < nF[sd]; i += g.size()) {
      const int off = RO_(sd)[i];
      if (off < 0) continue;
      const int t = RL_(sd)[i], L = t < 0 ? -t : t, dir = t < 0 ? -1 : 1;
      if (anyLong && L > kShortRun) continue;
      double* dst = O.xy + 2 * (nv0 + off);
      int w = A.ls(i);
      for (int j = 0; j < L; ++j) {
        w += dir;
        if (w >= m) w -= m;
        if (w < 0) w += m;
        dst[2 * j] = A.x(w);
        dst[2 * j + 1] = A.y(w);
      }
    }
    for (int i = 0; anyLong && i < nF[sd]; ++i) {
      const int off = RO_(sd)[i];
      const int t = RL_(sd)[i], L = t < 0 ? -t : t;
      if (off < 0 || L <= kShortRun) continue;
      const int dir = t < 0 ? -1 : 1, s0 = A.ls(i);
      double* dst = O.xy + 2 * (nv0 + off);
      for (int j = g.rank(); j < L; j += g.size()) {
        int w = s0 + dir * (j + 1);
        w %= m;
        if (w < 0) w += m;
        dst[2 * j] = A.x(w);
        dst[2 * j + 1] = A.y(w);
      }
    }
  }
  g.sync();
  return 0;
#undef RL_
#undef RN_
#undef RO_
}

// Tracing when neither ring has added vertices (rings in slot order): each run from V to
// the next vertex with the target entry/exit flag (or back at the start) is found with a
// group ballot and copied with coalesced stores.
template <class G>
__device__ bool grp_trace(const G& g, PairCtx& c) {
  Ring& P = c.R[0];
  OutRegion& O = c.O;
  long long budget = 4ll * (c.R[0].used + c.R[1].used) + 16;
  int from = 0;
  for (;;) {
    int I = grp_find_first(g, from, P.m, [&](int s) { return P.it(s) && P.lb(s) == L_CROSSING; });
    if (I >= P.m) break;
    O.begin();
    if (O.overflow) { if (g.rank() == 0) fail(c, DEV_CAPACITY); return false; }
    int side = 0, V = I;
    if (g.rank() == 0) P.it(V) = 0;
    g.sync();
    do {
      Ring& C = c.R[side];
      const int m = C.m;
      int8_t st = toggled(C.ee(V));
      const int dir = ((st == E_EXIT) ^ c.uni) ? 1 : -1;
      int L = -1;
      for (int j0 = 1; j0 <= m && L < 0; j0 += g.size()) {
        int j = j0 + g.rank();
        bool hit = false;
        if (j <= m) {
          int w = V + dir * (j % m);
          w = (w % m + m) % m;
          hit = (C.ee(w) == st) || (side == 0 && w == I);
        }
        int f = g.first(hit);
        if (f >= 0) L = j0 + f;
      }
      if (L < 0) { if (g.rank() == 0) fail(c, DEV_TRACE); return false; }
      budget -= L;
      if (budget < 0) { if (g.rank() == 0) fail(c, DEV_TRACE); return false; }
      if (O.nv + L > O.vcap) { if (g.rank() == 0) fail(c, DEV_CAPACITY); return false; }
      for (int j0 = 1; j0 <= L; j0 += g.size()) {
        int j = j0 + g.rank();
        if (j <= L) {
          int w = V + dir * (j % m);
          w = (w % m + m) % m;
          C.it(w) = 0;
          O.xy[2 * (O.nv + j - 1)] = C.x(w);
          O.xy[2 * (O.nv + j - 1) + 1] = C.y(w);
        }
      }
      O.nv += L;
      if (g.rank() == 0) O.csz[O.nc] += L;
      int W = V + dir * (L % m);
      V = (W % m + m) % m;
      g.sync();
      if (!(side == 0 && V == I)) {
        int nb = C.nb(V);
        if (nb < 0) { if (g.rank() == 0) fail(c, DEV_TRACE); return false; }
        V = nb;
        side = 1 - side;
        if (g.rank() == 0) c.R[side].it(V) = 0;
        g.sync();
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
template <class G>
__device__ void grp_cleanup(const G& g, PairCtx& c, int32_t* outNC, int64_t* outNV) {
  OutRegion& O = c.O;
  // Fast pass for pairs with many components: test every vertex of every component at
  // once (short components one member each, long ones by the whole group).  When nothing
  // is removable, the output stands as traced; otherwise (and for pairs with few
  // components) the per-component pass below removes and compacts.
  if (O.nc > 4) {
    int32_t* start = &c.R[0].tn(0);      // the trace's scratch is free now
    int carry = 0;
    for (int b = 0; b < O.nc; b += g.size()) {
      const int k = b + g.rank();
      const int v = (k < O.nc) ? O.csz[k] : 0;
      int tot;
      const int incl = g.incl_scan(v, tot);
      if (k < O.nc) start[k] = carry + incl - v;
      carry += tot;
    }
    g.sync();
    constexpr int kShortComp = 64;
    bool any = false;
    for (int k = g.rank(); k < O.nc; k += g.size()) {
      const int n = O.csz[k];
      if (n > kShortComp) continue;
      const double* src = O.xy + 2 * (int64_t)start[k];
      for (int j = 0; j < n && !any; ++j) {
        int p = (j > 0) ? j - 1 : n - 1, q = (j + 1 < n) ? j + 1 : 0;
        if (fabs(area2(src[2 * p], src[2 * p + 1], src[2 * j], src[2 * j + 1], src[2 * q], src[2 * q + 1])) <
            c.eps_clean)
          any = true;
      }
    }
    for (int k = 0; k < O.nc; ++k) {
      const int n = O.csz[k];
      if (n <= kShortComp) continue;
      const double* src = O.xy + 2 * (int64_t)start[k];
      for (int j = g.rank(); j < n && !any; j += g.size()) {
        int p = (j > 0) ? j - 1 : n - 1, q = (j + 1 < n) ? j + 1 : 0;
        if (fabs(area2(src[2 * p], src[2 * p + 1], src[2 * j], src[2 * j + 1], src[2 * q], src[2 * q + 1])) <
            c.eps_clean)
          any = true;
      }
    }
    if (!g.any(any)) {
      if (g.rank() == 0) { *outNC = O.nc; *outNV = O.nv; }
      return;
    }
    if constexpr (!G::kSolo) {
      // Removal with many components: each member cleans whole components in place (a
      // component's kept vertices move to the front of its own range), then the kept
      // vertices are compacted, through ring P's coordinate column (free after the
      // trace) when they fit there.  Per component this is the sequential pass.
      int32_t* keptA = &c.R[0].ls(0);
      int32_t* dstA = &c.R[0].tl(0);
      for (int k = g.rank(); k < O.nc; k += g.size()) {
        double* src = O.xy + 2 * (int64_t)start[k];
        keptA[k] = seq_cleanup_component(src, src, O.csz[k], c.eps_clean);
      }
      g.sync();
      long long total = 0;
      for (int b = 0; b < O.nc; b += g.size()) {
        const int k = b + g.rank();
        const int v = (k < O.nc) ? keptA[k] : 0;
        int tot;
        const int incl = g.incl_scan(v, tot);
        if (k < O.nc) dstA[k] = (int32_t)(total + incl - v);
        total += tot;
      }
      g.sync();
      if (total <= (long long)c.R[0].cap) {
        double2* stage = &c.R[0].xy(0);
        for (int k = g.rank(); k < O.nc; k += g.size()) {
          const int kept = keptA[k];
          const double* src = O.xy + 2 * (int64_t)start[k];
          double2* dst = stage + dstA[k];
          for (int j = 0; j < kept; ++j) dst[j] = make_double2(src[2 * j], src[2 * j + 1]);
        }
        g.sync();
        for (long long t = g.rank(); t < total; t += g.size()) {
          const double2 v = stage[t];
          O.xy[2 * t] = v.x;
          O.xy[2 * t + 1] = v.y;
        }
      } else {
        long long vout = 0;
        for (int k = 0; k < O.nc; ++k) {
          const int kept = keptA[k];
          const double* src = O.xy + 2 * (int64_t)start[k];
          double* dst = O.xy + 2 * vout;
          if (kept > 0 && dst != src) {
            for (int b = 0; b < 2 * kept; b += g.size()) {
              const int i = b + g.rank();
              const double v = (i < 2 * kept) ? src[i] : 0.0;
              g.sync();
              if (i < 2 * kept) dst[i] = v;
            }
          }
          g.sync();
          vout += kept;
        }
      }
      g.sync();
      int cc = 0;
      for (int b = 0; b < O.nc; b += g.size()) {
        const int k = b + g.rank();
        const int f = (k < O.nc && keptA[k] > 0) ? 1 : 0;
        int tot;
        const int incl = g.incl_scan(f, tot);
        if (f) O.csz[cc + incl - 1] = keptA[k];
        cc += tot;
      }
      if (g.rank() == 0) { *outNC = cc; *outNV = (int64_t)total; }
      g.sync();
      return;
    }
  }
  int64_t vin = 0, vout = 0;
  int nc = 0;
  for (int k = 0; k < O.nc; ++k) {
    const int n = O.csz[k];
    const double* src = O.xy + 2 * vin;
    double* dst = O.xy + 2 * vout;
    bool flag = false;
    for (int j = g.rank(); j < n; j += g.size()) {
      int p = (j > 0) ? j - 1 : n - 1, q = (j + 1 < n) ? j + 1 : 0;
      if (fabs(area2(src[2 * p], src[2 * p + 1], src[2 * j], src[2 * j + 1], src[2 * q], src[2 * q + 1])) <
          c.eps_clean)
        flag = true;
    }
    flag = g.any(flag);
    int kept;
    if (!flag) {
      if (dst != src) {
        for (int b = 0; b < 2 * n; b += g.size()) {
          int i = b + g.rank();
          double v = (i < 2 * n) ? src[i] : 0.0;
          g.sync();
          if (i < 2 * n) dst[i] = v;
        }
      }
      kept = n;
    } else {
      kept = 0;
      if (g.rank() == 0) kept = seq_cleanup_component(src, dst, n, c.eps_clean);
      kept = g.bcast0(kept);
    }
    g.sync();
    vin += n;
    if (kept == 0) continue;
    if (g.rank() == 0) O.csz[nc] = kept;
    ++nc;
    vout += kept;
    g.sync();
  }
  if (g.rank() == 0) { *outNC = nc; *outNV = vout; }
}

// Pulls a pair's ring arrays into L1 in one burst, one request per 128-byte line, so the
// labelling phases (each of which touches some of the arrays first) do not pay a DRAM
// round trip each.
__device__ __forceinline__ void prefetch_l1(const void* p) {
  asm volatile("prefetch.global.L1 [%0];" ::"l"(p));
}

template <class G>
__device__ void prefetch_ring(const G& g, const Ring& R) {
  for (int s = g.rank() * 8; s < R.m; s += g.size() * 8) {
    prefetch_l1(&R.xy(s));
    if ((s & 31) == 0) { prefetch_l1(&R.nx(s)); prefetch_l1(&R.pv(s)); prefetch_l1(&R.nb(s)); }
    if ((s & 127) == 0) { prefetch_l1(&R.it(s)); prefetch_l1(&R.lb(s)); prefetch_l1(&R.ee(s)); prefetch_l1(&R.fl(s)); }
  }
}

// Arguments of the labelling kernels (one struct so the warp and block kernels agree).
struct LabelArgs {
  PairDev D;
  int64_t K;
  const int32_t* mP; const int32_t* mQ;
  const int64_t* regP; const int64_t* regQ;
  const int64_t* regSizeP; const int64_t* regSizeQ;
  RingSet SP, SQ;
  double* outXY; const int64_t* outVOff; const int64_t* outVCap;
  int32_t* outCsz; const int64_t* outCOff; const int32_t* outCCap;
  int32_t* outNC; int64_t* outNV;
  ClipParams prm;
  int* err;
  int64_t tileLabelMax;       // rings up to: a tile of lanes per pair
  int64_t midLabelMin;        // rings above: a block per pair
  int64_t bigLabelMin;        // rings above: the grid path
  const unsigned long long* midCount;
  unsigned long long* midNext; // work-stealing cursor of the block kernel
  int blockRunCap;            // runs the block kernel's shared run table holds (0: none)
  // The one-thread, warp and block pairs in size order, largest first (label_order_kernel):
  // the one-thread kernel takes order[0, nTile), the warp kernel order[nTile, nTile + nWarp),
  // the block kernel the *midCount entries after those.
  const uint32_t* order;
  int64_t nTile, nWarp;
};

// One pair labelled and traced by group g.  The group phases give the sequential result
// whenever neighbour links are one-to-one (then labels written through a link never
// collide) and chains are well formed; otherwise member 0 runs the sequential phases from
// the first one that could differ.
template <int EX, class G>
__device__ void label_trace_pair(const G& g, const LabelArgs& a, int64_t k) {
  const bool lead = g.rank() == 0;
  int32_t* outNC = a.outNC + k;
  int64_t* outNV = a.outNV + k;
  PairCtx c;
  c.R[0] = ring_of(a.SP, a.regP[k], a.mP[k], (int)a.regSizeP[k]);
  c.R[1] = ring_of(a.SQ, a.regQ[k], a.mQ[k], (int)a.regSizeQ[k]);
  c.O.xy = a.outXY + 2 * a.outVOff[k]; c.O.csz = a.outCsz + a.outCOff[k];
  c.O.vcap = a.outVCap[k]; c.O.ccap = a.outCCap[k];
  c.O.nv = 0; c.O.nc = 0; c.O.overflow = false;
  c.uni = a.prm.union_mode != 0;
  c.eps_clean = a.prm.eps_clean;
  c.err = a.err;
  c.status = a.D.status + k;
  c.noInter[0] = c.noInter[1] = c.ident[0] = c.ident[1] = false;
  prefetch_ring(g, c.R[0]);
  prefetch_ring(g, c.R[1]);

  if (!grp_links_one_to_one(g, c.R[0], c.R[1])) {
    if (lead) seq_pair_from<EX>(c, 1, outNC, outNV);
    g.sync();
    return;
  }
  grp_step1<EX>(g, c);
  if (!grp_step2(g, c)) {
    if (lead) seq_pair_from<EX>(c, 2, outNC, outNV);
    g.sync();
    return;
  }
  grp_step35<EX>(g, c);
  int tempAfter[2], tempSlot[2];
  if (!grp_step4<EX>(g, c, tempAfter, tempSlot)) return;
  if (grp_any_split(g, c.R[0], c.R[1])) {
    bool ok = true;
    if (lead) ok = seq_step5<EX>(c);
    ok = g.bcast0((int)ok);
    c.R[0].used = g.bcast0(c.R[0].used);
    c.R[1].used = g.bcast0(c.R[1].used);
    g.sync();
    if (!ok) return;
  }
  grp_step6(g, c);
  const bool added = c.R[0].used != c.R[0].m || c.R[1].used != c.R[1].m;
  if (added) {
    // vertices were added to a ring: trace through the next/prev links on one member
    int ok = 1;
    if (lead) ok = seq_trace(c) ? 1 : 0;
    ok = g.bcast0(ok);
    c.O.nv = g.bcast0((long long)c.O.nv);
    c.O.nc = g.bcast0(c.O.nc);
    c.O.overflow = g.bcast0((int)c.O.overflow) != 0;
    g.sync();
    if (!ok) return;
  } else {
    int r;
    if constexpr (G::kBlock) r = grp_trace_runs(g, c);
    else r = grp_trace_runs_slots(g, c);
    if (r < 0) return;
    if (r > 0 && !grp_trace(g, c)) return;
  }
  if (c.O.overflow) {
    if (lead) fail(c, DEV_CAPACITY);
    return;
  }
  grp_cleanup(g, c, outNC, outNV);
}

// Two register budgets for the warp and one-thread kernels.  kWide (batches of at least
// ClipParams::wide_label_min pairs): 6 blocks of 128 (at most 80 registers) here and 12 blocks (40
// registers) for the tiles below -- both kernels wait on dependent loads, and on a full
// GPU the occupancy pays for the spills (label stage 2.59 -> 2.11 ms from the tile kernel,
// -0.07 ms from this one; with the column-buffer rings, 12 tile blocks measured 2.00 ms
// against 2.08 ms for 16).  Small batches (serving) leave most SMs idle, so there the
// kernels keep 4 blocks and spill nothing.  Exact-predicate instances always keep 4
// blocks: their expansion arithmetic would spill.
template <int EX, int kWide>
__global__ void __launch_bounds__(128, (kWide && !EX) ? 6 : 4)
label_trace_kernel(LabelArgs a) {
  const int64_t w = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (w >= a.nWarp) return;
  WarpGroup g;
  label_trace_pair<EX>(g, a, (int64_t)a.order[a.nTile + w]);
}

// Pairs whose merged rings have at most tileLabelMax slots: one thread per pair
// (SoloGroup, measured slightly faster than 2-lane tiles on the batched workload), the
// pairs in size order so that the 32 pairs of a warp take about as long as each other.
template <int EX, int kWide>
__global__ void __launch_bounds__(128, (kWide && !EX) ? 12 : 4)
label_trace_tile_kernel(LabelArgs a) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.nTile) return;
  SoloGroup g;
  label_trace_pair<EX>(g, a, (int64_t)a.order[i]);
}

// sizes in the labelling order, and the scanned offsets back to pair order
__global__ void permute_sizes_kernel(const uint32_t* __restrict__ order, int64_t K, const int64_t* __restrict__ sP,
                                     const int64_t* __restrict__ sQ, int64_t* __restrict__ oP, int64_t* __restrict__ oQ) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= K) return;
  const uint32_t k = order[i];
  oP[i] = sP[k];
  oQ[i] = sQ[k];
}

__global__ void unpermute_offsets_kernel(const uint32_t* __restrict__ order, int64_t K,
                                         const int64_t* __restrict__ offP, const int64_t* __restrict__ offQ,
                                         int64_t* __restrict__ regP, int64_t* __restrict__ regQ) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= K) return;
  const uint32_t k = order[i];
  regP[k] = offP[i];
  regQ[k] = offQ[i];
}

// Sort keys of the pairs by labelling class and size, for one 8-bit radix pass: one-thread
// pairs 0..84, warp pairs 85..169, block pairs 170..254 (85 size buckets each, largest
// first; the block class on a log scale, so that its largest pairs start first and do not
// trail the stage), the rest 255.  Class counts: cnt[2] one-thread, cnt[3] warp, cnt[0] block.
__global__ void label_order_kernel(const int32_t* __restrict__ mP, const int32_t* __restrict__ mQ,
                                   const int32_t* __restrict__ status, int64_t K, int64_t tileMax, int64_t midMin,
                                   int64_t bigMin, uint64_t* __restrict__ key, uint32_t* __restrict__ val,
                                   unsigned long long* __restrict__ cnt) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= K) return;
  const int64_t slots = (int64_t)mP[k] + mQ[k];
  const int64_t tl = tileMax < midMin ? tileMax : midMin;
  uint64_t kk = 255;
  if (status[k] == 0 && slots <= midMin) {
    if (slots <= tl) {
      kk = 84 - (uint64_t)((slots * 85) / (tl + 1));
      atomicAdd(cnt + 2, 1ull);
    } else {
      kk = 169 - (uint64_t)(((slots - tl) * 85) / (midMin - tl + 1));
      atomicAdd(cnt + 3, 1ull);
    }
  } else if (status[k] == 0 && slots <= bigMin) {
    const double r = log2((double)slots / (double)midMin) / log2((double)bigMin / (double)midMin);
    const int b = (int)fmin(84.0, fmax(0.0, 85.0 * r));
    kk = 254 - (uint64_t)b;
    atomicAdd(cnt, 1ull);
  }
  key[k] = kk;
  val[k] = (uint32_t)k;
}

// Pairs with midLabelMin < slots <= bigLabelMin: persistent blocks take pairs from the
// list through an atomic cursor (work stealing), one block of kBlockLabelThreads per pair.
template <int EX>
__global__ void __launch_bounds__(kBlockLabelThreads)
label_trace_block_kernel(LabelArgs a) {
  __shared__ long long sm[kBlockLabelThreads / 32 + 1];
  __shared__ long long next;
  extern __shared__ int32_t runTable[];
  BlockGroup g{sm, runTable, a.blockRunCap};
  const unsigned long long n = *a.midCount;
  for (;;) {
    if (threadIdx.x == 0) next = (long long)atomicAdd(a.midNext, 1ull);
    __syncthreads();
    const long long i = next;
    __syncthreads();
    if (i >= (long long)n) return;
    label_trace_pair<EX>(g, a, (int64_t)a.order[a.nTile + a.nWarp + i]);
    __syncthreads();
  }
}


// ================================================================ grid path for huge pairs
// Pairs whose merged rings exceed ClipParams::big_label_min slots are labelled and traced
// by grid-wide kernels, one phase per launch over the pair's ring slots, with the
// host reading the few per-pair flags between phases.  The phases give the sequential
// result under the same conditions as the warp path; otherwise one thread runs the
// sequential phases from the first one that could differ.
struct BigPair {
  int64_t k, regP, regQ, vOff, vCap, cOff;
  int32_t mP, mQ, capP, capQ, cCap, pad;
};

struct BigFlags {
  int bad;
  int notNone[2];
  int notAllOn[2];
  int firstFree[2];
  int firstMid[2];
  int anySplit;
  int pad;
  unsigned long long wind;
};

__device__ __forceinline__ Ring big_ring(const RingSet& S, int64_t reg, int m, int cap, int used) {
  Ring r = ring_of(S, reg, m, cap);
  r.used = used;
  return r;
}

// 0: P, 1: Q of one pair; slot s of ring A; its ring successor/predecessor before any
// vertex is added
__device__ __forceinline__ int nxt_slot(int s, int m) { return (s + 1 < m) ? s + 1 : 0; }
__device__ __forceinline__ int prv_slot(int s, int m) { return (s > 0) ? s - 1 : m - 1; }

__global__ void big_links_kernel(RingSet SP, RingSet SQ, BigPair bp, BigFlags* f) {
  Ring P = big_ring(SP, bp.regP, bp.mP, bp.capP, bp.mP), Q = big_ring(SQ, bp.regQ, bp.mQ, bp.capQ, bp.mQ);
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < (int64_t)P.m + Q.m;
       i += (int64_t)gridDim.x * blockDim.x) {
    bool bad = false;
    if (i < P.m) {
      int s = (int)i;
      if (P.it(s)) { int nb = P.nb(s); bad = nb < 0 || nb >= Q.m || Q.nb(nb) != s; }
    } else {
      int s = (int)(i - P.m);
      if (Q.it(s)) { int nb = Q.nb(s); bad = nb < 0 || nb >= P.m || P.nb(nb) != s; }
    }
    if (bad) atomicOr(&f->bad, 1);
  }
}

template <int EX>
__global__ void big_step1_kernel(RingSet SP, RingSet SQ, BigPair bp) {
  Ring P = big_ring(SP, bp.regP, bp.mP, bp.capP, bp.mP), Q = big_ring(SQ, bp.regQ, bp.mQ, bp.capQ, bp.mQ);
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < P.m; s += gridDim.x * blockDim.x) {
    if (!P.it(s)) continue;
    int nb = P.nb(s);
    int pm = prv_slot(s, P.m), pp = nxt_slot(s, P.m);
    int a = rel_position<EX>(P, Q, prv_slot(nb, Q.m), pm, s, pp);
    int b = rel_position<EX>(P, Q, nxt_slot(nb, Q.m), pm, s, pp);
    int8_t L = initial_label(a, b);
    if (L != L_NONE) { P.lb(s) = L; Q.lb(nb) = L; }
  }
}

// kMode 0: every chain must end at an ON_LEFT/ON_RIGHT intersection vertex; 1: resolve
template <int kMode>
__global__ void big_chain_kernel(RingSet SP, RingSet SQ, BigPair bp, BigFlags* f) {
  Ring P = big_ring(SP, bp.regP, bp.mP, bp.capP, bp.mP), Q = big_ring(SQ, bp.regQ, bp.mQ, bp.capQ, bp.mQ);
  const int m = P.m;
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < m; s += gridDim.x * blockDim.x) {
    int8_t l0 = P.lb(s);
    if (!P.it(s) || (l0 != L_LEFT_ON && l0 != L_RIGHT_ON)) continue;
    int I = nxt_slot(s, m), guard = m;
    if (kMode == 0) {
      while (P.lb(I) == L_ON_ON && --guard > 0) I = nxt_slot(I, m);
      if ((P.lb(I) != L_ON_LEFT && P.lb(I) != L_ON_RIGHT) || !P.it(I)) atomicOr(&f->bad, 1);
    } else {
      int x = l0 == L_LEFT_ON ? R_LEFT : R_RIGHT;
      Q.lb(P.nb(s)) = L_NONE;
      while (P.lb(I) == L_ON_ON) {
        P.lb(I) = L_NONE;
        Q.lb(P.nb(I)) = L_NONE;
        I = nxt_slot(I, m);
      }
      int y = P.lb(I) == L_ON_LEFT ? R_LEFT : R_RIGHT;
      int8_t ct = (x != y) ? L_DELAYED_CROSSING : L_DELAYED_BOUNCING;
      P.lb(s) = ct; P.lb(I) = ct;
      Q.lb(P.nb(s)) = ct; Q.lb(P.nb(I)) = ct;
    }
  }
}

// special-case flags of both rings (polygon.h:453-512 on the rings before any insertion)
__global__ void big_flags_kernel(RingSet SP, RingSet SQ, BigPair bp, int uni, BigFlags* f) {
  Ring R[2] = {big_ring(SP, bp.regP, bp.mP, bp.capP, bp.mP), big_ring(SQ, bp.regQ, bp.mQ, bp.capQ, bp.mQ)};
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < (int64_t)R[0].m + R[1].m;
       i += (int64_t)gridDim.x * blockDim.x) {
    int sd = i < R[0].m ? 0 : 1;
    int v = (int)(sd == 0 ? i : i - R[0].m);
    const Ring& A = R[sd];
    const Ring& B = R[1 - sd];
    int8_t l = A.lb(v);
    if (l != L_ON_ON) atomicOr(&f->notAllOn[sd], 1);
    if (A.it(v)) {
      if (l == L_CROSSING || l == L_DELAYED_CROSSING) atomicOr(&f->notNone[sd], 1);
      if (uni && (l == L_BOUNCING || l == L_DELAYED_BOUNCING)) atomicOr(&f->notNone[sd], 1);
    } else {
      atomicMin(&f->firstFree[sd], v);
    }
    int nb = A.nb(v), nx = nxt_slot(v, A.m);
    if (nb >= 0 && A.nb(nx) != prv_slot(nb, B.m) && A.nb(nx) != nxt_slot(nb, B.m)) atomicMin(&f->firstMid[sd], v);
  }
}

// first midpoint-rule vertex of ring A against ring B through B's current links (B may
// hold its temporary vertex)
__global__ void big_first_mid_kernel(RingSet SA, RingSet SB, int64_t regA, int mA, int capA, int64_t regB, int mB,
                                     int capB, int usedB, int* out) {
  Ring A = big_ring(SA, regA, mA, capA, mA), B = big_ring(SB, regB, mB, capB, usedB);
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < A.m; v += gridDim.x * blockDim.x) {
    int nb = A.nb(v), nx = nxt_slot(v, A.m);
    if (nb >= 0 && A.nb(nx) != B.pv(nb) && A.nb(nx) != B.nx(nb)) atomicMin(out, v);
  }
}

// winding parity test (polygon.h:427-448) of a point of ring A against ring B.
// point: slot v of A (mode 0), midpoint of v and its successor (mode 1).
// B's edges are (s, s+1); `after`/`T` splice a temporary vertex of B.
__global__ void big_wind_kernel(RingSet SA, int64_t regA, int mA, int v, int mode, RingSet SB, int64_t regB, int mB,
                                int after, int T, unsigned long long* wsum) {
  const double2* a = &SA.xy(regA);
  double Rx = a[v].x, Ry = a[v].y;
  if (mode == 1) { int n = nxt_slot(v, mA); Rx = 0.5 * (a[v].x + a[n].x); Ry = 0.5 * (a[v].y + a[n].y); }
  const double2* q = &SB.xy(regB);
  long long w = 0;
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < mB; s += gridDim.x * blockDim.x) {
    int n = nxt_slot(s, mB);
    if (s == after) {
      w += wind(q[s].x, q[s].y, q[T].x, q[T].y, Rx, Ry, SB.exact);
      w += wind(q[T].x, q[T].y, q[n].x, q[n].y, Rx, Ry, SB.exact);
    } else {
      w += wind(q[s].x, q[s].y, q[n].x, q[n].y, Rx, Ry, SB.exact);
    }
  }
  w = warp_sum(w);
  if (lane_id() == 0 && w) atomicAdd(wsum, (unsigned long long)w);
}

__global__ void big_copy_ring_kernel(RingSet S, int64_t reg, int m, double* __restrict__ oxy, int64_t at,
                                     int32_t* __restrict__ csz, int comp) {
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < m; s += gridDim.x * blockDim.x) {
    oxy[2 * (at + s)] = S.x(reg + s);
    oxy[2 * (at + s) + 1] = S.y(reg + s);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) csz[comp] = m;
}

__global__ void big_add_temp_kernel(RingSet S, int64_t reg, int m, int cap, int used, int v) {
  Ring A = big_ring(S, reg, m, cap, used);
  int n = A.nx(v);
  int T = add_vertex(A, 0.5 * (A.x(v) + A.x(n)), 0.5 * (A.y(v) + A.y(n)));
  if (T >= 0) insert_after(A, T, v);
}

// step 4 as scans over the ring rotated to start after V0 (see warp_step4)
__global__ void big_d_kernel(RingSet S, int64_t reg, int m, int V0, int32_t* __restrict__ d) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < m; j += gridDim.x * blockDim.x) {
    int s = V0 + 1 + j;
    if (s >= m) s -= m;
    int8_t L = S.lb(reg + s);
    d[j] = (S.it(reg + s) && (L == L_DELAYED_CROSSING || L == L_DELAYED_BOUNCING)) ? 1 : 0;
  }
}

__global__ void big_t_kernel(RingSet S, int64_t reg, int m, int V0, const int64_t* __restrict__ dEx,
                             int32_t* __restrict__ t) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < m; j += gridDim.x * blockDim.x) {
    int s = V0 + 1 + j;
    if (s >= m) s -= m;
    int8_t L = S.lb(reg + s);
    bool first = (dEx[j] & 1) == 0;
    t[j] = (S.it(reg + s) && (L == L_CROSSING || L == L_DELAYED_BOUNCING || (L == L_DELAYED_CROSSING && !first))) ? 1 : 0;
  }
}

__global__ void big_apply4_kernel(RingSet S, int64_t reg, int m, int V0, const int64_t* __restrict__ dEx,
                                  const int64_t* __restrict__ tEx, int8_t st0, int uni) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < m; j += gridDim.x * blockDim.x) {
    int s = V0 + 1 + j;
    if (s >= m) s -= m;
    const int64_t g = reg + s;
    if (!S.it(g)) continue;
    int8_t L = S.lb(g);
    bool first = (dEx[j] & 1) == 0;
    int8_t st = (tEx[j] & 1) ? toggled(st0) : st0;
    if (L == L_CROSSING) S.ee(g) = st;
    else if (L == L_BOUNCING) { if ((st == E_EXIT) ^ (uni != 0)) S.fl(g) |= 1; }
    else if (L == L_DELAYED_CROSSING) {
      S.ee(g) = st;
      if (first) { if ((st == E_EXIT) ^ (uni != 0)) S.lb(g) = L_CROSSING; }
      else if ((st == E_ENTRY) ^ (uni != 0)) S.lb(g) = L_CROSSING;
    } else if (L == L_DELAYED_BOUNCING) {
      S.ee(g) = st;
      if (first) { if ((st == E_EXIT) ^ (uni != 0)) S.fl(g) |= 2; }
      else if ((st == E_ENTRY) ^ (uni != 0)) S.fl(g) |= 2;
    }
  }
}

__global__ void big_split_any_kernel(RingSet SP, RingSet SQ, BigPair bp, BigFlags* f) {
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < bp.mP; s += gridDim.x * blockDim.x) {
    if (!(SP.fl(bp.regP + s) & 1)) continue;
    int nb = SP.nb(bp.regP + s);
    if (nb >= 0 && (SQ.fl(bp.regQ + nb) & 1)) atomicOr(&f->anySplit, 1);
  }
}

__global__ void big_step6_kernel(RingSet SP, RingSet SQ, BigPair bp) {
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < bp.mP; s += gridDim.x * blockDim.x) {
    if (!(SP.fl(bp.regP + s) & 2)) continue;
    int nb = SP.nb(bp.regP + s);
    if (nb >= 0 && (SQ.fl(bp.regQ + nb) & 2)) { SP.lb(bp.regP + s) = L_CROSSING; SQ.lb(bp.regQ + nb) = L_CROSSING; }
  }
}

// the sequential phases from step 5 (split pairs) or from the trace on, one thread
template <int EX>
__global__ void big_seq_tail_kernel(RingSet SP, RingSet SQ, BigPair bp, int usedP, int usedQ, int from_trace,
                                    double* __restrict__ oxy, int32_t* __restrict__ ocsz, int64_t nv0, int nc0,
                                    ClipParams prm, int* err, int32_t* status, int32_t* outNC, int64_t* outNV) {
  PairCtx c;
  c.R[0] = big_ring(SP, bp.regP, bp.mP, bp.capP, usedP);
  c.R[1] = big_ring(SQ, bp.regQ, bp.mQ, bp.capQ, usedQ);
  c.O.xy = oxy + 2 * bp.vOff; c.O.csz = ocsz + bp.cOff; c.O.vcap = bp.vCap; c.O.ccap = bp.cCap;
  c.O.nv = nv0; c.O.nc = nc0; c.O.overflow = false;
  c.uni = prm.union_mode != 0;
  c.eps_clean = prm.eps_clean;
  c.err = err;
  c.status = status + bp.k;
  if (!from_trace) {
    if (!seq_step5<EX>(c)) return;
    seq_step6(c);
  }
  if (!seq_trace(c)) return;
  seq_cleanup(c, outNC + bp.k, outNV + bp.k);
}

// the whole pair sequentially from `step` (links not one-to-one, malformed chains)
template <int EX>
__global__ void big_seq_pair_kernel(RingSet SP, RingSet SQ, BigPair bp, int step, double* __restrict__ oxy,
                                    int32_t* __restrict__ ocsz, ClipParams prm, int* err, int32_t* status,
                                    int32_t* outNC, int64_t* outNV) {
  PairCtx c;
  c.R[0] = big_ring(SP, bp.regP, bp.mP, bp.capP, bp.mP);
  c.R[1] = big_ring(SQ, bp.regQ, bp.mQ, bp.capQ, bp.mQ);
  c.O.xy = oxy + 2 * bp.vOff; c.O.csz = ocsz + bp.cOff; c.O.vcap = bp.vCap; c.O.ccap = bp.cCap;
  c.O.nv = 0; c.O.nc = 0; c.O.overflow = false;
  c.uni = prm.union_mode != 0;
  c.eps_clean = prm.eps_clean;
  c.err = err;
  c.status = status + bp.k;
  c.noInter[0] = c.noInter[1] = c.ident[0] = c.ident[1] = false;
  seq_pair_from<EX>(c, step, outNC + bp.k, outNV + bp.k);
}

// ---- parallel tracing.  With no added vertices, when every vertex carrying an entry/exit
// flag is an unvisited CROSSING vertex and vice versa, flags alternate along each ring
// and linked vertices carry opposite flags, a run from a flagged vertex V ends at the
// next flagged vertex in its direction, W(V), and continues at the twin of W(V).  Runs
// from ENTRY vertices form cycles (one per result component); the reference traces each
// component from its smallest-slot flagged P vertex I, forwards if I starts a run of the
// cycle, else (I ends one) along the reversed cycle.
__global__ void big_labeled_kernel(RingSet S, int64_t reg, int m, uint8_t* __restrict__ lab, BigFlags* f) {
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < m; s += gridDim.x * blockDim.x) {
    int8_t e = S.ee(reg + s);
    bool flagged = (e == E_ENTRY || e == E_EXIT);
    bool crossing = S.it(reg + s) && S.lb(reg + s) == L_CROSSING;
    lab[s] = flagged ? 1 : 0;
    if (flagged != crossing) atomicOr(&f->bad, 1);
  }
}

__global__ void big_lab_list_kernel(const uint8_t* __restrict__ lab, const int64_t* __restrict__ idx, int m,
                                    int32_t* __restrict__ list) {
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < m; s += gridDim.x * blockDim.x)
    if (lab[s]) list[idx[s]] = s;
}

// per flagged vertex u (P: [0,nP), Q: [nP,nP+nQ)): checks, run stop, length, successor
__global__ void big_runs_kernel(RingSet SP, RingSet SQ, BigPair bp, const int32_t* __restrict__ listP,
                                const int32_t* __restrict__ listQ, const int64_t* __restrict__ idxP,
                                const int64_t* __restrict__ idxQ, int nP, int nQ, int uni, int32_t* __restrict__ succ,
                                int32_t* __restrict__ len, int32_t* __restrict__ stop, BigFlags* f) {
  for (int u = blockIdx.x * blockDim.x + threadIdx.x; u < nP + nQ; u += gridDim.x * blockDim.x) {
    const bool onP = u < nP;
    const RingSet& A = onP ? SP : SQ;
    const RingSet& B = onP ? SQ : SP;
    const int64_t ra = onP ? bp.regP : bp.regQ, rb = onP ? bp.regQ : bp.regP;
    const int m = onP ? bp.mP : bp.mQ;
    const int n = onP ? nP : nQ;
    const int i = onP ? u : u - nP;
    const int32_t* list = onP ? listP : listQ;
    const int s = list[i];
    const int8_t e = A.ee(ra + s);
    bool bad = n < 2;
    int nxt = list[(i + 1 < n) ? i + 1 : 0];
    if (A.ee(ra + nxt) == e) bad = true;                         // alternation
    int nb = A.nb(ra + s);
    if (nb < 0 || B.ee(rb + nb) != toggled(e)) bad = true;        // twin carries the opposite flag
    const int8_t st = toggled(e);
    const int dir = ((st == E_EXIT) ^ (uni != 0)) ? 1 : -1;
    int W = list[(i + dir + n) % n];
    int L = dir > 0 ? W - s : s - W;
    if (L <= 0) L += m;
    int nbW = A.nb(ra + W);
    if (nbW < 0) bad = true;
    int v = 0;
    if (!bad) v = onP ? nP + (int)idxQ[nbW] : (int)idxP[nbW];
    succ[u] = v;
    len[u] = L;
    stop[u] = W;
    if (bad) atomicOr(&f->bad, 1);
  }
}

// pointer jumping over ENTRY-start vertices: cycle minima of the P-start slots (a) and
// of the P-stop slots (b)
__global__ void big_cycle_min_kernel(const int32_t* __restrict__ J, const int32_t* __restrict__ a,
                                     const int32_t* __restrict__ b, int32_t* __restrict__ J2, int32_t* __restrict__ a2,
                                     int32_t* __restrict__ b2, const uint8_t* __restrict__ isE, int N) {
  for (int u = blockIdx.x * blockDim.x + threadIdx.x; u < N; u += gridDim.x * blockDim.x) {
    if (!isE[u]) continue;
    int j = J[u];
    a2[u] = min(a[u], a[j]);
    b2[u] = min(b[u], b[j]);
    J2[u] = J[j];
  }
}

__global__ void big_cycle_init_kernel(RingSet SP, RingSet SQ, BigPair bp, const int32_t* __restrict__ listP,
                                      const int32_t* __restrict__ listQ, int nP, int nQ, const int32_t* __restrict__ succ,
                                      const int32_t* __restrict__ stop, int32_t* __restrict__ J, int32_t* __restrict__ a,
                                      int32_t* __restrict__ b, uint8_t* __restrict__ isE) {
  for (int u = blockIdx.x * blockDim.x + threadIdx.x; u < nP + nQ; u += gridDim.x * blockDim.x) {
    const bool onP = u < nP;
    const int s = onP ? listP[u] : listQ[u - nP];
    const int8_t e = onP ? SP.ee(bp.regP + s) : SQ.ee(bp.regQ + s);
    isE[u] = e == E_ENTRY ? 1 : 0;
    J[u] = succ[u];
    a[u] = onP ? s : INT_MAX;
    b[u] = onP ? stop[u] : INT_MAX;
  }
}

// per ENTRY vertex: the cycle's list-ranking start B and direction; list break
__global__ void big_cycle_start_kernel(const int32_t* __restrict__ a, const int32_t* __restrict__ b,
                                       const uint8_t* __restrict__ isE, const int64_t* __restrict__ idxP,
                                       const int32_t* __restrict__ listP, int nP, int N, int dirE,
                                       const int32_t* __restrict__ succ, const int32_t* __restrict__ len,
                                       int32_t* __restrict__ Bst, uint8_t* __restrict__ rev, int32_t* __restrict__ nxt,
                                       int64_t* __restrict__ sfx) {
  for (int u = blockIdx.x * blockDim.x + threadIdx.x; u < N; u += gridDim.x * blockDim.x) {
    if (!isE[u]) continue;
    int B;
    if (a[u] < b[u]) {
      B = (int)idxP[a[u]];                       // I starts a run: forwards from I
      rev[u] = 0;
    } else {
      int iI = (int)idxP[b[u]];                  // I ends the run of A
      int iA = ((iI - dirE) % nP + nP) % nP;
      B = succ[iA];
      rev[u] = 1;
    }
    Bst[u] = B;
    nxt[u] = (succ[u] == B) ? -1 : succ[u];
    sfx[u] = len[u];
  }
}

__global__ void big_rank_kernel(const int32_t* __restrict__ nxt, const int64_t* __restrict__ sfx,
                                int32_t* __restrict__ nxt2, int64_t* __restrict__ sfx2, const uint8_t* __restrict__ isE,
                                int N) {
  for (int u = blockIdx.x * blockDim.x + threadIdx.x; u < N; u += gridDim.x * blockDim.x) {
    if (!isE[u]) continue;
    int j = nxt[u];
    if (j >= 0) { sfx2[u] = sfx[u] + sfx[j]; nxt2[u] = nxt[j]; }
    else { sfx2[u] = sfx[u]; nxt2[u] = -1; }
  }
}

// one writer per cycle: its length at the slot of I (components in ascending I)
__global__ void big_comp_len_kernel(const uint8_t* __restrict__ isE, const int32_t* __restrict__ Bst,
                                    const int64_t* __restrict__ sfx, const int32_t* __restrict__ a,
                                    const int32_t* __restrict__ b, int N, int64_t* __restrict__ compLen,
                                    uint8_t* __restrict__ compFlag) {
  for (int u = blockIdx.x * blockDim.x + threadIdx.x; u < N; u += gridDim.x * blockDim.x) {
    if (!isE[u] || Bst[u] != u) continue;
    int I = min(a[u], b[u]);
    compLen[I] = sfx[u];
    compFlag[I] = 1;
  }
}

// warp per run: copies the run's vertices to their places in the component
__global__ void big_write_kernel(RingSet SP, RingSet SQ, BigPair bp, const int32_t* __restrict__ listP,
                                 const int32_t* __restrict__ listQ, int nP, int N, const uint8_t* __restrict__ isE,
                                 const int32_t* __restrict__ len, const int32_t* __restrict__ Bst,
                                 const uint8_t* __restrict__ rev, const int64_t* __restrict__ sfx,
                                 const int32_t* __restrict__ a, const int32_t* __restrict__ b,
                                 const int64_t* __restrict__ compBase, const int64_t* __restrict__ compIdx,
                                 int64_t nv0, int nc0, int uni, double* __restrict__ oxy, int32_t* __restrict__ ocsz) {
  const int64_t w = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (w >= N || !isE[w]) return;
  const int u = (int)w;
  const bool onP = u < nP;
  const RingSet& A = onP ? SP : SQ;
  const int64_t ra = onP ? bp.regP : bp.regQ;
  const int m = onP ? bp.mP : bp.mQ;
  const int s = onP ? listP[u] : listQ[u - nP];
  const int8_t st = toggled(A.ee(ra + s));
  const int dir = ((st == E_EXIT) ^ (uni != 0)) ? 1 : -1;
  const int I = min(a[u], b[u]);
  const int64_t L = sfx[Bst[u]];
  const int64_t off = L - sfx[u];
  const int lu = len[u];
  const bool r = rev[u];
  const int64_t base = nv0 + compBase[I];
  for (int j = lane_id(); j < lu; j += 32) {
    int v = s + dir * (j + 1);
    v = ((v % m) + m) % m;
    int64_t f = off + j;
    int64_t pos = r ? ((f < L - 1) ? L - 2 - f : L - 1) : f;
    oxy[2 * (base + pos)] = A.x(ra + v);
    oxy[2 * (base + pos) + 1] = A.y(ra + v);
  }
  if (lane_id() == 0 && Bst[u] == u) ocsz[bp.cOff + nc0 + compIdx[I]] = (int32_t)L;
}

// warp per component of the pair: clean-up in place (see warp_cleanup)
__global__ void big_cleanup_kernel(double* __restrict__ xy, const int32_t* __restrict__ csz,
                                   const int64_t* __restrict__ cstart, int nc, double eps, int32_t* __restrict__ kept) {
  const int64_t w = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (w >= nc) return;
  const int n = csz[w];
  double* src = xy + 2 * cstart[w];
  bool flag = false;
  for (int j = lane_id(); j < n; j += 32) {
    int p = (j > 0) ? j - 1 : n - 1, q = (j + 1 < n) ? j + 1 : 0;
    if (fabs(area2(src[2 * p], src[2 * p + 1], src[2 * j], src[2 * j + 1], src[2 * q], src[2 * q + 1])) < eps)
      flag = true;
  }
  flag = __any_sync(kFull, flag);
  if (lane_id() == 0) kept[w] = flag ? seq_cleanup_component(src, src, n, eps) : n;
}

__global__ void big_compact_kernel(const double* __restrict__ xy, const int64_t* __restrict__ cstart,
                                   const int32_t* __restrict__ kept, const int64_t* __restrict__ kstart, int nc,
                                   double* __restrict__ tmp) {
  const int64_t w = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (w >= nc) return;
  const double* src = xy + 2 * cstart[w];
  double* dst = tmp + 2 * kstart[w];
  for (int i = lane_id(); i < 2 * kept[w]; i += 32) dst[i] = src[i];
}

__global__ void big_finish_kernel(const int32_t* __restrict__ kept, const int64_t* __restrict__ cidx, int nc,
                                  int32_t* __restrict__ csz) {
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += gridDim.x * blockDim.x)
    if (kept[c] > 0) csz[cidx[c]] = kept[c];
}

__global__ void big_info_label_kernel(const int64_t* __restrict__ list, int n, const int64_t* __restrict__ regP,
                                      const int64_t* __restrict__ regQ, const int32_t* __restrict__ mP,
                                      const int32_t* __restrict__ mQ, const int64_t* __restrict__ regSizeP,
                                      const int64_t* __restrict__ regSizeQ, const int64_t* __restrict__ vOff,
                                      const int64_t* __restrict__ vCap, const int64_t* __restrict__ cOff,
                                      const int32_t* __restrict__ cCap, BigPair* __restrict__ out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int64_t k = list[i];
  BigPair b;
  b.k = k; b.regP = regP[k]; b.regQ = regQ[k]; b.vOff = vOff[k]; b.vCap = vCap[k]; b.cOff = cOff[k];
  b.mP = mP[k]; b.mQ = mQ[k]; b.capP = (int32_t)regSizeP[k]; b.capQ = (int32_t)regSizeQ[k]; b.cCap = cCap[k];
  b.pad = 0;
  out[i] = b;
}

__global__ void big_label_list_kernel(const int32_t* __restrict__ mP, const int32_t* __restrict__ mQ,
                                      const int32_t* __restrict__ status, int64_t K, int64_t minSlots,
                                      int64_t* __restrict__ list, unsigned long long* __restrict__ n) {
  int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= K || status[k] != 0) return;
  if ((int64_t)mP[k] + mQ[k] > minSlots) list[atomicAdd(n, 1ull)] = k;
}

__global__ void big_kflag_kernel(const int32_t* __restrict__ kept, int nc, uint8_t* __restrict__ f) {
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += gridDim.x * blockDim.x) f[c] = kept[c] > 0;
}

__global__ void big_set_counts_kernel(int32_t* outNC, int64_t* outNV, int nc, int64_t nv) {
  *outNC = nc;
  *outNV = nv;
}

__global__ void big_fail_kernel(int32_t* status, int* err, int code) {
  *status = 3;
  raise_error(err, code);
}

// Host driver of the grid path for one huge pair.
struct BigCtx {
  Arena& A;
  cudaStream_t s;
  int64_t* hs;
  int* d_err;
  RingSet SP, SQ;
  double* oxy;
  int32_t* ocsz;
  int32_t* status;
  int32_t* outNC;
  int64_t* outNV;
  ClipParams prm;
};

static unsigned grid_for(int64_t n) {
  int64_t b = (n + 255) / 256;
  return (unsigned)std::max<int64_t>(1, std::min<int64_t>(b, 148 * 32));
}

static int run_big_label_pair(BigCtx& c, const BigPair& bp, BigFlags* df) {
  cudaStream_t s = c.s;
  const bool uni = c.prm.union_mode != 0;
  auto sync = [&]() { return cudaStreamSynchronize(s) == cudaSuccess; };
  BigFlags h{};
  h.firstFree[0] = h.firstMid[0] = bp.mP;
  h.firstFree[1] = h.firstMid[1] = bp.mQ;
  cudaMemcpyAsync(df, &h, sizeof(BigFlags), cudaMemcpyHostToDevice, s);
  auto read_flags = [&]() {
    cudaMemcpyAsync(&h, df, sizeof(BigFlags), cudaMemcpyDeviceToHost, s);
    return sync();
  };
  auto seq_pair = [&](int step) {
    { (c.prm.exact ? big_seq_pair_kernel<1> : big_seq_pair_kernel<0>)<<<1, 1, 0, s>>>(c.SP, c.SQ, bp, step, c.oxy, c.ocsz, c.prm, c.d_err, c.status, c.outNC,
                                         c.outNV); note_launch(); }
    return ST_OK;
  };
  const int64_t nAll = (int64_t)bp.mP + bp.mQ;
  // ---- links one-to-one?
  { big_links_kernel<<<grid_for(nAll), 256, 0, s>>>(c.SP, c.SQ, bp, df); note_launch(); }
  if (!read_flags()) return ST_CUDA_ERROR;
  if (h.bad) return seq_pair(1);
  // ---- step 1, chains
  { (c.prm.exact ? big_step1_kernel<1> : big_step1_kernel<0>)<<<grid_for(bp.mP), 256, 0, s>>>(c.SP, c.SQ, bp); note_launch(); }
  { big_chain_kernel<0><<<grid_for(bp.mP), 256, 0, s>>>(c.SP, c.SQ, bp, df); note_launch(); }
  if (!read_flags()) return ST_CUDA_ERROR;
  if (h.bad) return seq_pair(2);
  { big_chain_kernel<1><<<grid_for(bp.mP), 256, 0, s>>>(c.SP, c.SQ, bp, df); note_launch(); }
  // ---- special cases (3.5)
  { big_flags_kernel<<<grid_for(nAll), 256, 0, s>>>(c.SP, c.SQ, bp, uni ? 1 : 0, df); note_launch(); }
  if (!read_flags()) return ST_CUDA_ERROR;
  const int m[2] = {bp.mP, bp.mQ};
  const int64_t reg[2] = {bp.regP, bp.regQ};
  const int cap[2] = {bp.capP, bp.capQ};
  const RingSet* S[2] = {&c.SP, &c.SQ};
  bool noInter[2], ident[2];
  for (int sd = 0; sd < 2; ++sd) {
    noInter[sd] = !h.notNone[sd];
    ident[sd] = noInter[sd] && !h.notAllOn[sd];
  }
  int64_t nv = 0;
  int nc = 0;
  unsigned long long* dwind = &df->wind;
  auto winding = [&](int sa, int v, int mode, int sb, int after, int T, bool& inside) {
    cudaMemsetAsync(dwind, 0, sizeof(unsigned long long), s);
    { big_wind_kernel<<<grid_for(m[sb]), 256, 0, s>>>(*S[sa], reg[sa], m[sa], v, mode, *S[sb], reg[sb], m[sb], after, T,
                                                      dwind); note_launch(); }
    unsigned long long w = 0;
    cudaMemcpyAsync(&w, dwind, sizeof(w), cudaMemcpyDeviceToHost, s);
    if (!sync()) return false;
    inside = ((long long)w % 2) != 0;
    return true;
  };
  auto push_ring = [&](int sd) {
    if (nv + m[sd] > bp.vCap || nc >= bp.cCap) return false;
    { big_copy_ring_kernel<<<grid_for(m[sd]), 256, 0, s>>>(*S[sd], reg[sd], m[sd], c.oxy, bp.vOff + nv,
                                                           c.ocsz + bp.cOff, nc); note_launch(); }
    nv += m[sd];
    ++nc;
    return true;
  };
  auto fail = [&](int code) {
    { big_fail_kernel<<<1, 1, 0, s>>>(c.status + bp.k, c.d_err, code); note_launch(); }
    return ST_OK;
  };
  for (int sd = 0; sd < 2; ++sd) {
    if (!noInter[sd] || ident[sd]) continue;
    int v = -1, mode = 0;
    if (h.firstFree[sd] < m[sd]) v = h.firstFree[sd];
    else if (h.firstMid[sd] < m[sd]) { v = h.firstMid[sd]; mode = 1; }
    if (v < 0) continue;
    bool inside;
    if (!winding(sd, v, mode, 1 - sd, -1, -1, inside)) return ST_CUDA_ERROR;
    if (inside ^ uni)
      if (!push_ring(sd)) return fail(DEV_CAPACITY);
  }
  if (ident[0] && ident[1])
    if (!push_ring(0)) return fail(DEV_CAPACITY);
  // ---- step 4 (entry/exit) as device scans over the rotated rings
  int used[2] = {bp.mP, bp.mQ};
  int tempAfter[2] = {-1, -1}, tempSlot[2] = {-1, -1};
  {
    const int mm = std::max(bp.mP, bp.mQ);
    int32_t* d = c.A.take_n<int32_t>(mm);
    int32_t* t = c.A.take_n<int32_t>(mm);
    int64_t* dEx = c.A.take_n<int64_t>(mm);
    int64_t* tEx = c.A.take_n<int64_t>(mm);
    void* st = c.A.take(scan_temp_bytes(mm));
    if (!d || !t || !dEx || !tEx || !st) return ST_OUT_OF_MEMORY;
    for (int sd = 0; sd < 2; ++sd) {
      if (noInter[sd]) continue;
      int V0 = -1, qslot = -1;
      if (h.firstFree[sd] < m[sd]) {
        V0 = qslot = h.firstFree[sd];
      } else {
        int mid = h.firstMid[sd];
        if (sd == 1 && tempSlot[0] >= 0) {        // against P's links including P's temporary vertex
          int* dm = &df->firstMid[1];
          cudaMemcpyAsync(dm, &m[1], sizeof(int), cudaMemcpyHostToDevice, s);
          { big_first_mid_kernel<<<grid_for(m[1]), 256, 0, s>>>(c.SQ, c.SP, reg[1], m[1], cap[1], reg[0], m[0], cap[0],
                                                                used[0], dm); note_launch(); }
          if (!read_flags()) return ST_CUDA_ERROR;
          mid = h.firstMid[1];
        }
        if (mid >= m[sd]) continue;
        if (used[sd] >= cap[sd]) return fail(DEV_CAPACITY);
        { big_add_temp_kernel<<<1, 1, 0, s>>>(*S[sd], reg[sd], m[sd], cap[sd], used[sd], mid); note_launch(); }
        tempAfter[sd] = mid;
        tempSlot[sd] = used[sd]++;
        V0 = mid;
        qslot = tempSlot[sd];
      }
      bool inside;
      if (!winding(sd, qslot, 0, 1 - sd, sd == 1 ? tempAfter[0] : -1, sd == 1 ? tempSlot[0] : -1, inside))
        return ST_CUDA_ERROR;
      const int8_t st0 = inside ? E_EXIT : E_ENTRY;
      { big_d_kernel<<<grid_for(m[sd]), 256, 0, s>>>(*S[sd], reg[sd], m[sd], V0, d); note_launch(); }
      exclusive_scan_i32(d, dEx, m[sd], nullptr, st, c.d_err, s);
      { big_t_kernel<<<grid_for(m[sd]), 256, 0, s>>>(*S[sd], reg[sd], m[sd], V0, dEx, t); note_launch(); }
      exclusive_scan_i32(t, tEx, m[sd], nullptr, st, c.d_err, s);
      { big_apply4_kernel<<<grid_for(m[sd]), 256, 0, s>>>(*S[sd], reg[sd], m[sd], V0, dEx, tEx, st0, uni ? 1 : 0); note_launch(); }
    }
  }
  auto seq_tail = [&](int from_trace) {
    { (c.prm.exact ? big_seq_tail_kernel<1> : big_seq_tail_kernel<0>)<<<1, 1, 0, s>>>(c.SP, c.SQ, bp, used[0], used[1], from_trace, c.oxy, c.ocsz, nv, nc, c.prm,
                                          c.d_err, c.status, c.outNC, c.outNV); note_launch(); }
    return ST_OK;
  };
  // ---- split pairs (sequential), crossing candidates
  { big_split_any_kernel<<<grid_for(bp.mP), 256, 0, s>>>(c.SP, c.SQ, bp, df); note_launch(); }
  if (!read_flags()) return ST_CUDA_ERROR;
  if (h.anySplit) return seq_tail(0);
  { big_step6_kernel<<<grid_for(bp.mP), 256, 0, s>>>(c.SP, c.SQ, bp); note_launch(); }
  if (used[0] != bp.mP || used[1] != bp.mQ) return seq_tail(1);
  // ---- parallel tracing
  uint8_t* labP = c.A.take_n<uint8_t>(bp.mP);
  uint8_t* labQ = c.A.take_n<uint8_t>(bp.mQ);
  int64_t* idxP = c.A.take_n<int64_t>(bp.mP);
  int64_t* idxQ = c.A.take_n<int64_t>(bp.mQ);
  int64_t* tots = c.A.take_n<int64_t>(4);
  void* st = c.A.take(scan_temp_bytes(std::max(bp.mP, bp.mQ)));
  if (!labP || !labQ || !idxP || !idxQ || !tots || !st) return ST_OUT_OF_MEMORY;
  { big_labeled_kernel<<<grid_for(bp.mP), 256, 0, s>>>(c.SP, bp.regP, bp.mP, labP, df); note_launch(); }
  { big_labeled_kernel<<<grid_for(bp.mQ), 256, 0, s>>>(c.SQ, bp.regQ, bp.mQ, labQ, df); note_launch(); }
  exclusive_scan_u8(labP, idxP, bp.mP, tots + 0, st, c.d_err, s);
  exclusive_scan_u8(labQ, idxQ, bp.mQ, tots + 1, st, c.d_err, s);
  cudaMemcpyAsync(c.hs, tots, 2 * sizeof(int64_t), cudaMemcpyDeviceToHost, s);
  if (!read_flags()) return ST_CUDA_ERROR;
  if (h.bad) return seq_tail(1);
  const int nP = (int)c.hs[0], nQ = (int)c.hs[1], N = nP + nQ;
  int64_t TV = 0, TC = 0;
  if (N > 0) {
    int32_t* listP = c.A.take_n<int32_t>(nP);
    int32_t* listQ = c.A.take_n<int32_t>(nQ);
    int32_t* succ = c.A.take_n<int32_t>(N);
    int32_t* len = c.A.take_n<int32_t>(N);
    int32_t* stop = c.A.take_n<int32_t>(N);
    int32_t* J[2] = {c.A.take_n<int32_t>(N), c.A.take_n<int32_t>(N)};
    int32_t* a[2] = {c.A.take_n<int32_t>(N), c.A.take_n<int32_t>(N)};
    int32_t* b[2] = {c.A.take_n<int32_t>(N), c.A.take_n<int32_t>(N)};
    uint8_t* isE = c.A.take_n<uint8_t>(N);
    int32_t* Bst = c.A.take_n<int32_t>(N);
    uint8_t* rev = c.A.take_n<uint8_t>(N);
    int32_t* nx[2] = {c.A.take_n<int32_t>(N), c.A.take_n<int32_t>(N)};
    int64_t* sf[2] = {c.A.take_n<int64_t>(N), c.A.take_n<int64_t>(N)};
    int64_t* compLen = c.A.take_n<int64_t>(bp.mP);
    uint8_t* compFlag = c.A.take_n<uint8_t>(bp.mP);
    int64_t* compBase = c.A.take_n<int64_t>(bp.mP);
    int64_t* compIdx = c.A.take_n<int64_t>(bp.mP);
    if (!listP || !listQ || !succ || !len || !stop || !J[0] || !J[1] || !a[0] || !a[1] || !b[0] || !b[1] || !isE ||
        !Bst || !rev || !nx[0] || !nx[1] || !sf[0] || !sf[1] || !compLen || !compFlag || !compBase || !compIdx)
      return ST_OUT_OF_MEMORY;
    { big_lab_list_kernel<<<grid_for(bp.mP), 256, 0, s>>>(labP, idxP, bp.mP, listP); note_launch(); }
    { big_lab_list_kernel<<<grid_for(bp.mQ), 256, 0, s>>>(labQ, idxQ, bp.mQ, listQ); note_launch(); }
    { big_runs_kernel<<<grid_for(N), 256, 0, s>>>(c.SP, c.SQ, bp, listP, listQ, idxP, idxQ, nP, nQ, uni ? 1 : 0, succ,
                                                  len, stop, df); note_launch(); }
    if (!read_flags()) return ST_CUDA_ERROR;
    if (h.bad) return seq_tail(1);
    { big_cycle_init_kernel<<<grid_for(N), 256, 0, s>>>(c.SP, c.SQ, bp, listP, listQ, nP, nQ, succ, stop, J[0], a[0],
                                                        b[0], isE); note_launch(); }
    int rounds = 1;
    while ((1ll << rounds) < (int64_t)N) ++rounds;
    int cur = 0;
    for (int r = 0; r <= rounds; ++r) {
      { big_cycle_min_kernel<<<grid_for(N), 256, 0, s>>>(J[cur], a[cur], b[cur], J[1 - cur], a[1 - cur], b[1 - cur],
                                                         isE, N); note_launch(); }
      cur = 1 - cur;
    }
    const int dirE = uni ? -1 : 1;   // ENTRY vertices run forwards in intersection mode
    { big_cycle_start_kernel<<<grid_for(N), 256, 0, s>>>(a[cur], b[cur], isE, idxP, listP, nP, N, dirE, succ, len, Bst,
                                                         rev, nx[0], sf[0]); note_launch(); }
    int rc = 0;
    for (int r = 0; r <= rounds; ++r) {
      { big_rank_kernel<<<grid_for(N), 256, 0, s>>>(nx[rc], sf[rc], nx[1 - rc], sf[1 - rc], isE, N); note_launch(); }
      rc = 1 - rc;
    }
    cudaMemsetAsync(compLen, 0, bp.mP * sizeof(int64_t), s);
    cudaMemsetAsync(compFlag, 0, bp.mP, s);
    { big_comp_len_kernel<<<grid_for(N), 256, 0, s>>>(isE, Bst, sf[rc], a[cur], b[cur], N, compLen, compFlag); note_launch(); }
    exclusive_scan_i64(compLen, compBase, bp.mP, tots + 2, st, c.d_err, s);
    exclusive_scan_u8(compFlag, compIdx, bp.mP, tots + 3, st, c.d_err, s);
    cudaMemcpyAsync(c.hs, tots + 2, 2 * sizeof(int64_t), cudaMemcpyDeviceToHost, s);
    if (!sync()) return ST_CUDA_ERROR;
    TV = c.hs[0];
    TC = c.hs[1];
    if (nv + TV > bp.vCap || nc + TC > bp.cCap) return fail(DEV_CAPACITY);
    { big_write_kernel<<<(unsigned)(((int64_t)N * 32 + 255) / 256), 256, 0, s>>>(
        c.SP, c.SQ, bp, listP, listQ, nP, N, isE, len, Bst, rev, sf[rc], a[cur], b[cur], compBase, compIdx, nv, nc,
        uni ? 1 : 0, c.oxy + 2 * bp.vOff, c.ocsz); note_launch(); }
  }
  nv += TV;
  nc += (int)TC;
  // ---- clean-up of every component of the pair, then compaction
  if (nc == 0) {
    { big_set_counts_kernel<<<1, 1, 0, s>>>(c.outNC + bp.k, c.outNV + bp.k, 0, 0); note_launch(); }
    return ST_OK;
  }
  int32_t* csz = c.ocsz + bp.cOff;
  double* xy = c.oxy + 2 * bp.vOff;
  int64_t* cstart = c.A.take_n<int64_t>(nc);
  int32_t* kept = c.A.take_n<int32_t>(nc);
  int64_t* kstart = c.A.take_n<int64_t>(nc);
  uint8_t* kflag = c.A.take_n<uint8_t>(nc);
  int64_t* cidx = c.A.take_n<int64_t>(nc);
  double* tmp = c.A.take_n<double>(2 * nv);
  void* st3 = c.A.take(scan_temp_bytes(nc));
  if (!cstart || !kept || !kstart || !kflag || !cidx || !tmp || !st3) return ST_OUT_OF_MEMORY;
  exclusive_scan_i32(csz, cstart, nc, nullptr, st3, c.d_err, s);
  { big_cleanup_kernel<<<(unsigned)(((int64_t)nc * 32 + 255) / 256), 256, 0, s>>>(xy, csz, cstart, nc, c.prm.eps_clean,
                                                                                  kept); note_launch(); }
  exclusive_scan_i32(kept, kstart, nc, tots + 0, st3, c.d_err, s);
  { big_kflag_kernel<<<grid_for(nc), 256, 0, s>>>(kept, nc, kflag); note_launch(); }
  exclusive_scan_u8(kflag, cidx, nc, tots + 1, st3, c.d_err, s);
  { big_compact_kernel<<<(unsigned)(((int64_t)nc * 32 + 255) / 256), 256, 0, s>>>(xy, cstart, kept, kstart, nc, tmp); note_launch(); }
  cudaMemcpyAsync(c.hs, tots, 2 * sizeof(int64_t), cudaMemcpyDeviceToHost, s);
  if (!sync()) return ST_CUDA_ERROR;
  const int64_t KV = c.hs[0];
  const int KC = (int)c.hs[1];
  cudaMemcpyAsync(xy, tmp, 2 * KV * sizeof(double), cudaMemcpyDeviceToDevice, s);
  { big_finish_kernel<<<grid_for(nc), 256, 0, s>>>(kept, cidx, nc, csz); note_launch(); }
  { big_set_counts_kernel<<<1, 1, 0, s>>>(c.outNC + bp.k, c.outNV + bp.k, KC, KV); note_launch(); }
  return ST_OK;
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

__global__ void __launch_bounds__(kThreads, 8)   // 32 registers: compact 0.33 -> 0.20 ms
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
             cudaStream_t s, Marks* mk, cudaStream_t aux, RingExport* ex, cudaStream_t aux2,
             const double* mbrB, const double* mbrO, const JoinEdges* je) {
  Marks dummy;
  if (!mk) mk = &dummy;
  C = ClipDev();
  const JoinEdges jed = je ? *je : JoinEdges{};
  mk->mark("clip:start", s);
  C.n_pairs = K;
  if (K <= 0) return ST_OK;
  auto sync = [&]() { return cudaStreamSynchronize(s) == cudaSuccess; };
  // layer MBRs (same definition as the join's)
  const double* mb = mbrB;
  const double* mo = mbrO;
  if (!mb) {
    double* m = A.take_n<double>(4 * Lb.n);
    if (!m) return ST_OUT_OF_MEMORY;
    layer_mbrs(Lb, m, s);
    mb = m;
  }
  if (!mo) {
    double* m = A.take_n<double>(4 * Lo.n);
    if (!m) return ST_OUT_OF_MEMORY;
    layer_mbrs(Lo, m, s);
    mo = m;
  }
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
  // The narrow-tile and whole-warp passes of the edge filter take disjoint pairs (by size):
  // with an auxiliary stream the warp pass runs beside the tile pass.
  cudaEvent_t fev[2] = {nullptr, nullptr};
  const bool two = aux && cudaEventCreateWithFlags(&fev[0], cudaEventDisableTiming) == cudaSuccess &&
                   cudaEventCreateWithFlags(&fev[1], cudaEventDisableTiming) == cudaSuccess;
  struct EvGuard { cudaEvent_t* e; ~EvGuard() { for (int i = 0; i < 2; ++i) if (e[i]) cudaEventDestroy(e[i]); } } fguard{fev};
  cudaStream_t sw = two ? aux : s;
  auto fork_aux = [&]() { if (two) { cudaEventRecord(fev[0], s); cudaStreamWaitEvent(aux, fev[0], 0); } };
  auto join_aux = [&]() { if (two) { cudaEventRecord(fev[1], aux); cudaStreamWaitEvent(s, fev[1], 0); } };
  // ---- G1 edge filter
  fork_aux();
  { edge_filter_kernel<0, kFilterTile><<<(unsigned)((K * kFilterTile + kThreads - 1) / kThreads), kThreads, 0, s>>>(
        Lb, Lo, D, K, cP, cQ, nullptr, nullptr, nullptr, nullptr, -1, kFilterTileMax, jed); note_launch(); }
  { edge_filter_kernel<0, 32><<<blocks_for_warps(K), kThreads, 0, sw>>>(Lb, Lo, D, K, cP, cQ, nullptr, nullptr,
                                                                       nullptr, nullptr, kFilterTileMax,
                                                                       INT64_MAX, jed); note_launch(); }
  join_aux();
  exclusive_scan_i32(cP, offP, K, tot + 0, stK, d_err, s);
  exclusive_scan_i32(cQ, offQ, K, tot + 1, stK, d_err, s);
  exclusive_scan_i32(D.nP, eoffP, K, tot + 2, stK, d_err, s);
  exclusive_scan_i32(D.nQ, eoffQ, K, tot + 3, stK, d_err, s);
  int64_t* bigList = A.take_n<int64_t>(K);
  unsigned long long* nBig = A.take_n<unsigned long long>(1);
  if (!bigList || !nBig) return ST_OUT_OF_MEMORY;
  cudaMemsetAsync(nBig, 0, sizeof(unsigned long long), s);
  { chunk_count_kernel<<<blocks_for(K), kThreads, 0, s>>>(cP, cQ, K, nchunk, bigList, nBig, prm.bin_grid); note_launch(); }
  exclusive_scan_i64(nchunk, chunkOff, K, tot + 4, stK, d_err, s);
  mk->mark("clip:setup+filter", s);
  cudaMemcpyAsync(hs, tot, 5 * sizeof(int64_t), cudaMemcpyDeviceToHost, s);
  cudaMemcpyAsync(hs + 5, nBig, sizeof(int64_t), cudaMemcpyDeviceToHost, s);
  if (!sync()) return ST_CUDA_ERROR;
  const int64_t nLP = hs[0], nLQ = hs[1], nEP = hs[2], nEQ = hs[3], nCh = hs[4];
  const int nBigPairs = (int)hs[5];
  int32_t* LP = A.take_n<int32_t>(nLP);
  int32_t* LQ = A.take_n<int32_t>(nLQ);
  // Count + emit in one pass (intersect_fused_kernel) unless the records are exported:
  // the export keeps them in (pair, P edge, Q edge) order.
  const bool fused = prm.fused_emit && !ex;
  int32_t* chunkPair = A.take_n<int32_t>(nCh);
  int32_t* chunkRec = nullptr;
  int32_t* chunkQ = nullptr;
  int64_t* recScan = nullptr;
  int64_t* qScan = nullptr;
  void* stC = nullptr;
  int32_t* pairRec = nullptr;
  int32_t* pairQ = nullptr;
  if (fused) {
    pairRec = A.take_n<int32_t>(K);
    pairQ = A.take_n<int32_t>(K);
    if (!pairRec || !pairQ) return ST_OUT_OF_MEMORY;
  } else {
    chunkRec = A.take_n<int32_t>(nCh);
    chunkQ = A.take_n<int32_t>(nCh);
    recScan = A.take_n<int64_t>(nCh);
    qScan = A.take_n<int64_t>(nCh);
    stC = A.take(scan_temp_bytes(std::max<int64_t>(nCh, 1)));
    if (!chunkRec || !chunkQ || !recScan || !qScan || !stC) return ST_OUT_OF_MEMORY;
  }
  int64_t* binRec = A.take_n<int64_t>(K);
  int64_t* binQ = A.take_n<int64_t>(K);
  if (!LP || !LQ || !chunkPair || !binRec || !binQ) return ST_OUT_OF_MEMORY;
  if (nCh > 0) { chunk_pair_kernel<<<blocks_for_warps(K), kThreads, 0, s>>>(chunkOff, nchunk, K, chunkPair); note_launch(); }
  cudaMemsetAsync(binRec, 0, K * sizeof(int64_t), s);
  cudaMemsetAsync(binQ, 0, K * sizeof(int64_t), s);
  fork_aux();
  { edge_filter_kernel<1, kFilterTile><<<(unsigned)((K * kFilterTile + kThreads - 1) / kThreads), kThreads, 0, s>>>(
        Lb, Lo, D, K, cP, cQ, offP, offQ, LP, LQ, -1, kFilterTileMax, jed); note_launch(); }
  { edge_filter_kernel<1, 32><<<blocks_for_warps(K), kThreads, 0, sw>>>(Lb, Lo, D, K, cP, cQ, offP, offQ, LP, LQ,
                                                                       kFilterTileMax, INT64_MAX, jed); note_launch(); }
  join_aux();
  // The binned pairs (below) go to the auxiliary stream when there is one: fork here, before
  // the chunked count is queued on s, so that the two run side by side.
  cudaStream_t sb = s;
  cudaEvent_t bev[2] = {nullptr, nullptr};
  struct BinEvGuard { cudaEvent_t* e; ~BinEvGuard() { for (int i = 0; i < 2; ++i) if (e[i]) cudaEventDestroy(e[i]); } } bguard{bev};
  if (nBigPairs > 0 && aux && cudaEventCreateWithFlags(&bev[0], cudaEventDisableTiming) == cudaSuccess &&
      cudaEventCreateWithFlags(&bev[1], cudaEventDisableTiming) == cudaSuccess) {
    cudaEventRecord(bev[0], s);
    cudaStreamWaitEvent(aux, bev[0], 0);
    sb = aux;
  }
  // ---- G2 count: chunked pairs
  Records R{};
  unsigned long long* recTot = reinterpret_cast<unsigned long long*>(tot + 15);
  int64_t recCap = 0;
  auto take_records = [&](int64_t n) {
    n = std::max<int64_t>(n, 1);
    R.p = A.take_n<int32_t>(n); R.q = A.take_n<int32_t>(n);
    R.a = A.take_n<double>(n); R.b = A.take_n<double>(n);
    R.t = A.take_n<int8_t>(n); R.k = A.take_n<int32_t>(n);
    return R.p && R.q && R.a && R.b && R.t && R.k;
  };
  auto launch_fused = [&](bool countPairs) {
    if (nCh == 0) return;
    const FusedRecords F{recTot, recCap, countPairs ? pairRec : nullptr, pairQ};
    auto kern = prm.exact ? (prm.fused_emit == 2 ? intersect_fused_kernel<1, 1> : intersect_fused_kernel<1, 0>)
                          : (prm.fused_emit == 2 ? intersect_fused_kernel<0, 1> : intersect_fused_kernel<0, 0>);
    kern<<<blocks_for_warps(nCh), kThreads, 0, s>>>(Lb, Lo, D, chunkOff, nCh, cP, cQ, offP, offQ, LP, LQ, prm.eps, R,
                                                    chunkPair, F);
    note_launch();
  };
  if (fused) {
    // Capacity: the last clip's record count with room to spare, else a first guess,
    // never more than one record per chunked edge pair when nothing is binned.  A clip
    // that counts more records runs the pass again with arrays of the counted size.
    recCap = prm.rec_hint > 0 ? prm.rec_hint + prm.rec_hint / 4 + 4096 : kFirstRecordCap;
    if (nBigPairs == 0) recCap = std::min(recCap, std::max<int64_t>(nCh * kChunk, 1));
    if (!take_records(recCap)) return ST_OUT_OF_MEMORY;
    cudaMemsetAsync(recTot, 0, sizeof(unsigned long long), s);
    cudaMemsetAsync(pairRec, 0, K * sizeof(int32_t), s);
    cudaMemsetAsync(pairQ, 0, K * sizeof(int32_t), s);
    launch_fused(true);
    if (sb != s) cudaEventRecord(bev[0], s);        // the binned records go after the chunked ones
  } else if (nCh > 0) {
    { (prm.exact ? intersect_kernel<0, 1> : intersect_kernel<0, 0>)<<<blocks_for_warps(nCh), kThreads, 0, s>>>(
        Lb, Lo, D, K, chunkOff, nCh, cP, cQ, offP, offQ, LP, LQ, prm.eps, chunkRec, chunkQ, nullptr, nullptr, R, chunkPair); note_launch(); }
    exclusive_scan_i32(chunkRec, recScan, nCh, nullptr, stC, d_err, s);
    exclusive_scan_i32(chunkQ, qScan, nCh, nullptr, stC, d_err, s);
  }
  // ---- G2 count: binned pairs, all in the same launches.  With an auxiliary stream they
  // run there, beside the chunked count; s waits for them before the per-pair totals.
  auto syncb = [&]() { return cudaStreamSynchronize(sb) == cudaSuccess; };
  BinSet BS{};
  int64_t nBinP = 0, nBinQ = 0;
  int64_t* cellOff = nullptr;
  int32_t* cellList = nullptr;
  int64_t* binRecPos = nullptr;
  if (nBigPairs > 0) {
    const int B = nBigPairs;
    BS.list = bigList;
    BS.cp = A.take_n<int32_t>(B); BS.cq = A.take_n<int32_t>(B);
    BS.pBase = A.take_n<int64_t>(B); BS.qBase = A.take_n<int64_t>(B);
    BS.ext = A.take_n<double>(2 * B); BS.grid = A.take_n<BinGrid>(B);
    BS.cellBase = A.take_n<int64_t>(B); BS.ncell = A.take_n<int32_t>(B);
    int64_t* d_t = A.take_n<int64_t>(4);
    void* stB = A.take(scan_temp_bytes(B));
    if (!BS.cp || !BS.cq || !BS.pBase || !BS.qBase || !BS.ext || !BS.grid || !BS.cellBase || !BS.ncell || !d_t ||
        !stB)
      return ST_OUT_OF_MEMORY;
    { bin_sizes_kernel<<<blocks_for(B), kThreads, 0, sb>>>(BS, B, cP, cQ); note_launch(); }
    exclusive_scan_i32(BS.cp, BS.pBase, B, d_t + 0, stB, d_err, sb);
    exclusive_scan_i32(BS.cq, BS.qBase, B, d_t + 1, stB, d_err, sb);
    cudaMemsetAsync(BS.ext, 0, 2 * (size_t)B * sizeof(double), sb);
    cudaMemcpyAsync(hs + 40, d_t, 2 * sizeof(int64_t), cudaMemcpyDeviceToHost, sb);
    if (!syncb()) return ST_CUDA_ERROR;
    nBinP = hs[40];
    nBinQ = hs[41];
    BS.ownP = A.take_n<int32_t>(nBinP);
    BS.ownQ = A.take_n<int32_t>(nBinQ);
    if (!BS.ownP || !BS.ownQ) return ST_OUT_OF_MEMORY;
    { range_owner_kernel<<<blocks_for_warps(B), kThreads, 0, sb>>>(BS.pBase, BS.cp, B, BS.ownP); note_launch(); }
    { range_owner_kernel<<<blocks_for_warps(B), kThreads, 0, sb>>>(BS.qBase, BS.cq, B, BS.ownQ); note_launch(); }
    if (nBinQ > 0)
      { bin_extent_kernel<<<blocks_for(nBinQ), kThreads, 0, sb>>>(Lb, Lo, D, BS, nBinQ, offQ, LQ); note_launch(); }
    { bin_grid_kernel<<<blocks_for(B), kThreads, 0, sb>>>(D, BS, B); note_launch(); }
    exclusive_scan_i32(BS.ncell, BS.cellBase, B, d_t + 2, stB, d_err, sb);
    cudaMemcpyAsync(hs + 42, d_t + 2, sizeof(int64_t), cudaMemcpyDeviceToHost, sb);
    if (!syncb()) return ST_CUDA_ERROR;
    const int64_t nCells = hs[42];
    int32_t* cellCnt = A.take_n<int32_t>(nCells + 1);
    cellOff = A.take_n<int64_t>(nCells + 1);
    int32_t* cursor = A.take_n<int32_t>(nCells);
    void* stCell = A.take(scan_temp_bytes(nCells + 1));
    if (!cellCnt || !cellOff || !cursor || !stCell) return ST_OUT_OF_MEMORY;
    cudaMemsetAsync(cellCnt, 0, (nCells + 1) * sizeof(int32_t), sb);
    cudaMemsetAsync(cursor, 0, nCells * sizeof(int32_t), sb);
    if (nBinQ > 0)
      { bin_cells_kernel<0><<<blocks_for(nBinQ), kThreads, 0, sb>>>(Lb, Lo, D, BS, nBinQ, offQ, LQ, cellCnt, nullptr,
                                                                   nullptr, nullptr); note_launch(); }
    exclusive_scan_i32(cellCnt, cellOff, nCells + 1, d_t + 3, stCell, d_err, sb);
    cudaMemcpyAsync(hs + 43, d_t + 3, sizeof(int64_t), cudaMemcpyDeviceToHost, sb);
    if (!syncb()) return ST_CUDA_ERROR;
    cellList = A.take_n<int32_t>(hs[43]);
    int32_t* binRecCnt = A.take_n<int32_t>(nBinP + 1);
    binRecPos = A.take_n<int64_t>(nBinP + 1);
    void* stP = A.take(scan_temp_bytes(nBinP + 1));
    if (!cellList || !binRecCnt || !binRecPos || !stP) return ST_OUT_OF_MEMORY;
    if (nBinQ > 0)
      { bin_cells_kernel<1><<<blocks_for(nBinQ), kThreads, 0, sb>>>(Lb, Lo, D, BS, nBinQ, offQ, LQ, nullptr, cellOff,
                                                                   cursor, cellList); note_launch(); }
    cudaMemsetAsync(binRecCnt + nBinP, 0, sizeof(int32_t), sb);     // so the scan's last entry is the total
    if (nBinP > 0)
      { (prm.exact ? bin_pairs_kernel<0, 1> : bin_pairs_kernel<0, 0>)<<<blocks_for(nBinP), kThreads, 0, sb>>>(
            Lb, Lo, D, BS, nBinP, offP, LP, cellOff, cellList, prm.eps, binRecCnt, binQ, nullptr, nullptr, R, nullptr,
            INT64_MAX); note_launch(); }
    exclusive_scan_i32(binRecCnt, binRecPos, nBinP + 1, nullptr, stP, d_err, sb);
    { bin_rec_total_kernel<<<blocks_for(B), kThreads, 0, sb>>>(BS, B, binRecPos, binRec); note_launch(); }
    if (fused && nBinP > 0) {                       // emit now, after the chunked records
      if (sb != s) cudaStreamWaitEvent(sb, bev[0], 0);
      { (prm.exact ? bin_pairs_kernel<1, 1> : bin_pairs_kernel<1, 0>)<<<blocks_for(nBinP), kThreads, 0, sb>>>(
            Lb, Lo, D, BS, nBinP, offP, LP, cellOff, cellList, prm.eps, nullptr, nullptr, binRecPos, nullptr, R,
            recTot, recCap); note_launch(); }
    }
  }
  if (sb != s) {
    cudaEventRecord(bev[1], sb);
    cudaStreamWaitEvent(s, bev[1], 0);
  }
  int64_t* nrec64 = A.take_n<int64_t>(K);
  int64_t* recOff = A.take_n<int64_t>(K);
  int32_t* nrec = A.take_n<int32_t>(K);
  if (!nrec64 || !recOff || !nrec) return ST_OUT_OF_MEMORY;
  { pair_records_kernel<<<blocks_for(K), kThreads, 0, s>>>(chunkOff, nchunk, recScan, qScan, chunkRec, chunkQ,
                                                         binRec, binQ, K, nrec64, nrec, C.count1, D,
                                                         pairRec, pairQ); note_launch(); }
  int64_t nR = 0;
  if (fused) {
    mk->mark("clip:count+emit", s);
    cudaMemcpyAsync(hs, recTot, sizeof(int64_t), cudaMemcpyDeviceToHost, s);
    if (nBinP > 0) cudaMemcpyAsync(hs + 1, binRecPos + nBinP, sizeof(int64_t), cudaMemcpyDeviceToHost, s);
    if (!sync()) return ST_CUDA_ERROR;
    nR = hs[0] + (nBinP > 0 ? hs[1] : 0);
    if (nR >= (1ll << kLinkKeyShift)) return ST_OUT_OF_MEMORY;
    if (nR > recCap) {                              // the arrays were short: again, at the counted size
      recCap = nR;
      if (!take_records(recCap)) return ST_OUT_OF_MEMORY;
      cudaMemsetAsync(recTot, 0, sizeof(unsigned long long), s);
      launch_fused(false);
      if (nBinP > 0)
        { (prm.exact ? bin_pairs_kernel<1, 1> : bin_pairs_kernel<1, 0>)<<<blocks_for(nBinP), kThreads, 0, s>>>(
              Lb, Lo, D, BS, nBinP, offP, LP, cellOff, cellList, prm.eps, nullptr, nullptr, binRecPos, nullptr, R,
              recTot, recCap); note_launch(); }
    }
  } else {
    exclusive_scan_i64(nrec64, recOff, K, tot + 5, stK, d_err, s);
    mk->mark("clip:count", s);
    cudaMemcpyAsync(hs, tot + 5, sizeof(int64_t), cudaMemcpyDeviceToHost, s);
    if (!sync()) return ST_CUDA_ERROR;
    nR = hs[0];
    if (nR >= (1ll << kLinkKeyShift)) return ST_OUT_OF_MEMORY;
    // ---- G3 emit
    if (!take_records(nR)) return ST_OUT_OF_MEMORY;
    if (sb != s && nBigPairs > 0) {                 // the binned pairs' emit beside the chunked one
      cudaEventRecord(bev[0], s);
      cudaStreamWaitEvent(sb, bev[0], 0);
    }
    if (nCh > 0)
      { (prm.exact ? intersect_kernel<1, 1> : intersect_kernel<1, 0>)<<<blocks_for_warps(nCh), kThreads, 0, s>>>(
          Lb, Lo, D, K, chunkOff, nCh, cP, cQ, offP, offQ, LP, LQ, prm.eps, nullptr, nullptr, recScan, recOff, R,
          chunkPair); note_launch(); }
    if (nBinP > 0)
      { (prm.exact ? bin_pairs_kernel<1, 1> : bin_pairs_kernel<1, 0>)<<<blocks_for(nBinP), kThreads, 0, sb>>>(
          Lb, Lo, D, BS, nBinP, offP, LP, cellOff, cellList, prm.eps, nullptr, nullptr, binRecPos, recOff, R, nullptr,
          INT64_MAX);
        note_launch(); }
    if (sb != s && nBigPairs > 0) {
      cudaEventRecord(bev[1], sb);
      cudaStreamWaitEvent(s, bev[1], 0);
    }
    mk->mark("clip:emit", s);
  }
  if (ex && ex->records_only) {
    ex->n_records = nR;
    ex->rec_p = R.p; ex->rec_q = R.q; ex->rec_a = R.a; ex->rec_b = R.b; ex->rec_t = R.t; ex->rec_k = R.k;
    C.n_records = nR;
    return ST_OK;
  }
  // ---- G4 ring layout
  int32_t* insP = A.take_n<int32_t>(nEP);
  int32_t* insQ = A.take_n<int32_t>(nEQ);
  int64_t* srcLinkP = A.take_n<int64_t>(nEP);
  int64_t* srcLinkQ = A.take_n<int64_t>(nEQ);
  int64_t* vposP = A.take_n<int64_t>(nEP);
  int64_t* vposQ = A.take_n<int64_t>(nEQ);
  int64_t* insBaseP = A.take_n<int64_t>(nEP);
  int64_t* insBaseQ = A.take_n<int64_t>(nEQ);
  int32_t* curP = A.take_n<int32_t>(nEP);
  int32_t* curQ = A.take_n<int32_t>(nEQ);
  int64_t* slotP = A.take_n<int64_t>(nR);
  int64_t* slotQ = A.take_n<int64_t>(nR);
  void* stE = A.take(scan_temp_bytes(std::max<int64_t>(std::max(nEP, nEQ), 1)));
  if (!insP || !insQ || !srcLinkP || !srcLinkQ || !vposP || !vposQ || !insBaseP ||
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
  exclusive_scan_i32(insP, insBaseP, nEP, tot + 9, stE, d_err, s);
  exclusive_scan_i32(insQ, insBaseQ, nEQ, tot + 10, stE, d_err, s);
  { edge_slots_kernel<<<blocks_for(nEP), kThreads, 0, s>>>(insBaseP, nEP, vposP); note_launch(); }
  { edge_slots_kernel<<<blocks_for(nEQ), kThreads, 0, s>>>(insBaseQ, nEQ, vposQ); note_launch(); }
  // Sizes: the record export reads the exact ones back; the clip takes bounds instead
  // and saves the two host round trips (a record inserts at most one vertex per side).
  const bool exactSizes = ex != nullptr;
  int64_t nInsP = nR, nInsQ = nR;
  if (exactSizes) {
    cudaMemcpyAsync(hs + 2, tot + 9, 2 * sizeof(int64_t), cudaMemcpyDeviceToHost, s);
    if (!sync()) return ST_CUDA_ERROR;
    nInsP = hs[2];
    nInsQ = hs[3];
  }
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
  unsigned long long* ringTot = reinterpret_cast<unsigned long long*>(tot + 6);
  cudaMemsetAsync(ringTot, 0, sizeof(unsigned long long), s);
  { pair_ring_kernel<<<blocks_for(K), kThreads, 0, s>>>(eoffP, vposP, D.nP, nrec, D.status, K, nEP, tot + 9, mP,
                                                      regSizeP, ringTot); note_launch(); }
  { pair_ring_kernel<<<blocks_for(K), kThreads, 0, s>>>(eoffQ, vposQ, D.nQ, nrec, D.status, K, nEQ, tot + 10, mQ,
                                                      regSizeQ, ringTot); note_launch(); }
  // The one-thread and warp labelling kernels take their pairs in size order (largest
  // first, label_order_kernel), and the ring regions are laid out in that order, so that
  // the pairs labelled side by side have neighbouring regions.  The record export keeps
  // the regions in pair order.
  const int64_t midMin = std::min(prm.mid_label_min, prm.big_label_min);
  unsigned long long* mcnt = A.take_n<unsigned long long>(4);
  uint32_t* oval = A.take_n<uint32_t>(K);
  if (!mcnt || !oval) return ST_OUT_OF_MEMORY;
  cudaMemsetAsync(mcnt, 0, 4 * sizeof(unsigned long long), s);
  if (!ex) {
    uint64_t* okey = A.take_n<uint64_t>(K);
    uint64_t* okeyAlt = A.take_n<uint64_t>(K);
    uint32_t* ovalAlt = A.take_n<uint32_t>(K);
    void* otmp = A.take(radix_temp_bytes(K));
    int64_t* sortedP = A.take_n<int64_t>(K);
    int64_t* sortedQ = A.take_n<int64_t>(K);
    int64_t* offSP = A.take_n<int64_t>(K);
    int64_t* offSQ = A.take_n<int64_t>(K);
    if (!okey || !okeyAlt || !ovalAlt || !otmp || !sortedP || !sortedQ || !offSP || !offSQ) return ST_OUT_OF_MEMORY;
    { label_order_kernel<<<blocks_for(K), kThreads, 0, s>>>(mP, mQ, D.status, K, std::max<int64_t>(prm.tile_label_max, 0),
                                                           midMin, prm.big_label_min, okey, oval, mcnt); note_launch(); }
    radix_sort_pairs(okey, oval, okeyAlt, ovalAlt, K, 8, otmp, d_err, s);
    { permute_sizes_kernel<<<blocks_for(K), kThreads, 0, s>>>(oval, K, regSizeP, regSizeQ, sortedP, sortedQ); note_launch(); }
    exclusive_scan_i64(sortedP, offSP, K, tot + 11, stK, d_err, s);
    exclusive_scan_i64(sortedQ, offSQ, K, tot + 12, stK, d_err, s);
    { unpermute_offsets_kernel<<<blocks_for(K), kThreads, 0, s>>>(oval, K, offSP, offSQ, regP, regQ); note_launch(); }
  } else {
    exclusive_scan_i64(regSizeP, regP, K, tot + 11, stK, d_err, s);
    exclusive_scan_i64(regSizeQ, regQ, K, tot + 12, stK, d_err, s);
  }
  // region slots: merged rings (edges + insertions) + 2 + 2 records per valid pair
  int64_t regTotP = nEP + nInsP + 2 * K + 2 * nR, regTotQ = nEQ + nInsQ + 2 * K + 2 * nR;
  if (exactSizes) {
    cudaMemcpyAsync(hs, tot + 11, 2 * sizeof(int64_t), cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(hs + 2, tot + 6, sizeof(int64_t), cudaMemcpyDeviceToHost, s);
    if (!sync()) return ST_CUDA_ERROR;
    regTotP = hs[0];
    regTotQ = hs[1];
    C.n_ring_vertices = hs[2];
  }
  C.n_records = nR;
  auto take_ring = [&](int64_t n, RingSet& S) {
    const int64_t slots = (std::max<int64_t>(n, 1) + 15) & ~int64_t(15);
    char* buf = static_cast<char*>(A.take((size_t)(kRingSlotBytes * slots)));
    S.set(buf, slots);
    return buf != nullptr;
  };
  RingSet SP, SQ;
  if (!take_ring(regTotP, SP) || !take_ring(regTotQ, SQ)) return ST_OUT_OF_MEMORY;
  SP.exact = SQ.exact = prm.exact;
  mk->mark("clip:layout", s);
  // ---- G5 ring fill (light edges per thread, heavy edges per block).  The P and Q rings
  // are independent, and each side's latency-bound fill leaves room on the GPU for the
  // other, so the Q side runs on the auxiliary stream when there is one.
  {
    const size_t smem = (size_t)kHeavySmem * (sizeof(uint64_t) + 2 * sizeof(uint32_t));
    cudaFuncSetAttribute(heavy_fill_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaFuncSetAttribute(heavy_fill_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    unsigned long long* nHeavy = A.take_n<unsigned long long>(2);
    if (!nHeavy) return ST_OUT_OF_MEMORY;
    cudaMemsetAsync(nHeavy, 0, 2 * sizeof(unsigned long long), s);
    cudaStream_t sq = s;
    cudaEvent_t fork = nullptr, join = nullptr;
    if (aux && cudaEventCreateWithFlags(&fork, cudaEventDisableTiming) == cudaSuccess &&
        cudaEventCreateWithFlags(&join, cudaEventDisableTiming) == cudaSuccess) {
      cudaEventRecord(fork, s);
      cudaStreamWaitEvent(aux, fork, 0);
      sq = aux;
    }
    int st = ST_OK;
    for (int side = 0; side < 2 && st == ST_OK; ++side) {
      cudaStream_t ss = side == 0 ? s : sq;
      const int64_t nE = side == 0 ? nEP : nEQ, nIns = side == 0 ? nInsP : nInsQ;
      int64_t* heavy = A.take_n<int64_t>(nE);
      uint64_t* gkey = A.take_n<uint64_t>(2 * nIns);
      uint32_t* gtie = A.take_n<uint32_t>(2 * nIns);
      uint32_t* gidx = A.take_n<uint32_t>(2 * nIns);
      int32_t* edgePair = A.take_n<int32_t>(nE);                    // edge -> pair
      if (!heavy || !gkey || !gtie || !gidx || !edgePair) { st = ST_OUT_OF_MEMORY; break; }
      if (nE == 0) continue;
      if (side == 0) {
        { range_owner_kernel<<<blocks_for_warps(K), kThreads, 0, ss>>>(eoffP, D.nP, K, edgePair); note_launch(); }
        { ring_fill_kernel<0><<<blocks_for(nEP), kThreads, 0, ss>>>(Lb, Lo, D, R, eoffP, nEP, edgePair, vposP, regP, mP,
                                                                  SP, slotP, insBaseP, curP, insListP, heavy,
                                                                  nHeavy); note_launch(); }
        { heavy_fill_kernel<0><<<2 * nsm, kHeavyThreads, smem, ss>>>(Lb, Lo, D, R, eoffP, edgePair, vposP, regP, mP, SP,
                                                                     slotP, insBaseP, curP, insListP, heavy, nHeavy,
                                                                     gkey, gtie, gidx); note_launch(); }
      } else {
        { range_owner_kernel<<<blocks_for_warps(K), kThreads, 0, ss>>>(eoffQ, D.nQ, K, edgePair); note_launch(); }
        { ring_fill_kernel<1><<<blocks_for(nEQ), kThreads, 0, ss>>>(Lb, Lo, D, R, eoffQ, nEQ, edgePair, vposQ, regQ, mQ,
                                                                  SQ, slotQ, insBaseQ, curQ, insListQ, heavy,
                                                                  nHeavy + 1); note_launch(); }
        { heavy_fill_kernel<1><<<2 * nsm, kHeavyThreads, smem, ss>>>(Lb, Lo, D, R, eoffQ, edgePair, vposQ, regQ, mQ, SQ,
                                                                     slotQ, insBaseQ, curQ, insListQ, heavy, nHeavy + 1,
                                                                     gkey, gtie, gidx); note_launch(); }
      }
    }
    if (sq != s) {
      cudaEventRecord(join, sq);
      cudaStreamWaitEvent(s, join, 0);
    }
    if (fork) cudaEventDestroy(fork);
    if (join) cudaEventDestroy(join);
    if (st != ST_OK) return st;
  }
  // ---- G6 links
  if (nR > 0)
    { link_kernel<<<blocks_for(nR), kThreads, 0, s>>>(R, nR, D.status, eoffP, eoffQ, vposP, vposQ, regP, regQ,
                                                    slotP, slotQ, srcLinkP, srcLinkQ, SP, SQ); note_launch(); }
  // ---- export of the merged rings instead of labelling (calculateIntersections)
  if (ex) {
    unsigned long long* keyP = A.take_n<unsigned long long>(std::max<int64_t>(regTotP, 1));
    unsigned long long* keyQ = A.take_n<unsigned long long>(std::max<int64_t>(regTotQ, 1));
    int32_t* cnt = A.take_n<int32_t>(2 * K);
    double* xyP = A.take_n<double>(2 * std::max<int64_t>(regTotP, 1));
    double* xyQ = A.take_n<double>(2 * std::max<int64_t>(regTotQ, 1));
    int32_t* iP = A.take_n<int32_t>(3 * std::max<int64_t>(regTotP, 1));
    int32_t* iQ = A.take_n<int32_t>(3 * std::max<int64_t>(regTotQ, 1));
    if (!keyP || !keyQ || !cnt || !xyP || !xyQ || !iP || !iQ) return ST_OUT_OF_MEMORY;
    cudaMemsetAsync(keyP, 0, std::max<int64_t>(regTotP, 1) * sizeof(unsigned long long), s);
    cudaMemsetAsync(keyQ, 0, std::max<int64_t>(regTotQ, 1) * sizeof(unsigned long long), s);
    cudaMemsetAsync(cnt, 0, 2 * K * sizeof(int32_t), s);
    if (nR > 0)
      { export_key_kernel<<<blocks_for(nR), kThreads, 0, s>>>(R, nR, D.status, eoffP, eoffQ, vposP, vposQ, regP,
                                                              regQ, slotP, slotQ, keyP, keyQ, cnt, cnt + K); note_launch(); }
    const int64_t rP = std::max<int64_t>(regTotP, 1), rQ = std::max<int64_t>(regTotQ, 1);
    { export_ring_kernel<<<(unsigned)K, kThreads, 0, s>>>(K, D.status, mP, mQ, regP, regQ, SP, SQ, keyP, keyQ, xyP,
                                                         xyQ, iP, iQ, iP + rP, iQ + rQ, iP + 2 * rP,
                                                         iQ + 2 * rQ); note_launch(); }
    // pair 0: status, record counts per ring, edges, merged sizes, region offsets
    int32_t h32[6];
    int64_t h64[2];
    cudaMemcpyAsync(h32 + 0, D.status, sizeof(int32_t), cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(h32 + 1, cnt, sizeof(int32_t), cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(h32 + 2, cnt + K, sizeof(int32_t), cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(h32 + 3, D.nP, sizeof(int32_t), cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(h32 + 4, D.nQ, sizeof(int32_t), cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(h32 + 5, mP, sizeof(int32_t), cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(h64 + 0, regP, sizeof(int64_t), cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(h64 + 1, regQ, sizeof(int64_t), cudaMemcpyDeviceToHost, s);
    if (!sync()) return ST_CUDA_ERROR;
    ex->status = h32[0];
    ex->edges_p = h32[3];
    ex->edges_q = h32[4];
    ex->n_p = (int64_t)h32[3] + h32[1];
    ex->n_q = (int64_t)h32[4] + h32[2];
    if (ex->status == 0) {
      if (h32[5] != ex->n_p) return ST_DEVICE_ERROR;   // the ring layout disagrees with the records
      const int64_t np = ex->n_p, nq = ex->n_q, oP = h64[0], oQ = h64[1];
      ex->xy_p.resize(2 * np); ex->xy_q.resize(2 * nq);
      ex->alpha_p.resize(np); ex->label_p.resize(np); ex->nb_p.resize(np);
      ex->alpha_q.resize(nq); ex->label_q.resize(nq); ex->nb_q.resize(nq);
      cudaMemcpyAsync(ex->xy_p.data(), xyP + 2 * oP, 2 * np * sizeof(double), cudaMemcpyDeviceToHost, s);
      cudaMemcpyAsync(ex->xy_q.data(), xyQ + 2 * oQ, 2 * nq * sizeof(double), cudaMemcpyDeviceToHost, s);
      cudaMemcpyAsync(ex->alpha_p.data(), iP + oP, np * sizeof(int32_t), cudaMemcpyDeviceToHost, s);
      cudaMemcpyAsync(ex->label_p.data(), iP + rP + oP, np * sizeof(int32_t), cudaMemcpyDeviceToHost, s);
      cudaMemcpyAsync(ex->nb_p.data(), iP + 2 * rP + oP, np * sizeof(int32_t), cudaMemcpyDeviceToHost, s);
      cudaMemcpyAsync(ex->alpha_q.data(), iQ + oQ, nq * sizeof(int32_t), cudaMemcpyDeviceToHost, s);
      cudaMemcpyAsync(ex->label_q.data(), iQ + rQ + oQ, nq * sizeof(int32_t), cudaMemcpyDeviceToHost, s);
      cudaMemcpyAsync(ex->nb_q.data(), iQ + 2 * rQ + oQ, nq * sizeof(int32_t), cudaMemcpyDeviceToHost, s);
      if (!sync()) return ST_CUDA_ERROR;
    }
    return ST_OK;
  }
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
  // the pairs of the one-thread, warp and block kernels, in order, and their counts came
  // with the ring layout; the counts are read with the output sizes
  cudaMemcpyAsync(hs, tot + 13, 2 * sizeof(int64_t), cudaMemcpyDeviceToHost, s);
  cudaMemcpyAsync(hs + 2, mcnt, sizeof(int64_t), cudaMemcpyDeviceToHost, s);
  cudaMemcpyAsync(hs + 3, mcnt + 2, 2 * sizeof(int64_t), cudaMemcpyDeviceToHost, s);
  cudaMemcpyAsync(hs + 5, tot + 6, sizeof(int64_t), cudaMemcpyDeviceToHost, s);
  if (!sync()) return ST_CUDA_ERROR;
  C.n_ring_vertices = hs[5];
  double* oxy = A.take_n<double>(2 * hs[0]);
  int32_t* ocsz = A.take_n<int32_t>(hs[1]);
  const int64_t nMid = hs[2], nTile = hs[3], nWarp = hs[4];
  if (!oxy || !ocsz) return ST_OUT_OF_MEMORY;
  mk->mark("clip:fill+link", s);
  {
    cudaMemsetAsync(nc, 0, K * sizeof(int32_t), s);
    cudaMemsetAsync(nv, 0, K * sizeof(int64_t), s);
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    LabelArgs la{D, K, mP, mQ, regP, regQ, regSizeP, regSizeQ, SP, SQ, oxy, vOff, vcap, ocsz, cOff, ccap, nc, nv,
                 prm, d_err, prm.tile_label_max, midMin, prm.big_label_min, mcnt, mcnt + 1, 0, oval,
                 nTile, nWarp};
    // long pairs: a block each, on the auxiliary stream when there is one, so they start
    // first and overlap the warp-per-pair kernel instead of trailing it
    cudaStream_t ls = s;
    cudaEvent_t fork = nullptr, join = nullptr;
    if (aux && cudaEventCreateWithFlags(&fork, cudaEventDisableTiming) == cudaSuccess &&
        cudaEventCreateWithFlags(&join, cudaEventDisableTiming) == cudaSuccess) {
      cudaEventRecord(fork, s);
      cudaStreamWaitEvent(aux, fork, 0);
      ls = aux;
    }
    if (nMid > 0) {
      // The run table goes to shared memory only when block pairs make up at least a
      // quarter of the batch: otherwise the one-thread and warp kernels beside this one
      // need the SMs' L1 more (batched workload: label stage 2.02 -> 2.52 ms with it).
      const int smem = (4 * nMid >= K) ? kBlockRunTableBytes : 0;
      auto kern = prm.exact ? label_trace_block_kernel<1> : label_trace_block_kernel<0>;
      if (smem) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
      la.blockRunCap = smem / 12;
      kern<<<(unsigned)std::min<int64_t>(2 * nsm, nMid), kBlockLabelThreads, smem, ls>>>(la);
      note_launch();
    }
    const bool wide = K >= prm.wide_label_min;
    // the warp-per-pair pairs on the third stream, beside the one-thread pairs on s
    cudaStream_t ws = s;
    cudaEvent_t wfork = nullptr, wjoin = nullptr;
    if (aux2 && cudaEventCreateWithFlags(&wfork, cudaEventDisableTiming) == cudaSuccess &&
        cudaEventCreateWithFlags(&wjoin, cudaEventDisableTiming) == cudaSuccess) {
      cudaEventRecord(wfork, s);
      cudaStreamWaitEvent(aux2, wfork, 0);
      ws = aux2;
    }
    if (nWarp > 0)
      { (prm.exact ? label_trace_kernel<1, 0>
                   : (wide ? label_trace_kernel<0, 1> : label_trace_kernel<0, 0>))<<<(unsigned)((nWarp + 3) / 4), 128, 0, ws>>>(la); note_launch(); }
    if (nTile > 0)
      { (prm.exact ? label_trace_tile_kernel<1, 0>
                   : (wide ? label_trace_tile_kernel<0, 1> : label_trace_tile_kernel<0, 0>))<<<(unsigned)((nTile + 127) / 128), 128, 0, s>>>(la); note_launch(); }
    if (ws != s) {
      cudaEventRecord(wjoin, ws);
      cudaStreamWaitEvent(s, wjoin, 0);
    }
    if (wfork) cudaEventDestroy(wfork);
    if (wjoin) cudaEventDestroy(wjoin);
    if (ls != s) {
      cudaEventRecord(join, ls);
      cudaStreamWaitEvent(s, join, 0);
    }
    if (fork) cudaEventDestroy(fork);
    if (join) cudaEventDestroy(join);
  }
  // ---- G7 grid path for huge pairs
  {
    int64_t* blist = A.take_n<int64_t>(K);
    unsigned long long* nbl = A.take_n<unsigned long long>(1);
    BigFlags* dflags = A.take_n<BigFlags>(1);
    if (!blist || !nbl || !dflags) return ST_OUT_OF_MEMORY;
    cudaMemsetAsync(nbl, 0, sizeof(unsigned long long), s);
    { big_label_list_kernel<<<blocks_for(K), kThreads, 0, s>>>(mP, mQ, D.status, K, prm.big_label_min, blist, nbl); note_launch(); }
    cudaMemcpyAsync(hs, nbl, sizeof(int64_t), cudaMemcpyDeviceToHost, s);
    if (!sync()) return ST_CUDA_ERROR;
    const int nbig = (int)hs[0];
    if (nbig > 0) {
      BigPair* dbp = A.take_n<BigPair>(nbig);
      if (!dbp) return ST_OUT_OF_MEMORY;
      { big_info_label_kernel<<<blocks_for(nbig), kThreads, 0, s>>>(blist, nbig, regP, regQ, mP, mQ, regSizeP, regSizeQ,
                                                                    vOff, vcap, cOff, ccap, dbp); note_launch(); }
      std::vector<BigPair> hbp(nbig);
      cudaMemcpyAsync(hbp.data(), dbp, nbig * sizeof(BigPair), cudaMemcpyDeviceToHost, s);
      if (!sync()) return ST_CUDA_ERROR;
      std::sort(hbp.begin(), hbp.end(), [](const BigPair& x, const BigPair& y) { return x.k < y.k; });
      BigCtx bc{A, s, hs, d_err, SP, SQ, oxy, ocsz, D.status, nc, nv, prm};
      for (const BigPair& bp : hbp) {
        int st = run_big_label_pair(bc, bp, dflags);
        if (st != ST_OK) return st;
      }
    }
  }
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
