// join.cu -- GCMF spatial join on sm_100a: MBR build, sort-and-sweep MBR filter,
// common MBR + containment candidates, point-in-polygon, common-MBR edge filter and
// segment-intersection refine.
//
// Reference path (spatialJoin3.cu:254-348): SortBaseMBROverlap (Join.h:5-153), GetCMBR
// (Join.h:397-432), PointInPolygonTest (Join.h:437-467), CountCMF/ApplyCMF
// (Join.h:157-287), SegmentIntersectJoin (Join.h:356-393).
//
// Layout in HBM: layers stay in the reference's interleaved FP64 layout (16 B per
// vertex, read as one 128-bit load per vertex).  Per layer the MBRs are kept as
// [minx, miny, maxx, maxy] FP64 rows plus a sorted structure-of-arrays copy (x1, x2,
// y1, y2, id) in ascending x1 order, which is what the sweep streams.
#include <algorithm>
#include <vector>
#include "common.cuh"
#include "engine.cuh"
#include "grid.cuh"
#include "prims.cuh"

namespace gcmfgh {

namespace {

constexpr int kThreads = 256;
constexpr int kWarpsPerBlock = kThreads / 32;

inline unsigned blocks_for_warps(int64_t warps) {
  return (unsigned)((warps + kWarpsPerBlock - 1) / kWarpsPerBlock);
}
inline unsigned blocks_for(int64_t n) { return (unsigned)((n + kThreads - 1) / kThreads); }
inline unsigned blocks_for_tiles(int64_t units, int w) {
  const int64_t per = (int64_t)kThreads / w;
  return (unsigned)((units + per - 1) / per);
}

// W lanes of a warp working on one pair (W = 32: the whole warp).  Pairs are small in the
// bulk of a join, so narrow tiles put more pairs in flight per warp; the launches split
// pairs by size between a narrow-tile pass and a whole-warp pass.
template <int W>
struct JTile {
  static constexpr unsigned kBits = (W == 32) ? 0xffffffffu : ((1u << (W & 31)) - 1u);
  int lane, base;
  unsigned mask;
  __device__ __forceinline__ JTile() {
    lane = (int)(threadIdx.x & (W - 1));
    base = (int)(lane_id() & ~(unsigned)(W - 1));
    mask = kBits << base;
  }
  __device__ __forceinline__ unsigned ballot(bool v) const {
    const unsigned b = __ballot_sync(mask, v);
    return (W == 32) ? b : ((b >> base) & kBits);
  }
  __device__ __forceinline__ unsigned lanes_below() const { return (1u << lane) - 1u; }
  static __device__ __forceinline__ int64_t unit() {
    return ((int64_t)blockIdx.x * kThreads + threadIdx.x) / W;
  }
};

// ---------------------------------------------------------------- J0: MBRs
// 128-bit vertex loads.  The MBR covers every stored vertex, the closing one included
// (SEQ_Overlay.h:316-344).  Zero-width or zero-height MBRs are rejected like the
// reference reader does (SEQ_Overlay.h:336-344): such a polygon never joins.  Valid
// polygons get the order-preserving key of their x1 for the sweep sort.  A warp takes four
// consecutive polygons: 8 lanes each when all four have at most 64 stored vertices (most
// polygons), else all 32 lanes for one polygon after another.
// Sweep sort key of a valid polygon: the order-preserving bits of x1 rounded down to FP32,
// at most 0xFFFFFFFE (0xFFFFFFFF marks the invalid ones, which sort last).  Monotone in x1,
// so sorting these 32 bits (4 radix passes instead of 8) orders the polygons by x1 up to
// runs of equal keys, which x1_fixup_kernel puts in exact (x1, id) order.
__device__ __forceinline__ uint64_t x1_key32(double x1) {
  const uint32_t b = __float_as_uint(__double2float_rd(x1));
  const uint32_t k = (b & 0x80000000u) ? ~b : (b | 0x80000000u);
  return k < 0xFFFFFFFFu ? k : 0xFFFFFFFEu;
}

template <int W>
__device__ __forceinline__ void mbr_reduce(double& x1, double& y1, double& x2, double& y2) {
#pragma unroll
  for (int o = W / 2; o > 0; o >>= 1) {
    double t = __shfl_xor_sync(0xffffffffu, x1, o); x1 = t < x1 ? t : x1;
    t = __shfl_xor_sync(0xffffffffu, y1, o); y1 = t < y1 ? t : y1;
    t = __shfl_xor_sync(0xffffffffu, x2, o); x2 = t > x2 ? t : x2;
    t = __shfl_xor_sync(0xffffffffu, y2, o); y2 = t > y2 ? t : y2;
  }
}

__device__ __forceinline__ bool mbr_write(int64_t w, int nv, double x1, double y1, double x2, double y2,
                                          double* __restrict__ mbr, uint8_t* __restrict__ valid,
                                          uint64_t* __restrict__ key, uint32_t* __restrict__ id) {
  const bool ok = nv >= 2 && x1 != x2 && y1 != y2;
  reinterpret_cast<double4*>(mbr)[w] = make_double4(x1, y1, x2, y2);
  valid[w] = ok ? 1 : 0;
  key[w] = ok ? x1_key32(x1) : ~0ull;
  id[w] = (uint32_t)w;
  return ok;
}

constexpr int kMbrPerWarp = 4;
constexpr int kMbrSmallMax = 64;

__global__ void __launch_bounds__(kThreads)
mbr_kernel(LayerDev L, double* __restrict__ mbr, uint8_t* __restrict__ valid,
           uint64_t* __restrict__ key, uint32_t* __restrict__ id, unsigned long long* n_valid,
           float2* __restrict__ xyf) {
  const int64_t p0 = (((int64_t)blockIdx.x * kThreads + threadIdx.x) >> 5) * kMbrPerWarp;
  if (p0 >= L.n) return;
  const int lane = (int)lane_id();
  const int mine = (lane < kMbrPerWarp && p0 + lane < L.n) ? L.vnum[p0 + lane] : 0;
  int ok = 0;
  if (__all_sync(0xffffffffu, mine <= kMbrSmallMax)) {
    constexpr int W = 32 / kMbrPerWarp;
    const int g = lane / W, t = lane % W;
    const int64_t w = p0 + g;
    const int nv = __shfl_sync(0xffffffffu, mine, g);
    double x1 = INFINITY, y1 = INFINITY, x2 = -INFINITY, y2 = -INFINITY;
    if (w < L.n) {
      const int64_t s = L.vps[w] - nv;
      const double2* v = reinterpret_cast<const double2*>(L.xy) + s;
      for (int k = t; k < nv; k += W) {
        double2 p = __ldg(v + k);
        if (xyf) xyf[s + k] = make_float2(__double2float_rn(p.x), __double2float_rn(p.y));
        x1 = fmin(x1, p.x); x2 = fmax(x2, p.x);
        y1 = fmin(y1, p.y); y2 = fmax(y2, p.y);
      }
    }
    mbr_reduce<W>(x1, y1, x2, y2);
    if (t == 0 && w < L.n) ok = mbr_write(w, nv, x1, y1, x2, y2, mbr, valid, key, id) ? 1 : 0;
  } else {
    for (int g = 0; g < kMbrPerWarp && p0 + g < L.n; ++g) {
      const int64_t w = p0 + g;
      const int nv = __shfl_sync(0xffffffffu, mine, g);
      const int64_t s = L.vps[w] - nv;
      const double2* v = reinterpret_cast<const double2*>(L.xy) + s;
      double x1 = INFINITY, y1 = INFINITY, x2 = -INFINITY, y2 = -INFINITY;
      for (int k = lane; k < nv; k += 32) {
        double2 p = __ldg(v + k);
        if (xyf) xyf[s + k] = make_float2(__double2float_rn(p.x), __double2float_rn(p.y));
        x1 = fmin(x1, p.x); x2 = fmax(x2, p.x);
        y1 = fmin(y1, p.y); y2 = fmax(y2, p.y);
      }
      mbr_reduce<32>(x1, y1, x2, y2);
      if (lane == 0) ok += mbr_write(w, nv, x1, y1, x2, y2, mbr, valid, key, id) ? 1 : 0;
    }
  }
  ok = __reduce_add_sync(0xffffffffu, ok);
  if (lane == 0 && ok) atomicAdd(n_valid, (unsigned long long)ok);
}

// Runs of equal 32-bit keys among the first nv sorted entries: each run's first thread
// sorts the run's ids by (ordered_key(x1), id), which makes the order that of a stable sort
// on the full 64-bit key.  Runs longer than kFixupMaxRun set *flag instead (the caller then
// sorts on 64 bits).
constexpr int kFixupMaxRun = 256;
__global__ void x1_fixup_kernel(const uint64_t* __restrict__ key, uint32_t* __restrict__ id, int64_t nv,
                                const double* __restrict__ mbr, unsigned long long* __restrict__ flag) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nv) return;
  const uint64_t k = key[i];
  if (i > 0 && key[i - 1] == k) return;                 // not the first of its run
  if (i + 1 >= nv || key[i + 1] != k) return;           // a run of one
  int64_t j = i + 1;
  while (j < nv && key[j] == k) {
    if (j - i >= kFixupMaxRun) { atomicAdd(flag, 1ull); return; }
    ++j;
  }
  for (int64_t a = i + 1; a < j; ++a) {                 // insertion sort, stable in id
    const uint32_t v = id[a];
    const uint64_t kv = ordered_key(mbr[4 * (int64_t)v]);
    int64_t b = a - 1;
    while (b >= i) {
      const uint32_t u = id[b];
      const uint64_t ku = ordered_key(mbr[4 * (int64_t)u]);
      if (ku < kv || (ku == kv && u < v)) break;
      id[b + 1] = u;
      --b;
    }
    id[b + 1] = v;
  }
}

// the full 64-bit sweep keys (for layers whose 32-bit keys leave long runs)
__global__ void x1_key64_kernel(const double* __restrict__ mbr, const uint8_t* __restrict__ valid, int64_t n,
                                uint64_t* __restrict__ key, uint32_t* __restrict__ id) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  key[i] = valid[i] ? ordered_key(mbr[4 * i]) : ~0ull;
  id[i] = (uint32_t)i;
}

// yf: (y1 rounded down, y2 rounded up) in FP32 -- a box that contains the FP64 one
struct SortedMbr { double *x1, *x2, *y1, *y2; uint32_t* id; int64_t n; float2* yf; };

__global__ void gather_sorted_kernel(const double* __restrict__ mbr, const uint32_t* __restrict__ ids,
                                     int64_t n, SortedMbr S) {
  int64_t i = (int64_t)blockIdx.x * kThreads + threadIdx.x;
  if (i >= n) return;
  uint32_t id = ids[i];
  double4 m = reinterpret_cast<const double4*>(mbr)[id];
  S.x1[i] = m.x; S.y1[i] = m.y; S.x2[i] = m.z; S.y2[i] = m.w; S.id[i] = id;
  if (S.yf) S.yf[i] = make_float2(__double2float_rd(m.y), __double2float_ru(m.w));
}

// Warp-cooperative search in an ascending array (all 32 lanes call it with the same
// arguments): the first index whose element is not "before" x, where before means
// a[i] < x (lower bound) or a[i] <= x (upper bound).  Each round the lanes probe 32
// evenly spaced elements at once and the range shrinks 32-fold, so a search costs
// log32(n) dependent loads instead of log2(n).
template <bool kUpper>
__device__ __forceinline__ int64_t warp_bound(const double* a, int64_t n, double x) {
  int64_t lo = 0, hi = n;                       // the answer lies in [lo, hi]
  const int l = (int)lane_id();
  while (hi - lo > 32) {
    const int64_t seg = (hi - lo + 31) / 32;
    int64_t p = lo + (int64_t)(l + 1) * seg - 1;
    const bool in = p < hi;
    const double v = in ? a[p] : 0.0;
    const bool before = in && (kUpper ? v <= x : v < x);
    const int c = __popc(__ballot_sync(0xffffffffu, before));
    const int64_t plo = lo + (int64_t)c * seg - 1;            // last probe that is before
    const int64_t phi = lo + (int64_t)(c + 1) * seg - 1;      // first probe that is not
    if (c > 0) lo = plo + 1;
    if (c < 32 && phi < hi) hi = phi;
  }
  const int64_t q = lo + l;
  const bool before = q < hi && (kUpper ? a[q] <= x : a[q] < x);
  return lo + __popc(__ballot_sync(0xffffffffu, before));
}
// first index with a[i] >= x / with a[i] > x
__device__ __forceinline__ int64_t lower_bound_d(const double* a, int64_t n, double x) { return warp_bound<false>(a, n, x); }
__device__ __forceinline__ int64_t upper_bound_d(const double* a, int64_t n, double x) { return warp_bound<true>(a, n, x); }

// ---------------------------------------------------------------- J2: sweep
// The reference sorts all x endpoints (stable on endpoint index, base before overlay)
// and lets each polygon scan the sorted positions strictly between its own endpoints
// for other-layer starts, then checks y (GPU_MBR.h:339-415, 420-539).  On values this
// accepts (b, o) iff [x1b <= x1o < x2b] or [x1o < x1b <= x2o], with closed y overlap.
// Here each base polygon takes the overlays that start in [x1b, x2b) and each overlay
// takes the bases that start in (x1o, x2o]; both ranges are binary searches in the
// other layer's x1-sorted array, and only the y test remains inside the range.
// mode 0: count per element, mode 1: emit keys (b << obits | o) at offs[element].
// kF32: the y test first on outward-rounded FP32 boxes (8 bytes per candidate; a superset,
// as rd(y1) <= y1 <= my2 <= ru(my2)), then in FP64 for the boxes that pass -- the same
// candidates either way.
template <int kMode, int kF32>
__global__ void __launch_bounds__(kThreads, 8)
sweep_kernel(SortedMbr B, SortedMbr O, int32_t* __restrict__ cnt, const int64_t* __restrict__ offs,
             uint64_t* __restrict__ keys, int obits) {
  int64_t w = ((int64_t)blockIdx.x * kThreads + threadIdx.x) >> 5;
  if (w >= B.n + O.n) return;
  const bool base_side = w < B.n;
  const SortedMbr& me = base_side ? B : O;
  const SortedMbr& ot = base_side ? O : B;
  const int64_t i = base_side ? w : w - B.n;
  const double mx1 = me.x1[i], mx2 = me.x2[i], my1 = me.y1[i], my2 = me.y2[i];
  const float my1d = kF32 ? __double2float_rd(my1) : 0.f, my2u = kF32 ? __double2float_ru(my2) : 0.f;
  int64_t lo, hi;
  if (base_side) { lo = lower_bound_d(ot.x1, ot.n, mx1); hi = lower_bound_d(ot.x1, ot.n, mx2); }
  else { lo = upper_bound_d(ot.x1, ot.n, mx1); hi = upper_bound_d(ot.x1, ot.n, mx2); }
  int c = 0;
  int64_t pos = (kMode == 1) ? offs[w] : 0;
  const uint64_t myid = me.id[i];
  for (int64_t k0 = lo; k0 < hi; k0 += 32) {
    int64_t k = k0 + lane_id();
    bool hit = false;
    if (k < hi) {
      if (kF32) {
        const float2 q = ot.yf[k];
        hit = q.x <= my2u && my1d <= q.y;
        if (hit) hit = ot.y1[k] <= my2 && my1 <= ot.y2[k];
      } else {
        hit = ot.y1[k] <= my2 && my1 <= ot.y2[k];
      }
    }
    unsigned m = __ballot_sync(0xffffffffu, hit);
    if (kMode == 1 && hit) {
      uint64_t oid = ot.id[k];
      uint64_t b = base_side ? myid : oid, o = base_side ? oid : myid;
      keys[pos + __popc(m & lanemask_lt())] = (b << obits) | o;
    }
    c += __popc(m);
    pos += __popc(m);
  }
  if (kMode == 0 && lane_id() == 0) cnt[w] = c;
}

// The sweep's count and emit in one pass: the same range scan and tests as sweep_kernel,
// with each warp staging its keys in shared memory (up to kSweepStage; a fuller stage is
// appended by the warp itself) and the block appending all staged keys at one range of a
// global counter.  Keys land in no particular order (the caller sorts them); those at or
// past cap are counted and not written, and the caller runs the pass again with room for
// the counted total.
constexpr int kSweepStage = 64;
template <int kF32>
__global__ void __launch_bounds__(kThreads, 8)
sweep_append_kernel(SortedMbr B, SortedMbr O, uint64_t* __restrict__ keys, int64_t cap,
                    unsigned long long* __restrict__ total, int obits) {
  __shared__ uint64_t stage[kWarpsPerBlock][kSweepStage];
  __shared__ int sOff[kWarpsPerBlock + 1];
  __shared__ unsigned long long sBase;
  const int wib = (int)(threadIdx.x >> 5);
  const int64_t w = ((int64_t)blockIdx.x * kThreads + threadIdx.x) >> 5;
  int staged = 0;
  if (w < B.n + O.n) {
    const bool base_side = w < B.n;
    const SortedMbr& me = base_side ? B : O;
    const SortedMbr& ot = base_side ? O : B;
    const int64_t i = base_side ? w : w - B.n;
    const double mx1 = me.x1[i], mx2 = me.x2[i], my1 = me.y1[i], my2 = me.y2[i];
    const float my1d = kF32 ? __double2float_rd(my1) : 0.f, my2u = kF32 ? __double2float_ru(my2) : 0.f;
    int64_t lo, hi;
    if (base_side) { lo = lower_bound_d(ot.x1, ot.n, mx1); hi = lower_bound_d(ot.x1, ot.n, mx2); }
    else { lo = upper_bound_d(ot.x1, ot.n, mx1); hi = upper_bound_d(ot.x1, ot.n, mx2); }
    const uint64_t myid = me.id[i];
    for (int64_t k0 = lo; k0 < hi; k0 += 32) {
      const int64_t k = k0 + lane_id();
      bool hit = false;
      if (k < hi) {
        if (kF32) {
          const float2 q = ot.yf[k];
          hit = q.x <= my2u && my1d <= q.y;
          if (hit) hit = ot.y1[k] <= my2 && my1 <= ot.y2[k];
        } else {
          hit = ot.y1[k] <= my2 && my1 <= ot.y2[k];
        }
      }
      const unsigned m = __ballot_sync(0xffffffffu, hit);
      const int nh = __popc(m);
      if (staged + nh > kSweepStage) {              // append the full stage now
        unsigned long long b = 0;
        if (lane_id() == 0) b = atomicAdd(total, (unsigned long long)staged);
        b = __shfl_sync(0xffffffffu, b, 0);
        for (int j = lane_id(); j < staged; j += 32)
          if ((int64_t)b + j < cap) keys[b + j] = stage[wib][j];
        __syncwarp();
        staged = 0;
      }
      if (hit) {
        const uint64_t oid = ot.id[k];
        const uint64_t bb = base_side ? myid : oid, oo = base_side ? oid : myid;
        stage[wib][staged + __popc(m & lanemask_lt())] = (bb << obits) | oo;
      }
      __syncwarp();
      staged += nh;
    }
  }
  if (lane_id() == 0) sOff[wib] = staged;
  __syncthreads();
  if (threadIdx.x == 0) {
    int run = 0;
    for (int j = 0; j < kWarpsPerBlock; ++j) { const int n = sOff[j]; sOff[j] = run; run += n; }
    sOff[kWarpsPerBlock] = run;
    sBase = run ? atomicAdd(total, (unsigned long long)run) : 0ull;
  }
  __syncthreads();
  const int64_t base = (int64_t)sBase + sOff[wib];
  for (int j = lane_id(); j < staged; j += 32)
    if (base + j < cap) keys[base + j] = stage[wib][j];
}

// ---------------------------------------------------------------- J3: common MBR
// GPU_Join.h:468-506: CMBR = intersection of the FP64 MBRs; pip_type 1 when the base
// MBR equals the CMBR (the overlay may contain the base), 2 when the overlay MBR does.
__global__ void cmbr_kernel(const uint64_t* __restrict__ keys, int64_t K, int obits,
                            const double* __restrict__ mb, const double* __restrict__ mo,
                            int32_t* __restrict__ ob, int32_t* __restrict__ oo,
                            double* __restrict__ cmbr, int8_t* __restrict__ pip_type) {
  int64_t k = (int64_t)blockIdx.x * kThreads + threadIdx.x;
  if (k >= K) return;
  uint64_t key = keys[k];
  int32_t b = (int32_t)(key >> obits);
  int32_t o = (int32_t)(key & ((1ull << obits) - 1));
  ob[k] = b; oo[k] = o;
  double4 B = reinterpret_cast<const double4*>(mb)[b];
  double4 O = reinterpret_cast<const double4*>(mo)[o];
  double x1 = B.x, y1 = B.y, x2 = B.z, y2 = B.w;
  double a1 = O.x, b1 = O.y, a2 = O.z, b2 = O.w;
  double cx1 = (a1 > x1 ? a1 : x1), cx2 = (a2 < x2 ? a2 : x2);
  double cy1 = (b1 > y1 ? b1 : y1), cy2 = (b2 < y2 ? b2 : y2);
  reinterpret_cast<double4*>(cmbr)[k] = make_double4(cx1, cy1, cx2, cy2);
  int8_t t = 0;
  if (x1 == cx1 && x2 == cx2 && y1 == cy1 && y2 == cy2) t = 1;
  else if (a1 == cx1 && a2 == cx2 && b1 == cy1 && b2 == cy2) t = 2;
  pip_type[k] = t;
}

// ---------------------------------------------------------------- J4: containment
// Crossing parity of the contained candidate's first vertex against the other polygon's
// stored ring, edges (i, i-1) for every stored vertex i (GPU_Join.h:856-939).  A warp per
// candidate pair; the parity of the per-lane parities equals the reference's XOR scan.
template <int W>
__global__ void __launch_bounds__(kThreads, 6)
pip_kernel(LayerDev Lb, LayerDev Lo, const int32_t* __restrict__ pb, const int32_t* __restrict__ po,
           const int8_t* __restrict__ pip_type, int64_t K, int8_t* __restrict__ pip_flag,
           int8_t* __restrict__ join_flag, int64_t lo, int64_t hi) {
  const JTile<W> T;
  const int64_t w = JTile<W>::unit();
  if (w >= K) return;
  int t = pip_type[w];
  if (t == 0) {
    if (W != 32 && T.lane == 0) { pip_flag[w] = 0; join_flag[w] = 1; }
    return;
  }
  int b = pb[w], o = po[w];
  const LayerDev& Lp = (t == 1) ? Lb : Lo;     // layer of the point
  const LayerDev& Lr = (t == 1) ? Lo : Lb;     // layer of the ring
  int ip = (t == 1) ? b : o, ir = (t == 1) ? o : b;
  const double2* pt = reinterpret_cast<const double2*>(Lp.xy) + (Lp.vps[ip] - Lp.vnum[ip]);
  const double2 P = pt[0];
  const int nv = Lr.vnum[ir];
  if (nv <= lo || nv > hi) return;                 // the other pass takes this pair
  const double2* v = reinterpret_cast<const double2*>(Lr.xy) + (Lr.vps[ir] - nv);
  int par = 0;
  for (int i = T.lane; i < nv; i += W) {
    int j = (i == 0) ? nv - 1 : i - 1;
    double2 a = __ldg(v + i), c = __ldg(v + j);
    double Y1 = a.y, Y2 = c.y, X1 = a.x, X2 = c.x;
    if ((Y1 > P.y) == (Y2 > P.y)) continue;
    if (P.x < (X2 - X1) * (P.y - Y1) / (Y2 - Y1) + X1) par ^= 1;
  }
  int inside = __popc(T.ballot(par)) & 1;
  if (T.lane == 0) { pip_flag[w] = (int8_t)inside; join_flag[w] = inside ? 0 : 1; }
}

// ---------------------------------------------------------------- J5: common-MBR filter
// (Launch bounds here and on the sweep and point-in-polygon kernels trade registers for
// resident warps: these loops wait on loads, and the extra warps hide more of it --
// sweep 1.09 -> 0.94 ms, CMF 0.92 -> 0.73 ms on the batched workload.)
// Edges whose box touches the CMBR (GPU_Join.h:562-580); edge k of a stored ring runs
// from vertex k to k+1 and the last one from the closing vertex back to vertex 0.
// mode 0 counts (and drops pairs with an empty side, :604-613), mode 1 writes the
// surviving edge ids in ascending order (Apply_CMF :676-733, 32-bit ids here).
// kF32: each edge is first tested on the FP32 copies of its vertices, rejected only when
// the rejection holds with one FP32 ulp of room on each side (rn(v) is within half an ulp of
// v, so nextafter(rn(v)) bounds v); the edges that pass are tested in FP64.  The edge sets
// are those of the FP64 test alone.
__device__ __forceinline__ bool f32_rejects(float2 a, float2 b, float cx1d, float cy1d, float cx2u, float cy2u) {
  const float xmax = nextafterf(fmaxf(a.x, b.x), INFINITY), xmin = nextafterf(fminf(a.x, b.x), -INFINITY);
  const float ymax = nextafterf(fmaxf(a.y, b.y), INFINITY), ymin = nextafterf(fminf(a.y, b.y), -INFINITY);
  return cx1d > xmax || cx2u < xmin || cy1d > ymax || cy2u < ymin;
}

template <int kMode, int W, int kF32>
__global__ void __launch_bounds__(kThreads, 8)
cmf_kernel(LayerDev Lb, LayerDev Lo, const int32_t* __restrict__ pb, const int32_t* __restrict__ po,
           const double* __restrict__ cmbr, int64_t K, int8_t* __restrict__ join_flag,
           int32_t* __restrict__ bE, int32_t* __restrict__ oE,
           const int64_t* __restrict__ bOff, const int64_t* __restrict__ oOff,
           int32_t* __restrict__ bList, int32_t* __restrict__ oList, int64_t lo, int64_t hi) {
  const JTile<W> T;
  const int64_t w = JTile<W>::unit();
  if (w >= K) return;
  if (!join_flag[w]) {
    if (kMode == 0 && W != 32 && T.lane == 0) { bE[w] = 0; oE[w] = 0; }
    return;
  }
  if (kMode == 1 && bE[w] == 0) return;
  {
    const int64_t size = (int64_t)Lb.vnum[pb[w]] + Lo.vnum[po[w]];
    if (size <= lo || size > hi) return;             // the other pass takes this pair
  }
  double4 c = reinterpret_cast<const double4*>(cmbr)[w];
  const float cx1d = kF32 ? __double2float_rd(c.x) : 0.f, cy1d = kF32 ? __double2float_rd(c.y) : 0.f;
  const float cx2u = kF32 ? __double2float_ru(c.z) : 0.f, cy2u = kF32 ? __double2float_ru(c.w) : 0.f;
  int counts[2];
  for (int side = 0; side < 2; ++side) {
    const LayerDev& L = side == 0 ? Lb : Lo;
    int id = side == 0 ? pb[w] : po[w];
    const int nv = L.vnum[id];
    const double2* v = reinterpret_cast<const double2*>(L.xy) + (L.vps[id] - nv);
    const float2* vf = kF32 ? L.xyf + (L.vps[id] - nv) : nullptr;
    int64_t pos = 0;
    int32_t* list = nullptr;
    if (kMode == 1) { pos = side == 0 ? bOff[w] : oOff[w]; list = side == 0 ? bList : oList; }
    int cnt = 0;
    for (int k0 = 0; k0 < nv; k0 += W) {
      int k = k0 + T.lane;
      bool hit = false;
      if (k < nv) {
        const int k2 = (k < nv - 1) ? k + 1 : 0;
        if (!kF32 || !f32_rejects(__ldg(vf + k), __ldg(vf + k2), cx1d, cy1d, cx2u, cy2u)) {
          double2 a = __ldg(v + k), b = __ldg(v + k2);
          hit = edge_touches_box(a.x, a.y, b.x, b.y, c.x, c.y, c.z, c.w);
        }
      }
      unsigned m = T.ballot(hit);
      if (kMode == 1 && hit) list[pos + cnt + __popc(m & T.lanes_below())] = k;
      cnt += __popc(m);
    }
    counts[side] = cnt;
  }
  if (kMode == 0 && T.lane == 0) {
    if (counts[0] == 0 || counts[1] == 0) { join_flag[w] = 0; bE[w] = 0; oE[w] = 0; }
    else { bE[w] = counts[0]; oE[w] = counts[1]; }
  }
}

// The common-MBR filter's count and lists in one pass.  Each tile (W lanes per pair) tests
// its pair's edges once to count them, as cmf_kernel's count pass does; the block then takes
// one range of each list array for all its pairs (two atomics per block), and each tile
// tests its edges again, from L1, to write them in ascending order at its pair's offset.
// A pair's lists stay contiguous and ascending; pairs sit in no particular order
// (bOff/oOff say where).  Entries at or past cap are counted and not written: the caller
// runs the pass again with room for the counted totals.
struct CmfOut {
  int64_t* bOff; int64_t* oOff;
  int32_t* bList; int32_t* oList;
  int64_t bCap, oCap;
  unsigned long long* total;     // [2] entries taken so far (base, overlay)
};

template <int W, int kF32>
__global__ void __launch_bounds__(kThreads, 8)
cmf_append_kernel(LayerDev Lb, LayerDev Lo, const int32_t* __restrict__ pb, const int32_t* __restrict__ po,
                  const double* __restrict__ cmbr, int64_t K, int8_t* __restrict__ join_flag,
                  int32_t* __restrict__ bE, int32_t* __restrict__ oE, CmfOut out, int64_t lo, int64_t hi) {
  constexpr int kTiles = kThreads / W;
  __shared__ int sCnt[2][kTiles];
  __shared__ unsigned long long sBase[2];
  const JTile<W> T;
  const int64_t w = JTile<W>::unit();
  const int tib = (int)(threadIdx.x / W);
  bool mine = w < K && join_flag[w];
  if (w < K && !join_flag[w] && W != 32 && T.lane == 0) { bE[w] = 0; oE[w] = 0; }
  if (mine) {
    const int64_t size = (int64_t)Lb.vnum[pb[w]] + Lo.vnum[po[w]];
    mine = size > lo && size <= hi;                 // else the other pass takes this pair
  }
  double4 c = make_double4(0, 0, 0, 0);
  float cx1d = 0.f, cy1d = 0.f, cx2u = 0.f, cy2u = 0.f;
  int counts[2] = {0, 0};
  if (mine) {
    c = reinterpret_cast<const double4*>(cmbr)[w];
    if (kF32) {
      cx1d = __double2float_rd(c.x); cy1d = __double2float_rd(c.y);
      cx2u = __double2float_ru(c.z); cy2u = __double2float_ru(c.w);
    }
  }
  // pass 0 counts, pass 1 writes
  for (int pass = 0; pass < 2; ++pass) {
    if (pass == 1) {
      if (T.lane == 0) {
        const bool keep = mine && counts[0] > 0 && counts[1] > 0;
        sCnt[0][tib] = keep ? counts[0] : 0;
        sCnt[1][tib] = keep ? counts[1] : 0;
        if (mine && !keep) { join_flag[w] = 0; bE[w] = 0; oE[w] = 0; }
      }
      __syncthreads();
      if (threadIdx.x < 2) {
        int run = 0;
        for (int j = 0; j < kTiles; ++j) { const int n = sCnt[threadIdx.x][j]; sCnt[threadIdx.x][j] = run; run += n; }
        sBase[threadIdx.x] = run ? atomicAdd(out.total + threadIdx.x, (unsigned long long)run) : 0ull;
      }
      __syncthreads();
      if (!(mine && counts[0] > 0 && counts[1] > 0)) break;
      if (T.lane == 0) {
        out.bOff[w] = (int64_t)sBase[0] + sCnt[0][tib];
        out.oOff[w] = (int64_t)sBase[1] + sCnt[1][tib];
        bE[w] = counts[0];
        oE[w] = counts[1];
      }
    } else if (!mine) {
      continue;
    }
    for (int side = 0; side < 2; ++side) {
      const LayerDev& L = side == 0 ? Lb : Lo;
      const int id = side == 0 ? pb[w] : po[w];
      const int nv = L.vnum[id];
      const double2* v = reinterpret_cast<const double2*>(L.xy) + (L.vps[id] - nv);
      const float2* vf = kF32 ? L.xyf + (L.vps[id] - nv) : nullptr;
      const int64_t pos = pass == 1 ? (int64_t)sBase[side] + sCnt[side][tib] : 0;
      int32_t* list = side == 0 ? out.bList : out.oList;
      const int64_t cap = side == 0 ? out.bCap : out.oCap;
      int cnt = 0;
      for (int k0 = 0; k0 < nv; k0 += W) {
        const int k = k0 + T.lane;
        bool hit = false;
        if (k < nv) {
          const int k2 = (k < nv - 1) ? k + 1 : 0;
          if (!kF32 || !f32_rejects(__ldg(vf + k), __ldg(vf + k2), cx1d, cy1d, cx2u, cy2u)) {
            const double2 a = __ldg(v + k), b = __ldg(v + k2);
            hit = edge_touches_box(a.x, a.y, b.x, b.y, c.x, c.y, c.z, c.w);
          }
        }
        const unsigned m = T.ballot(hit);
        if (pass == 1 && hit) {
          const int64_t r = pos + cnt + __popc(m & T.lanes_below());
          if (r < cap) list[r] = k;
        }
        cnt += __popc(m);
      }
      if (pass == 0) counts[side] = cnt;
    }
  }
}

// ---------------------------------------------------------------- J6: refine
// Does any surviving (base edge, overlay edge) pair intersect?  The closed-form test of
// GPU_Join.h:373-446 in its operation order: zero-length base edges are skipped, box
// rejects, the collinear branch via slopes and intercepts, then the intersection point
// against both edges' extents.  A warp per pair over the flattened bE x oE grid, with an
// early exit as soon as any lane finds an intersection (the reference's shared joinFlag).
__device__ __forceinline__ bool segment_hit(double bX1, double bY1, double bX2, double bY2,
                                            double oX1, double oY1, double oX2, double oY2) {
  if (bX1 == bX2 && bY1 == bY2) return false;
  if (((bX2 < oX1) && (bX2 < oX2)) && ((bX1 < oX1) && (bX1 < oX2))) return false;
  if (((bX2 > oX1) && (bX2 > oX2)) && ((bX1 > oX1) && (bX1 > oX2))) return false;
  if (((bY2 < oY1) && (bY2 < oY2)) && ((bY1 < oY1) && (bY1 < oY2))) return false;
  if (((bY2 > oY1) && (bY2 > oY2)) && ((bY1 > oY1) && (bY1 > oY2))) return false;
  double denom = ((bX1 - bX2) * (oY1 - oY2)) - ((bY1 - bY2) * (oX1 - oX2));
  if (denom == 0) {
    if ((oX1 == oX2 && oX1 == bX1) || (bX1 == bX2 && bX1 == oX1)) return true;
    double oM = (oY2 - oY1) / (oX2 - oX1);
    double bM = (bY2 - bY1) / (bX2 - bX1);
    double oB = oY1 - oM * oX1;
    double bB = bY1 - bM * bX1;
    return oB == bB;
  }
  double nomX = (((bX1 * bY2) - (bY1 * bX2)) * (oX1 - oX2)) - ((bX1 - bX2) * ((oX1 * oY2) - (oY1 * oX2)));
  double nomY = ((((bX1 * bY2) - (bY1 * bX2)) * (oY1 - oY2)) - (((bY1 - bY2) * ((oX1 * oY2) - (oY1 * oX2)))));
  double x0 = nomX / denom, y0 = nomY / denom;
  if ((x0 > bX1 && x0 > bX2) || (x0 < bX1 && x0 < bX2)) return false;
  if ((x0 > oX1 && x0 > oX2) || (x0 < oX1 && x0 < oX2)) return false;
  if ((y0 > bY1 && y0 > bY2) || (y0 < bY1 && y0 < bY2)) return false;
  if ((y0 > oY1 && y0 > oY2) || (y0 < oY1 && y0 < oY2)) return false;
  return true;
}

template <int W>
__global__ void __launch_bounds__(kThreads, 4)   // 64 registers: occupancy for a latency-bound loop
refine_kernel(LayerDev Lb, LayerDev Lo, const int32_t* __restrict__ pb, const int32_t* __restrict__ po,
              int64_t K, const int8_t* __restrict__ join_flag,
              const int32_t* __restrict__ bE, const int32_t* __restrict__ oE,
              const int64_t* __restrict__ bOff, const int64_t* __restrict__ oOff,
              const int32_t* __restrict__ bList, const int32_t* __restrict__ oList,
              int8_t* __restrict__ seg_flag, int64_t lo, int64_t hi) {
  const JTile<W> T;
  const int64_t w = JTile<W>::unit();
  if (w >= K) return;
  if (!join_flag[w]) { if (W != 32 && T.lane == 0) seg_flag[w] = 0; return; }
  const int nb = bE[w], no = oE[w];
  if ((int64_t)nb * no <= lo || (int64_t)nb * no > hi) return;   // the other pass takes this pair
  const int b = pb[w], o = po[w];
  const int bV = Lb.vnum[b], oV = Lo.vnum[o];
  const double2* bv = reinterpret_cast<const double2*>(Lb.xy) + (Lb.vps[b] - bV);
  const double2* ov = reinterpret_cast<const double2*>(Lo.xy) + (Lo.vps[o] - oV);
  const int32_t* bl = bList + bOff[w];
  const int32_t* ol = oList + oOff[w];
  const int64_t total = (int64_t)nb * no;
  int found = 0;
  for (int64_t t0 = 0; t0 < total && !found; t0 += W) {
    int64_t t = t0 + T.lane;
    bool hit = false;
    if (t < total) {
      int be, oe;
      if (total <= INT32_MAX) {                    // 32-bit division when it suffices
        const int tt = (int)t, r = tt / no;
        be = bl[r];
        oe = ol[tt - r * no];
      } else {
        be = bl[t / no];
        oe = ol[t % no];
      }
      double2 b1 = __ldg(bv + be), b2 = __ldg(bv + ((be < bV - 1) ? be + 1 : 0));
      double2 o1 = __ldg(ov + oe), o2 = __ldg(ov + ((oe < oV - 1) ? oe + 1 : 0));
      hit = segment_hit(b1.x, b1.y, b2.x, b2.y, o1.x, o1.y, o2.x, o2.y);
    }
    found = T.ballot(hit) != 0u;
  }
  if (T.lane == 0) seg_flag[w] = (int8_t)found;
}

// ---------------------------------------------------------------- clip set + stats
__global__ void clip_flag_kernel(const int8_t* __restrict__ pip_type, const int8_t* __restrict__ pip,
                                 const int8_t* __restrict__ join, const int8_t* __restrict__ seg,
                                 int64_t K, int8_t* __restrict__ clip, uint8_t* __restrict__ clip_u8,
                                 unsigned long long* stats) {
  int64_t k = (int64_t)blockIdx.x * kThreads + threadIdx.x;
  unsigned long long s[4] = {0, 0, 0, 0};
  if (k < K) {
    int8_t c = (pip[k] || seg[k]) ? 1 : 0;
    clip[k] = c;
    clip_u8[k] = (uint8_t)c;
    s[0] = pip_type[k] != 0; s[1] = pip[k] != 0; s[2] = join[k] != 0; s[3] = seg[k] != 0;
  }
  for (int j = 0; j < 4; ++j) {
    unsigned long long v = warp_sum(s[j]);
    if (lane_id() == 0 && v) atomicAdd(&stats[j], v);
  }
}

__global__ void clip_compact_kernel(const int8_t* __restrict__ clip, const int64_t* __restrict__ off,
                                    const int32_t* __restrict__ b, const int32_t* __restrict__ o,
                                    int64_t K, int32_t* __restrict__ cb, int32_t* __restrict__ co,
                                    int64_t* __restrict__ cand) {
  int64_t k = (int64_t)blockIdx.x * kThreads + threadIdx.x;
  if (k >= K || !clip[k]) return;
  cb[off[k]] = b[k];
  co[off[k]] = o[k];
  cand[off[k]] = k;
}

// MBRs only (the clip pipeline's common MBRs), same definition as mbr_kernel
__global__ void __launch_bounds__(kThreads)
mbr_only_kernel(LayerDev L, double* __restrict__ mbr) {
  int64_t w = ((int64_t)blockIdx.x * kThreads + threadIdx.x) >> 5;
  if (w >= L.n) return;
  const int nv = L.vnum[w];
  const double2* v = reinterpret_cast<const double2*>(L.xy) + (L.vps[w] - nv);
  double x1 = INFINITY, y1 = INFINITY, x2 = -INFINITY, y2 = -INFINITY;
  for (int k = lane_id(); k < nv; k += 32) {
    double2 p = __ldg(v + k);
    x1 = fmin(x1, p.x); x2 = fmax(x2, p.x);
    y1 = fmin(y1, p.y); y2 = fmax(y2, p.y);
  }
  x1 = warp_min(x1); y1 = warp_min(y1); x2 = warp_max(x2); y2 = warp_max(y2);
  if (lane_id() == 0) reinterpret_cast<double4*>(mbr)[w] = make_double4(x1, y1, x2, y2);
}

int bits_for(int64_t n) {
  int b = 1;
  while ((1ll << b) < n) ++b;
  return b;
}

}  // namespace

int layer_mbrs(const LayerDev& L, double* mbr, cudaStream_t s) {
  if (L.n > 0) { mbr_only_kernel<<<blocks_for_warps(L.n), kThreads, 0, s>>>(L, mbr); note_launch(); }
  return ST_OK;
}

int run_join(const LayerDev& Lb0, const LayerDev& Lo0, Arena& A, JoinDev& J, int* d_err,
             int64_t* h_scratch, cudaStream_t s, Marks* mk, cudaStream_t aux, int f32, cudaEvent_t ovl_ready,
             int64_t cand_hint, int64_t list_hint_b, int64_t list_hint_o) {
  // f32 bit 0: FP32 prefilter of the sweep's y test; bit 1: of the common-MBR edge test
  // (needs the layers' vertex counts, for their FP32 copies)
  const bool f32cmf = (f32 & 2) && Lb0.nverts > 0 && Lo0.nverts > 0;
  const bool forceSweep = (f32 & 4) != 0;          // bit 2: the sort-sweep MBR filter, never the grid
  const int joinOpts = f32;                         // bit 3: the sweep's count and emit as two passes
  f32 &= 1;
  LayerDev Lb = Lb0, Lo = Lo0;
  Marks dummy;
  if (!mk) mk = &dummy;
  J = JoinDev();
  mk->mark("join:start", s);
  const int64_t nb = Lb.n, no = Lo.n;
  if (nb <= 0 || no <= 0) return ST_OK;
  // ---- J0 MBRs + sort keys
  J.mbr_b = A.take_n<double>(4 * nb); J.mbr_o = A.take_n<double>(4 * no);
  J.valid_b = A.take_n<uint8_t>(nb); J.valid_o = A.take_n<uint8_t>(no);
  uint64_t* keyB = A.take_n<uint64_t>(nb);
  uint64_t* keyO = A.take_n<uint64_t>(no);
  uint32_t* idB = A.take_n<uint32_t>(nb);
  uint32_t* idO = A.take_n<uint32_t>(no);
  uint64_t* kAlt = A.take_n<uint64_t>(nb);
  uint32_t* vAlt = A.take_n<uint32_t>(nb);
  uint64_t* kAltO = A.take_n<uint64_t>(no);
  uint32_t* vAltO = A.take_n<uint32_t>(no);
  unsigned long long* d_cnt = A.take_n<unsigned long long>(8);
  float2* xyfB = nullptr;
  float2* xyfO = nullptr;
  if (f32cmf) {
    xyfB = A.take_n<float2>(Lb.nverts);
    xyfO = A.take_n<float2>(Lo.nverts);
    if (!xyfB || !xyfO) return ST_OUT_OF_MEMORY;
    Lb.xyf = xyfB;
    Lo.xyf = xyfO;
  }
  void* tmp = A.take(std::max(radix_temp_bytes(nb), scan_temp_bytes(nb)));
  void* tmpO = A.take(std::max(radix_temp_bytes(no), scan_temp_bytes(no)));
  if (!J.mbr_b || !J.mbr_o || !J.valid_b || !J.valid_o || !keyB || !keyO || !idB || !idO || !kAlt ||
      !vAlt || !kAltO || !vAltO || !d_cnt || !tmp || !tmpO)
    return ST_OUT_OF_MEMORY;
  cudaMemsetAsync(d_cnt, 0, 8 * sizeof(unsigned long long), s);
  // The two layers' MBRs and sorts are independent and each fills under half of the GPU
  // (about 100 blocks per pass), so the overlay's run on the auxiliary stream.
  cudaStream_t so = s;
  cudaEvent_t fork = nullptr, join = nullptr;
  struct EvGuard { cudaEvent_t* a; cudaEvent_t* b; ~EvGuard() { if (*a) cudaEventDestroy(*a); if (*b) cudaEventDestroy(*b); } } evg{&fork, &join};
  if (aux && cudaEventCreateWithFlags(&fork, cudaEventDisableTiming) == cudaSuccess &&
      cudaEventCreateWithFlags(&join, cudaEventDisableTiming) == cudaSuccess) {
    cudaEventRecord(fork, s);
    cudaStreamWaitEvent(aux, fork, 0);
    so = aux;
  }
  { mbr_kernel<<<blocks_for_warps((nb + kMbrPerWarp - 1) / kMbrPerWarp), kThreads, 0, s>>>(Lb, J.mbr_b, J.valid_b, keyB, idB,
                                                                                       d_cnt + 0, xyfB); note_launch(); }
  // the overlay may still be on its way to the device (ovl_ready, recorded after its copy)
  if (ovl_ready) cudaStreamWaitEvent(so, ovl_ready, 0);
  { mbr_kernel<<<blocks_for_warps((no + kMbrPerWarp - 1) / kMbrPerWarp), kThreads, 0, so>>>(Lo, J.mbr_o, J.valid_o, keyO, idO,
                                                                                        d_cnt + 1, xyfO); note_launch(); }
  // the overlay's extent and mean box size, for the grid of the MBR filter
  constexpr int kExtentBlocks = 148;
  double* part = A.take_n<double>(7 * kExtentBlocks);
  if (!part) return ST_OUT_OF_MEMORY;
  if (!forceSweep) { mbr_extent_kernel<<<kExtentBlocks, kExtentThreads, 0, so>>>(J.mbr_o, J.valid_o, no, part); note_launch(); }
  if (so != s) {
    cudaEventRecord(join, so);
    cudaStreamWaitEvent(s, join, 0);
  }
  cudaMemcpyAsync(h_scratch, d_cnt, 2 * sizeof(int64_t), cudaMemcpyDeviceToHost, s);
  std::vector<double> hpart(7 * kExtentBlocks);
  if (!forceSweep) cudaMemcpyAsync(hpart.data(), part, hpart.size() * sizeof(double), cudaMemcpyDeviceToHost, s);
  if (cudaStreamSynchronize(s) != cudaSuccess) return ST_CUDA_ERROR;
  const int64_t nvb = h_scratch[0], nvo = h_scratch[1];
  const int obits = bits_for(no);
  const int bbits = bits_for(nb);
  if (obits + bbits > 64) return ST_INVALID_ARGUMENT;
  int64_t* d_total = A.take_n<int64_t>(4);
  if (!d_total) return ST_OUT_OF_MEMORY;
  // ---- J2 MBR filter as a grid probe (grid.cuh): the overlay's valid MBRs listed in the
  // cells of a uniform grid, every base polygon testing the entries of its cells.  The
  // sort-sweep below, the reference's own form, takes over when the listing would be
  // large (boxes spanning many cells).
  uint64_t* pkeys = nullptr;
  int64_t K = 0;
  bool swept = true;
  if (nvb > 0 && nvo > 0 && !forceSweep) {
    double ext[7] = {INFINITY, INFINITY, -INFINITY, -INFINITY, 0.0, 0.0, 0.0};
    for (int j = 0; j < kExtentBlocks; ++j) {
      const double* r = &hpart[7 * j];
      ext[0] = std::min(ext[0], r[0]); ext[1] = std::min(ext[1], r[1]);
      ext[2] = std::max(ext[2], r[2]); ext[3] = std::max(ext[3], r[3]);
      for (int k = 4; k < 7; ++k) ext[k] += r[k];
    }
    GridIndex G = grid_over(ext[0], ext[1], ext[2], ext[3], ext[4] / ext[6], ext[5] / ext[6]);
    const int64_t ncell = (int64_t)G.gx * G.gy;
    int32_t* cellCnt = A.take_n<int32_t>(ncell + 1);
    int64_t* cellOff = A.take_n<int64_t>(ncell + 1);
    void* ctmp = A.take(scan_temp_bytes(std::max<int64_t>(ncell + 1, nb)));
    if (!cellCnt || !cellOff || !ctmp) return ST_OUT_OF_MEMORY;
    cudaMemsetAsync(cellCnt, 0, (ncell + 1) * sizeof(int32_t), s);
    { index_kernel<0><<<blocks_for(no), kThreads, 0, s>>>(J.mbr_o, J.valid_o, no, G, cellCnt, nullptr, nullptr); note_launch(); }
    exclusive_scan_i32(cellCnt, cellOff, ncell + 1, d_total + 1, ctmp, d_err, s);
    cudaMemcpyAsync(h_scratch, d_total + 1, sizeof(int64_t), cudaMemcpyDeviceToHost, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) return ST_CUDA_ERROR;
    const int64_t nent = h_scratch[0];
    if (nent <= 8 * nvo + (1ll << 22)) {
      swept = false;
      int32_t* cellList = A.take_n<int32_t>(std::max<int64_t>(nent, 1));
      int32_t* cnt = A.take_n<int32_t>(nb);
      int64_t* offs = A.take_n<int64_t>(nb);
      if (!cellList || !cnt || !offs) return ST_OUT_OF_MEMORY;
      cudaMemsetAsync(cellCnt, 0, (ncell + 1) * sizeof(int32_t), s);
      { index_kernel<1><<<blocks_for(no), kThreads, 0, s>>>(J.mbr_o, J.valid_o, no, G, cellCnt, cellOff, cellList); note_launch(); }
      G.cellOff = cellOff;
      G.cellList = cellList;
      mk->mark("join:mbr+grid", s);
      { candidate_kernel<0><<<blocks_for_warps(nb), kThreads, 0, s>>>(J.mbr_b, J.valid_b, nb, J.mbr_o, G, cnt,
                                                                       nullptr, nullptr, obits); note_launch(); }
      exclusive_scan_i32(cnt, offs, nb, d_total, ctmp, d_err, s);
      mk->mark("join:cand-count", s);
      cudaMemcpyAsync(h_scratch, d_total, sizeof(int64_t), cudaMemcpyDeviceToHost, s);
      if (cudaStreamSynchronize(s) != cudaSuccess) return ST_CUDA_ERROR;
      K = h_scratch[0];
      J.n_pairs = K;
      if (K == 0) return ST_OK;
      pkeys = A.take_n<uint64_t>(K);
      uint32_t* pvals = A.take_n<uint32_t>(K);
      uint64_t* pkAlt = A.take_n<uint64_t>(K);
      uint32_t* pvAlt = A.take_n<uint32_t>(K);
      void* rtmp = A.take(radix_temp_bytes(K));
      if (!pkeys || !pvals || !pkAlt || !pvAlt || !rtmp) return ST_OUT_OF_MEMORY;
      { candidate_kernel<1><<<blocks_for_warps(nb), kThreads, 0, s>>>(J.mbr_b, J.valid_b, nb, J.mbr_o, G, nullptr,
                                                                       offs, pkeys, obits); note_launch(); }
      radix_sort_pairs(pkeys, pvals, pkAlt, pvAlt, K, ((obits + bbits + 7) / 8) * 8, rtmp, d_err, s);
      mk->mark("join:cand-emit+sort", s);
    }
  }
  if (swept) {
    SortedMbr SB{A.take_n<double>(nvb), A.take_n<double>(nvb), A.take_n<double>(nvb), A.take_n<double>(nvb),
                 A.take_n<uint32_t>(nvb), nvb, f32 ? A.take_n<float2>(nvb) : nullptr};
    SortedMbr SO{A.take_n<double>(nvo), A.take_n<double>(nvo), A.take_n<double>(nvo), A.take_n<double>(nvo),
                 A.take_n<uint32_t>(nvo), nvo, f32 ? A.take_n<float2>(nvo) : nullptr};
    if (f32 && (!SB.yf || !SO.yf)) return ST_OUT_OF_MEMORY;
    int32_t* cnt = A.take_n<int32_t>(nvb + nvo);
    int64_t* offs = A.take_n<int64_t>(nvb + nvo);
    const int64_t ne = nvb + nvo;
    void* stmp = A.take(scan_temp_bytes(std::max<int64_t>(ne, 1)));
    if (!SB.x1 || !SB.x2 || !SB.y1 || !SB.y2 || !SB.id || !SO.x1 || !SO.x2 || !SO.y1 || !SO.y2 ||
        !SO.id || !cnt || !offs || !stmp)
      return ST_OUT_OF_MEMORY;
    // Attempt 0 sorts the 32-bit keys of mbr_kernel and mends the runs of equal keys;
    // attempt 1, only for a layer with a run too long to mend, sorts the 64-bit keys.
    // One-pass sweep: the keys go straight into an array sized from the last join's
    // candidate count (with room to spare) or a first guess of 8 per polygon.
    const bool fusedSweep = !(joinOpts & 8);
    int64_t keyCap = 0;
    if (fusedSweep) {
      keyCap = cand_hint > 0 ? cand_hint + cand_hint / 4 + 65536 : 8 * ne + 65536;
      pkeys = A.take_n<uint64_t>(keyCap);
      if (!pkeys) return ST_OUT_OF_MEMORY;
    }
    bool redo[2] = {true, true};
    for (int attempt = 0; attempt < 2; ++attempt) {
      // ---- J1 sort both layers by x1 (stable: equal x1 keep ascending id)
      if (so != s) {                                  // the overlay's sort beside the base's
        cudaEventRecord(fork, s);
        cudaStreamWaitEvent(so, fork, 0);
      }
      for (int side = 0; side < 2; ++side) {
        if (!redo[side]) continue;
        cudaStream_t ss = side == 0 ? s : so;
        const int64_t n = side == 0 ? nb : no, nv = side == 0 ? nvb : nvo;
        uint64_t* key = side == 0 ? keyB : keyO;
        uint32_t* id = side == 0 ? idB : idO;
        const double* mbr = side == 0 ? J.mbr_b : J.mbr_o;
        if (attempt == 1)
          { x1_key64_kernel<<<blocks_for(n), kThreads, 0, ss>>>(mbr, side == 0 ? J.valid_b : J.valid_o, n, key, id); note_launch(); }
        radix_sort_pairs(key, id, side == 0 ? kAlt : kAltO, side == 0 ? vAlt : vAltO, n, attempt == 0 ? 32 : 64,
                         side == 0 ? tmp : tmpO, d_err, ss);
        if (attempt == 0 && nv > 1)
          { x1_fixup_kernel<<<blocks_for(nv), kThreads, 0, ss>>>(key, id, nv, mbr, d_cnt + 6 + side); note_launch(); }
      }
      if (so != s) {
        cudaEventRecord(join, so);
        cudaStreamWaitEvent(s, join, 0);
      }
      if (attempt == 0) mk->mark("join:mbr+sort", s);
      if (nvb) { gather_sorted_kernel<<<blocks_for(nvb), kThreads, 0, s>>>(J.mbr_b, idB, nvb, SB); note_launch(); }
      if (nvo) { gather_sorted_kernel<<<blocks_for(nvo), kThreads, 0, s>>>(J.mbr_o, idO, nvo, SO); note_launch(); }
      // ---- J2 sweep: count + emit in one pass (or count, scan, emit), then the canonical sort
      if (fusedSweep) {
        cudaMemsetAsync(d_total, 0, sizeof(int64_t), s);
        if (ne > 0)
          { (f32 ? sweep_append_kernel<1> : sweep_append_kernel<0>)<<<blocks_for_warps(ne), kThreads, 0, s>>>(
                SB, SO, pkeys, keyCap, reinterpret_cast<unsigned long long*>(d_total), obits); note_launch(); }
      } else if (ne > 0) {
        { (f32 ? sweep_kernel<0, 1> : sweep_kernel<0, 0>)<<<blocks_for_warps(ne), kThreads, 0, s>>>(SB, SO, cnt, nullptr,
                                                                                                 nullptr, obits); note_launch(); }
        exclusive_scan_i32(cnt, offs, ne, d_total, stmp, d_err, s);
      } else {
        cudaMemsetAsync(d_total, 0, sizeof(int64_t), s);
      }
      if (attempt == 0) mk->mark(fusedSweep ? "join:sweep" : "join:sweep-count", s);
      cudaMemcpyAsync(h_scratch, d_total, sizeof(int64_t), cudaMemcpyDeviceToHost, s);
      cudaMemcpyAsync(h_scratch + 1, d_cnt + 6, 2 * sizeof(int64_t), cudaMemcpyDeviceToHost, s);   // fix-up flags
      if (cudaStreamSynchronize(s) != cudaSuccess) return ST_CUDA_ERROR;
      redo[0] = h_scratch[1] != 0;
      redo[1] = h_scratch[2] != 0;
      if (!redo[0] && !redo[1]) break;
    }
    K = h_scratch[0];
    J.n_pairs = K;
    if (K == 0) return ST_OK;
    if (fusedSweep && K > keyCap) {               // the key array was short: again, at the counted size
      keyCap = K;
      pkeys = A.take_n<uint64_t>(K);
      if (!pkeys) return ST_OUT_OF_MEMORY;
      cudaMemsetAsync(d_total, 0, sizeof(int64_t), s);
      { (f32 ? sweep_append_kernel<1> : sweep_append_kernel<0>)<<<blocks_for_warps(ne), kThreads, 0, s>>>(
            SB, SO, pkeys, keyCap, reinterpret_cast<unsigned long long*>(d_total), obits); note_launch(); }
    }
    if (!fusedSweep) pkeys = A.take_n<uint64_t>(K);
    uint32_t* pvals = A.take_n<uint32_t>(K);
    uint64_t* pkAlt = A.take_n<uint64_t>(K);
    uint32_t* pvAlt = A.take_n<uint32_t>(K);
    void* rtmp = A.take(radix_temp_bytes(K));
    if (!pkeys || !pvals || !pkAlt || !pvAlt || !rtmp) return ST_OUT_OF_MEMORY;
    if (!fusedSweep)
      { (f32 ? sweep_kernel<1, 1> : sweep_kernel<1, 0>)<<<blocks_for_warps(ne), kThreads, 0, s>>>(SB, SO, nullptr, offs,
                                                                                               pkeys, obits); note_launch(); }
    radix_sort_pairs(pkeys, pvals, pkAlt, pvAlt, K, ((obits + bbits + 7) / 8) * 8, rtmp, d_err, s);
    mk->mark(fusedSweep ? "join:sort" : "join:sweep-emit+sort", s);
  }
  if (K == 0) return ST_OK;
  return join_from_keys(Lb, Lo, pkeys, K, obits, A, J, d_total, d_cnt, d_err, h_scratch, s, mk, aux, list_hint_b,
                        list_hint_o, (joinOpts & 8) != 0);
}

// Stages J3-J6 and the clip set over candidate pairs given as packed keys
// (b << obits | o) sorted ascending; J.mbr_b/J.mbr_o hold the layers' MBRs.  d_total
// (4 entries) and d_cnt (8 entries, zeroed) are device scratch counters.
// lanes per pair of the narrow-tile passes, and the pair size up to which they are used
constexpr int kJoinTile = 4;
constexpr int64_t kJoinTileMax = 64;

int join_from_keys(const LayerDev& Lb, const LayerDev& Lo, const uint64_t* pkeys, int64_t K, int obits,
                   Arena& A, JoinDev& J, int64_t* d_total, unsigned long long* d_cnt, int* d_err,
                   int64_t* h_scratch, cudaStream_t s, Marks* mk, cudaStream_t aux, int64_t hintB,
                   int64_t hintO, bool twoPass) {
  Marks dummy;
  if (!mk) mk = &dummy;
  J.n_pairs = K;
  if (K == 0) return ST_OK;
  // The narrow-tile and whole-warp passes of each stage take disjoint pairs (by size), so
  // with an auxiliary stream the warp pass, whose few large pairs make the tail, runs
  // beside the tile pass; both are joined back into s before the stage's results are used.
  cudaEvent_t ev[2] = {nullptr, nullptr};
  const bool two = aux && cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming) == cudaSuccess &&
                   cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming) == cudaSuccess;
  struct EvGuard { cudaEvent_t* e; ~EvGuard() { for (int i = 0; i < 2; ++i) if (e[i]) cudaEventDestroy(e[i]); } } guard{ev};
  cudaStream_t sw = two ? aux : s;
  auto fork_aux = [&]() { if (two) { cudaEventRecord(ev[0], s); cudaStreamWaitEvent(aux, ev[0], 0); } };
  auto join_aux = [&]() { if (two) { cudaEventRecord(ev[1], aux); cudaStreamWaitEvent(s, ev[1], 0); } };
  // ---- J3 CMBR + containment candidates
  J.b = A.take_n<int32_t>(K); J.o = A.take_n<int32_t>(K);
  J.cmbr = A.take_n<double>(4 * K);
  J.pip_type = A.take_n<int8_t>(K); J.pip_flag = A.take_n<int8_t>(K);
  J.join_flag = A.take_n<int8_t>(K); J.seg_flag = A.take_n<int8_t>(K); J.clip = A.take_n<int8_t>(K);
  J.bE = A.take_n<int32_t>(K); J.oE = A.take_n<int32_t>(K);
  int64_t* bOff = A.take_n<int64_t>(K);
  int64_t* oOff = A.take_n<int64_t>(K);
  uint8_t* clipU8 = A.take_n<uint8_t>(K);
  int64_t* clipOff = A.take_n<int64_t>(K);
  void* stmpK = A.take(scan_temp_bytes(K));
  if (!J.b || !J.o || !J.cmbr || !J.pip_type || !J.pip_flag || !J.join_flag || !J.seg_flag || !J.clip ||
      !J.bE || !J.oE || !bOff || !oOff || !clipU8 || !clipOff || !stmpK)
    return ST_OUT_OF_MEMORY;
  { cmbr_kernel<<<blocks_for(K), kThreads, 0, s>>>(pkeys, K, obits, J.mbr_b, J.mbr_o, J.b, J.o, J.cmbr,
                                                 J.pip_type); note_launch(); }
  // ---- J4 point in polygon
  // narrow tiles for small pairs first (they also set the flags of pairs with nothing to
  // test), then whole warps for the rest
  fork_aux();
  { pip_kernel<kJoinTile><<<blocks_for_tiles(K, kJoinTile), kThreads, 0, s>>>(
        Lb, Lo, J.b, J.o, J.pip_type, K, J.pip_flag, J.join_flag, -1, kJoinTileMax); note_launch(); }
  { pip_kernel<32><<<blocks_for_warps(K), kThreads, 0, sw>>>(Lb, Lo, J.b, J.o, J.pip_type, K, J.pip_flag,
                                                           J.join_flag, kJoinTileMax, INT64_MAX); note_launch(); }
  join_aux();
  mk->mark("join:cmbr+pip", s);
  // ---- J5 common-MBR edge filter: count, offsets, lists
  const bool f32 = Lb.xyf && Lo.xyf;
  int32_t* bList = nullptr;
  int32_t* oList = nullptr;
  if (twoPass) {
    fork_aux();
    { (f32 ? cmf_kernel<0, kJoinTile, 1> : cmf_kernel<0, kJoinTile, 0>)<<<blocks_for_tiles(K, kJoinTile), kThreads, 0, s>>>(
          Lb, Lo, J.b, J.o, J.cmbr, K, J.join_flag, J.bE, J.oE, nullptr, nullptr, nullptr, nullptr, -1,
          kJoinTileMax); note_launch(); }
    { (f32 ? cmf_kernel<0, 32, 1> : cmf_kernel<0, 32, 0>)<<<blocks_for_warps(K), kThreads, 0, sw>>>(Lb, Lo, J.b, J.o, J.cmbr, K, J.join_flag, J.bE,
                                                                J.oE, nullptr, nullptr, nullptr, nullptr, kJoinTileMax,
                                                                INT64_MAX); note_launch(); }
    join_aux();
    exclusive_scan_i32(J.bE, bOff, K, d_total + 1, stmpK, d_err, s);
    exclusive_scan_i32(J.oE, oOff, K, d_total + 2, stmpK, d_err, s);
    cudaMemcpyAsync(h_scratch, d_total + 1, 2 * sizeof(int64_t), cudaMemcpyDeviceToHost, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) return ST_CUDA_ERROR;
    const int64_t nBl = h_scratch[0], nOl = h_scratch[1];
    bList = A.take_n<int32_t>(nBl);
    oList = A.take_n<int32_t>(nOl);
    if (!bList || !oList) return ST_OUT_OF_MEMORY;
    J.n_blist = nBl; J.n_olist = nOl;
    fork_aux();
    { (f32 ? cmf_kernel<1, kJoinTile, 1> : cmf_kernel<1, kJoinTile, 0>)<<<blocks_for_tiles(K, kJoinTile), kThreads, 0, s>>>(
          Lb, Lo, J.b, J.o, J.cmbr, K, J.join_flag, J.bE, J.oE, bOff, oOff, bList, oList, -1, kJoinTileMax); note_launch(); }
    { (f32 ? cmf_kernel<1, 32, 1> : cmf_kernel<1, 32, 0>)<<<blocks_for_warps(K), kThreads, 0, sw>>>(Lb, Lo, J.b, J.o, J.cmbr, K, J.join_flag, J.bE,
                                                                J.oE, bOff, oOff, bList, oList, kJoinTileMax,
                                                                INT64_MAX); note_launch(); }
    join_aux();
  } else {
    // one pass (cmf_append_kernel) into lists sized from the last join's totals, or a
    // first guess of 8 edges per pair and side; again at the counted sizes on overflow
    CmfOut out{bOff, oOff, nullptr, nullptr, hintB > 0 ? hintB + hintB / 4 + 65536 : 8 * K + 65536,
               hintO > 0 ? hintO + hintO / 4 + 65536 : 8 * K + 65536,
               reinterpret_cast<unsigned long long*>(d_total + 1)};
    for (int attempt = 0; attempt < 2; ++attempt) {
      bList = A.take_n<int32_t>(out.bCap);
      oList = A.take_n<int32_t>(out.oCap);
      if (!bList || !oList) return ST_OUT_OF_MEMORY;
      out.bList = bList; out.oList = oList;
      cudaMemsetAsync(d_total + 1, 0, 2 * sizeof(int64_t), s);
      fork_aux();
      { (f32 ? cmf_append_kernel<kJoinTile, 1> : cmf_append_kernel<kJoinTile, 0>)<<<blocks_for_tiles(K, kJoinTile), kThreads, 0, s>>>(
            Lb, Lo, J.b, J.o, J.cmbr, K, J.join_flag, J.bE, J.oE, out, -1, kJoinTileMax); note_launch(); }
      { (f32 ? cmf_append_kernel<32, 1> : cmf_append_kernel<32, 0>)<<<blocks_for_warps(K), kThreads, 0, sw>>>(
            Lb, Lo, J.b, J.o, J.cmbr, K, J.join_flag, J.bE, J.oE, out, kJoinTileMax, INT64_MAX); note_launch(); }
      join_aux();
      cudaMemcpyAsync(h_scratch, d_total + 1, 2 * sizeof(int64_t), cudaMemcpyDeviceToHost, s);
      if (cudaStreamSynchronize(s) != cudaSuccess) return ST_CUDA_ERROR;
      J.n_blist = h_scratch[0]; J.n_olist = h_scratch[1];
      if (J.n_blist <= out.bCap && J.n_olist <= out.oCap) break;
      out.bCap = std::max<int64_t>(J.n_blist, 1);
      out.oCap = std::max<int64_t>(J.n_olist, 1);
    }
  }
  mk->mark("join:cmf", s);
  // ---- J6 refine
  fork_aux();
  { refine_kernel<kJoinTile><<<blocks_for_tiles(K, kJoinTile), kThreads, 0, s>>>(
        Lb, Lo, J.b, J.o, K, J.join_flag, J.bE, J.oE, bOff, oOff, bList, oList, J.seg_flag, -1,
        kJoinTileMax * 4); note_launch(); }
  { refine_kernel<32><<<blocks_for_warps(K), kThreads, 0, sw>>>(Lb, Lo, J.b, J.o, K, J.join_flag, J.bE, J.oE,
                                                              bOff, oOff, bList, oList, J.seg_flag, kJoinTileMax * 4,
                                                              INT64_MAX); note_launch(); }
  join_aux();
  mk->mark("join:refine", s);
  // ---- clip set = containment pairs + pairs with intersecting edges
  { clip_flag_kernel<<<blocks_for(K), kThreads, 0, s>>>(J.pip_type, J.pip_flag, J.join_flag, J.seg_flag, K,
                                                      J.clip, clipU8, d_cnt + 2); note_launch(); }
  exclusive_scan_u8(clipU8, clipOff, K, d_total + 3, stmpK, d_err, s);
  cudaMemcpyAsync(h_scratch, d_total + 3, sizeof(int64_t), cudaMemcpyDeviceToHost, s);
  cudaMemcpyAsync(h_scratch + 1, d_cnt + 2, 4 * sizeof(int64_t), cudaMemcpyDeviceToHost, s);
  if (cudaStreamSynchronize(s) != cudaSuccess) return ST_CUDA_ERROR;
  J.n_clip = h_scratch[0];
  J.n_pip_candidates = h_scratch[1];
  J.n_within = h_scratch[2];
  J.n_cmf = h_scratch[3];
  J.n_seg = h_scratch[4];
  J.clip_b = A.take_n<int32_t>(J.n_clip);
  J.clip_o = A.take_n<int32_t>(J.n_clip);
  J.clip_cand = A.take_n<int64_t>(J.n_clip);
  if (!J.clip_b || !J.clip_o || !J.clip_cand) return ST_OUT_OF_MEMORY;
  { clip_compact_kernel<<<blocks_for(K), kThreads, 0, s>>>(J.clip, clipOff, J.b, J.o, K, J.clip_b, J.clip_o,
                                                         J.clip_cand); note_launch(); }
  J.bOff = bOff; J.oOff = oOff; J.bList = bList; J.oList = oList;
  mk->mark("join:clipset", s);
  return ST_OK;
}

}  // namespace gcmfgh
