// engine.cuh -- host-side plumbing shared by the join and clip pipelines: the device
// workspace arena, layer views and the result records the C ABI hands out.
#pragma once
#include <cstdint>
#include <cstddef>
#include <vector>
#include <cuda_runtime.h>

namespace gcmfgh {

// Status codes of the C ABI (mirrored in include/gcmfgh.h).
enum Status : int {
  ST_OK = 0,
  ST_INVALID_ARGUMENT = 1,
  ST_CUDA_ERROR = 2,
  ST_OUT_OF_MEMORY = 3,
  ST_DEVICE_ERROR = 4,     // a kernel raised its error word (capacity, trace budget, timeout)
  ST_NOT_READY = 5,
  ST_CAPACITY = 6,         // caller buffer too small (two-call size query)
  ST_NO_DEVICE = 7,
};

// Bump allocator over device chunks.  Chunks are kept across calls and reused after
// reset(); a request goes to the first chunk with room, else opens a new chunk
// (cudaMalloc), so pointers handed out since the last reset() stay valid.
class Arena {
 public:
  ~Arena() { release(); }
  void reset() { for (auto& c : chunks_) c.off = 0; }
  void* take(size_t bytes);           // nullptr on allocation failure
  template <class T> T* take_n(int64_t n) { return static_cast<T*>(take(sizeof(T) * (size_t)(n > 0 ? n : 1))); }
  void release();
  size_t reserved() const { size_t s = 0; for (auto& c : chunks_) s += c.cap; return s; }
 private:
  struct Chunk { char* base; size_t cap; size_t off; };
  std::vector<Chunk> chunks_;
};

// A polygon layer in the reference's join layout, device pointers:
// coords interleaved x,y with each polygon's closing vertex stored (spatialJoin3.cu:211),
// vnum = vertices per polygon including the closing one, vps = inclusive prefix of vnum.
struct LayerDev {
  const double* xy;
  const int32_t* vnum;
  const int64_t* vps;
  int64_t n;
  int64_t nverts = 0;          // stored vertices (0: unknown)
  const float2* xyf = nullptr; // FP32 copy of xy (round to nearest) for the join's prefilters
};

// Join outputs (device, owned by the join arena).  Pairs are sorted by (base, overlay).
struct JoinDev {
  int64_t n_pairs = 0, n_pip_candidates = 0, n_within = 0, n_cmf = 0, n_seg = 0, n_clip = 0;
  int32_t* b = nullptr;          // [n_pairs]
  int32_t* o = nullptr;
  double* cmbr = nullptr;        // [4 n_pairs]
  int8_t* pip_type = nullptr;    // 0 none, 1 overlay may contain base, 2 base may contain overlay
  int8_t* pip_flag = nullptr;    // containment confirmed
  int8_t* join_flag = nullptr;   // survived the common-MBR edge filter
  int32_t* bE = nullptr;         // edges touching the common MBR (0 when filtered out)
  int32_t* oE = nullptr;
  int8_t* seg_flag = nullptr;    // some surviving edge pair intersects
  int8_t* clip = nullptr;        // pip_flag || seg_flag
  int32_t* clip_b = nullptr;     // [n_clip] the clip set, same order
  int32_t* clip_o = nullptr;
  double* mbr_b = nullptr;       // [4 nb] layer MBRs
  double* mbr_o = nullptr;
  uint8_t* valid_b = nullptr;
  uint8_t* valid_o = nullptr;
  int64_t* clip_cand = nullptr;  // [n_clip] each clip pair's candidate index
  int64_t* bOff = nullptr;       // [n_pairs] first entry of each candidate's edge lists
  int64_t* oOff = nullptr;
  int32_t* bList = nullptr;      // edges of the common-MBR filter (join_flag pairs), ascending
  int32_t* oList = nullptr;
  int64_t n_blist = 0, n_olist = 0;   // list entries (the next join's capacity hints)
};

// The join's common-MBR edge lists seen from its clip set (gh_clip_joined): the clip's
// edge filter (G1) takes a pair's lists from here instead of testing every edge again.
struct JoinEdges {
  const int64_t* cand = nullptr;   // per clip pair: candidate index (null: no lists)
  const int8_t* flag = nullptr;    // per candidate: lists present (join_flag)
  const int32_t* bE = nullptr;
  const int32_t* oE = nullptr;
  const int64_t* bOff = nullptr;
  const int64_t* oOff = nullptr;
  const int32_t* bList = nullptr;
  const int32_t* oList = nullptr;
};

// Clip parameters (reference defaults: EPSILON 1e-7 in GH-CUDA/lib/constants.h:4).
struct ClipParams {
  double eps = 1e-7;          // intersection classification
  double eps_clean = 1e-7;    // collinear-vertex removal in the clean-up
  int union_mode = 0;         // polyclip.h:42 UNION
  int no_swap = 0;            // 1: clip base as P even when it has fewer vertices
  int exact = 0;              // 1: exact orientation/classification signs (eps unused there)
  int64_t bin_grid = 1ll << 16;        // edge-pair grid above which a pair's edges are binned
  int64_t tile_label_max = 96;         // merged-ring slots up to which one thread labels a pair
  int64_t wide_label_min = 1 << 16;    // clip batches of at least this many pairs use the
                                       // high-occupancy labelling kernels
  int64_t mid_label_min = 1ll << 10;   // merged-ring slots above which a block labels a pair
  int64_t big_label_min = 1ll << 18;   // merged-ring slots above which a pair is labelled grid-wide
  int fused_emit = 1;                  // count and emit the intersection records in one pass
  int64_t rec_hint = 0;                // records expected (the last clip's count; 0 unknown)
};

// Clip outputs (device, owned by the clip arena).
struct ClipDev {
  int64_t n_pairs = 0, n_components = 0, n_vertices = 0;
  int64_t n_records = 0;          // intersection records (all pairs)
  int64_t n_ring_vertices = 0;    // merged-ring vertices, P and Q sides (valid pairs)
  int32_t* status = nullptr;      // per pair: 0 ok, 1 invalid (P/Q counts differ), 2 disjoint MBRs, 3 trace error
  int32_t* ncomp = nullptr;       // per pair
  int64_t* comp_off = nullptr;    // per pair, first component index
  int64_t* count1 = nullptr;      // per pair, edge pairs classified as intersecting (P side)
  int32_t* comp_size = nullptr;   // per component vertex count
  int64_t* vert_off = nullptr;    // per pair, first vertex
  double* xy = nullptr;           // [2 n_vertices]
  int32_t* swapped = nullptr;     // per pair: 1 when the overlay polygon was P
};

// Optional stage timing: an event is recorded on the launching stream at each mark, so
// the time between consecutive marks is the device time of the stage in between.
struct Marks {
  static constexpr int kMax = 24;
  cudaEvent_t ev[kMax] = {};
  const char* name[kMax] = {};
  int n = 0;
  bool on = false;
  void mark(const char* label, cudaStream_t s) {
    if (!on || n >= kMax) return;
    name[n] = label;
    cudaEventRecord(ev[n++], s);
  }
};

int layer_mbrs(const LayerDev& L, double* mbr, cudaStream_t s);

// aux: optional second stream; the overlay layer's MBRs and sort run on it, beside the
// base layer's on s.
int run_join(const LayerDev& base, const LayerDev& ovl, Arena& arena, JoinDev& out,
             int* d_err, int64_t* h_scratch, cudaStream_t s, Marks* marks = nullptr,
             cudaStream_t aux = nullptr, int f32 = 0, cudaEvent_t ovl_ready = nullptr,
             int64_t cand_hint = 0, int64_t list_hint_b = 0, int64_t list_hint_o = 0);

int join_from_keys(const LayerDev& Lb, const LayerDev& Lo, const uint64_t* pkeys, int64_t K, int obits,
                   Arena& A, JoinDev& J, int64_t* d_total, unsigned long long* d_cnt, int* d_err,
                   int64_t* h_scratch, cudaStream_t s, Marks* marks = nullptr,
                   cudaStream_t aux = nullptr, int64_t hintB = 0, int64_t hintO = 0, bool twoPass = false);

// Merged rings of pair 0 after the neighbour links, as the reference's
// calculateIntersections hands them back (gppolyclip_mDIV512.cu:1298-1640): vertices in
// ring order, the integer parameter key (int)(1e7 * alpha) of every vertex that carries an
// intersection (-100 at plain vertices), the initial label (-100 where no key), and the
// 1-based slot of the neighbour in the other ring (0 = none).
//
// With records_only set, the clip instead stops after the emit stage (G3) and hands back
// the device arrays of every pair's intersection records, valid until the arena is reset.
struct RingExport {
  bool records_only = false;
  int64_t n_records = 0;
  const int32_t* rec_p = nullptr;    // pair-local P edge
  const int32_t* rec_q = nullptr;    // pair-local Q edge
  const double* rec_a = nullptr;     // alpha (on P)
  const double* rec_b = nullptr;     // beta (on Q)
  const int8_t* rec_t = nullptr;     // intersection type 1..8
  const int32_t* rec_k = nullptr;    // pair
  int status = 0;                    // pair status: 0 ok, 1 invalid, 2 disjoint MBRs
  int64_t n_p = 0, n_q = 0;          // merged ring sizes
  int64_t edges_p = 0, edges_q = 0;  // ring edges (vertices without the closing one)
  std::vector<double> xy_p, xy_q;
  std::vector<int32_t> alpha_p, alpha_q, label_p, label_q, nb_p, nb_q;
};

// aux: optional second stream (ideally of higher priority); long pairs are labelled on it
// while the warp-per-pair kernel runs on s.  Without it everything runs on s.
// aux2: optional third stream; the warp-per-pair labelling runs on it beside the one-thread
// labelling on s.
// mbrB / mbrO: the layers' polygon MBRs when the caller already has them (the join
// computes the same ones), else they are computed here.
// ex: when given, the clip stops after the neighbour links and pair 0's merged rings are
// exported into it instead of being labelled and traced.
int run_clip(const LayerDev& base, const LayerDev& ovl, const int32_t* d_pid, const int32_t* d_qid,
             int64_t n_pairs, const ClipParams& prm, Arena& arena, ClipDev& out,
             int* d_err, int64_t* h_scratch, cudaStream_t s, Marks* marks = nullptr,
             cudaStream_t aux = nullptr, RingExport* ex = nullptr, cudaStream_t aux2 = nullptr,
             const double* mbrB = nullptr, const double* mbrO = nullptr, const JoinEdges* je = nullptr);

// One pair of multi-component polygons (rings: host, interleaved, open; ring c has
// sizes[c] >= 3 vertices), P clipped against Q as given.  Result as one pair of ClipDev.
int run_clip_multi(const double* P, const int32_t* sizesP, int kP, const double* Q, const int32_t* sizesQ, int kQ,
                   const ClipParams& prm, Arena& arena, ClipDev& out, int* d_err, int64_t* h_scratch,
                   cudaStream_t s);
// n pairs of multi-component polygons in one batch: pair i's P has ringsP[i] rings, taken
// in order from sizesP / P (all pairs' rings one after the other), and the same for Q.
// Results as n pairs of ClipDev (one thread per pair runs the phases after the records).
int run_clip_multi_batch(int64_t n, const double* P, const int32_t* sizesP, const int32_t* ringsP,
                         const double* Q, const int32_t* sizesQ, const int32_t* ringsQ, const ClipParams& prm,
                         Arena& arena, ClipDev& out, int* d_err, int64_t* h_scratch, cudaStream_t s);

// a non-blocking stream at the device's highest priority (nullptr on failure)
cudaStream_t create_priority_stream();

}  // namespace gcmfgh
