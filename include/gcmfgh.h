/*
 * gcmfgh.h -- C ABI of the B200 spatial-join-and-clip engine (libgcmfgh.so).
 *
 * The engine replaces the hot path of the GCMF-GH reference: the GCMF join driver
 * behind main.cpp (spatialJoin, main.h:5-7, spatialJoin3.cu:40-412) and the GH-CUDA
 * clip call (ghcuda, main.h:8-11, GH-CUDA/ghcuda.cpp:385-425, with its inner
 * calculateIntersections, GH-CUDA/ghcuda.h:6-14).  The reference exports those three
 * with C++ linkage and no status returns; the C entry points below carry the same data
 * in plain pointers and sizes, return a status code, and never exit the process.
 * gcmfgh_shims.h declares C++ functions with the reference's exact signatures.
 *
 * Layer layout (the reference's, spatialJoin3.cu:205-212 and SEQ_Overlay.h:352-380):
 *   coords  interleaved FP64 x,y; each polygon stores its closing vertex (a copy of its
 *           first vertex) after its last one; 16-byte aligned
 *   vnum    per polygon, vertex count including the closing vertex (bVNum)
 *   vps     per polygon, inclusive prefix sum of vnum (bVPSNum)
 * Polygon i occupies vertices [vps[i]-vnum[i], vps[i]).
 *
 * Unless a function says otherwise, layer and pair pointers are device pointers on the
 * context's device, and every call is ordered on the context's stream and returns when
 * its results are ready.  Results stay owned by the context and are valid until the
 * next call of the same kind (join or clip); the *_get functions copy them out.
 */
#ifndef GCMFGH_H
#define GCMFGH_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  GCMFGH_OK = 0,
  GCMFGH_INVALID_ARGUMENT = 1,
  GCMFGH_CUDA_ERROR = 2,
  GCMFGH_OUT_OF_MEMORY = 3,
  GCMFGH_DEVICE_ERROR = 4,   /* a kernel reported a capacity, trace-budget or wait-limit error */
  GCMFGH_NOT_READY = 5,      /* no result of that kind yet */
  GCMFGH_CAPACITY = 6,       /* destination smaller than the result (size query first) */
  GCMFGH_NO_DEVICE = 7
} gcmfgh_status;

typedef struct gcmfgh_ctx gcmfgh_ctx;

typedef struct {
  const double* coords;
  const int32_t* vnum;
  const int64_t* vps;
  int64_t n_polys;
  int64_t n_vertices; /* = vps[n_polys-1]; needed for host-resident layers */
} gcmfgh_layer;

/* Counts of one join (spatialJoin3.cu:256-363 prints the same stages). */
typedef struct {
  int64_t n_pairs;          /* MBR candidates (SortBaseMBROverlap, Join.h:5) */
  int64_t n_pip_candidates; /* one MBR equals the common MBR (GetCMBR, Join.h:397) */
  int64_t n_within;         /* containment confirmed (PointInPolygonTest, Join.h:437) */
  int64_t n_cmf;            /* survived the common-MBR edge filter (CountCMF, Join.h:157) */
  int64_t n_seg;            /* some edge pair intersects (SegmentIntersectJoin, Join.h:356) */
  int64_t n_clip;           /* clip set = n_within + n_seg pairs */
} gcmfgh_join_info;

typedef struct {
  int64_t n_pairs;
  int64_t n_components;
  int64_t n_vertices;
  int64_t n_invalid;        /* P/Q intersection counts disagree (gppolyclip_mDIV512.cu:1461) */
  int64_t n_disjoint;       /* MBRs do not overlap (ghcuda.cpp:109-116 exits instead) */
  int64_t n_error;          /* tracing did not close within its step budget */
  int64_t n_records;        /* intersecting edge pairs found (all pairs) */
  int64_t n_ring_vertices;  /* vertices of the merged P and Q rings (valid pairs) */
} gcmfgh_clip_info;

/* Join result fields for gcmf_join_get / gcmf_join_ptr. */
typedef enum {
  GCMF_PAIR_BASE = 0,    /* int32 [n_pairs], pairs sorted by (base, overlay) */
  GCMF_PAIR_OVERLAY,     /* int32 [n_pairs] */
  GCMF_CMBR,             /* f64 [4 n_pairs] minx, miny, maxx, maxy */
  GCMF_PIP_TYPE,         /* int8 [n_pairs]: 1 overlay may contain base, 2 base may contain overlay */
  GCMF_PIP_FLAG,         /* int8 [n_pairs] */
  GCMF_JOIN_FLAG,        /* int8 [n_pairs] */
  GCMF_BASE_EDGES,       /* int32 [n_pairs] base edges touching the common MBR */
  GCMF_OVERLAY_EDGES,    /* int32 [n_pairs] */
  GCMF_SEG_FLAG,         /* int8 [n_pairs] */
  GCMF_CLIP_FLAG,        /* int8 [n_pairs] */
  GCMF_CLIP_BASE,        /* int32 [n_clip] */
  GCMF_CLIP_OVERLAY,     /* int32 [n_clip] */
  GCMF_MBR_BASE,         /* f64 [4 n_base] */
  GCMF_MBR_OVERLAY,      /* f64 [4 n_overlay] */
  GCMF_VALID_BASE,       /* uint8 [n_base] nonzero-area MBR */
  GCMF_VALID_OVERLAY     /* uint8 [n_overlay] */
} gcmf_join_field;

/* Clip result fields for gh_clip_get / gh_clip_ptr. */
typedef enum {
  GH_STATUS = 0,         /* int32 [n_pairs]: 0 ok, 1 invalid, 2 disjoint, 3 trace error */
  GH_NCOMP,              /* int32 [n_pairs] result components per pair */
  GH_COMP_OFFSET,        /* int64 [n_pairs] first component of each pair */
  GH_COUNT1,             /* int64 [n_pairs] intersecting edge pairs (psP1 total) */
  GH_COMP_SIZE,          /* int32 [n_components] vertices per component */
  GH_VERT_OFFSET,        /* int64 [n_pairs] first vertex of each pair */
  GH_XY,                 /* f64 [2 n_vertices] component vertices, interleaved */
  GH_SWAPPED             /* int32 [n_pairs] 1 when the overlay polygon was clipped as P */
} gh_clip_field;

/* ---- context */
gcmfgh_status gcmfgh_create(int device, gcmfgh_ctx** out);
gcmfgh_status gcmfgh_destroy(gcmfgh_ctx* ctx);
/* cudaStream_t as void*; NULL = the context's own stream */
gcmfgh_status gcmfgh_set_stream(gcmfgh_ctx* ctx, void* stream);
/* eps: classification tolerance (GH-CUDA/lib/constants.h:4, 1e-7); eps_clean: clean-up
 * tolerance (polyclip.h:795; 1e-12 where Constants.h:29 overrides it in the merged
 * build); union_mode: polyclip.h:42 UNION. */
gcmfgh_status gcmfgh_set_params(gcmfgh_ctx* ctx, double eps, double eps_clean, int union_mode);
/* Predicate precision of the clip.  GCMFGH_PRECISION_REFERENCE (default): FP64 values
 * compared against eps, as gppolyclip_mDIV512.cu:95-169 and polyclip.h:297-326 do.
 * GCMFGH_PRECISION_EXACT: every orientation/order sign of the classification, labelling,
 * inside tests and split rule is exact (error-bounded FP64 filter, exact expansion
 * arithmetic when the filter cannot decide); eps is unused there, eps_clean still sets
 * the clean-up tolerance.  In exact mode P-side and Q-side counts agree by construction,
 * so no pair is invalid. */
#define GCMFGH_PRECISION_REFERENCE 0
#define GCMFGH_PRECISION_EXACT 1
gcmfgh_status gcmfgh_set_precision(gcmfgh_ctx* ctx, int mode);
const char* gcmfgh_status_string(gcmfgh_status s);
/* Work-distribution thresholds of the clip (results do not depend on them):
 * GCMFGH_TUNE_BIN_GRID: a pair whose common-MBR edge grid exceeds this many edge pairs
 * has its edges binned on a uniform grid instead of enumerated (default 2^16);
 * GCMFGH_TUNE_MID_LABEL: a pair whose merged rings exceed this many vertices is labelled
 * and traced by one thread block (persistent, work-stealing) instead of one warp
 * (default 2^10);
 * GCMFGH_TUNE_BIG_LABEL: a pair whose merged rings exceed this many vertices is labelled
 * and traced by grid-wide kernels (default 2^18). */
#define GCMFGH_TUNE_BIN_GRID 0
#define GCMFGH_TUNE_BIG_LABEL 1
#define GCMFGH_TUNE_MID_LABEL 2
/* GCMFGH_TUNE_TILE_LABEL: a pair whose merged rings have at most this many vertices is
 * labelled and traced by one thread, 32 pairs per warp (default 96; 0: never) */
#define GCMFGH_TUNE_TILE_LABEL 3
/* GCMFGH_TUNE_WIDE_LABEL: clip batches of at least this many pairs are labelled by the
 * kernels built for a full GPU (fewer registers, more resident warps); smaller batches
 * by the ones built for per-pair latency (default 65536) */
#define GCMFGH_TUNE_WIDE_LABEL 4
/* GCMFGH_TUNE_F32_FILTER: bit 0 runs the join's MBR y test (GPU_MBR.h:339-415) first on
 * outward-rounded FP32 boxes, bit 1 the common-MBR edge test (GPU_Join.h:576-577) first
 * on FP32 vertex copies with one ulp of room; both are guaranteed supersets, and the
 * survivors are confirmed in FP64, so candidates and edge lists are those of the FP64
 * tests.  Default 1: on the batched workload the MBR prefilter saves 0.03 ms and the
 * edge prefilter costs 0.24 ms (most edges pass it and are tested twice).  Bit 1 needs
 * the layers' n_vertices. */
#define GCMFGH_TUNE_F32_FILTER 5
/* GCMFGH_TUNE_FUSED_EMIT: 1 (default) classifies the candidate edge pairs once and writes
 * the intersection records in the same pass (the reference counts with
 * gpuCountIntersections, gppolyclip_mDIV512.cu:1389-1420, and classifies again to write,
 * :1567); 0 runs a count pass and an emit pass.  The results are the same. */
#define GCMFGH_TUNE_FUSED_EMIT 6
/* GCMFGH_TUNE_RECORD_HINT: intersection records the next clips should expect (the fused
 * pass sizes its record arrays from it and runs again, at the counted size, when a clip
 * finds more).  0 (default): the last clip's count. */
#define GCMFGH_TUNE_RECORD_HINT 7
/* GCMFGH_TUNE_JOIN_SWEEP: 1 (default) finds the MBR candidates with the reference's
 * sort-sweep on x (GPU_MBR.h:339-539); 0 with a grid probe (the overlay's boxes listed in a
 * uniform grid, each base box testing the entries of the cells it covers), which falls
 * back to the sweep when boxes span so many cells that the listing would be large.  Both
 * give the same candidates.  The FP32 prefilter bit 0 of GCMFGH_TUNE_F32_FILTER applies
 * to the sweep only.  On the batched star workload the sweep measured faster (1.54 ms
 * against 1.78 ms for the MBR stages). */
#define GCMFGH_TUNE_JOIN_SWEEP 8
/* GCMFGH_TUNE_SWEEP_TWO_PASS: 1 runs the join's MBR sweep and common-MBR edge filter as
 * the reference does, a counting pass and then a writing pass (GPU_MBR.h:420-539,
 * Join.h:157-287); 0 (default) runs each as one pass that writes what it finds into arrays
 * sized from the last join's totals (again, at the counted sizes, when a join finds
 * more).  Candidates, flags, counts and edge lists are the same. */
#define GCMFGH_TUNE_SWEEP_TWO_PASS 9
gcmfgh_status gcmfgh_set_tuning(gcmfgh_ctx* ctx, int key, int64_t value);

/* ---- autotuner of the work-distribution thresholds.  No counterpart in the reference
 * (its block sizes are picked per dataset by hand: switch (DATASET) at Join.h:112, 185,
 * 262, 363, 442).
 * A workload's signature is (GPU name, floor(log2 pairs), floor(log2 mean vertices per
 * polygon of the two layers), precision mode).  gcmfgh_autotune_joined times
 * gh_clip_joined on the last join's clip set under candidate thresholds (one pass of
 * coordinate descent over bin grid, tile, block and wide-batch limits; median of three
 * runs each), keeps the fastest, and records it for the signature.  Later clips of the
 * context whose signature matches use the recorded thresholds, unless gcmfgh_set_tuning
 * was called (explicit settings win).  When the environment variable
 * GCMFGH_TUNING_FILE names a file, gcmfgh_create loads the records from it (JSON, one
 * object per line) and gcmfgh_autotune_joined writes them back.  Results do not depend on
 * the thresholds: only the time does. */
typedef struct {
  int64_t bin_grid, tile_label, mid_label, big_label, wide_label;
  int pairs_log2, verts_log2, exact;
  double ms_default;     /* clip time under the thresholds in force before tuning */
  double ms_tuned;       /* clip time under the chosen thresholds */
  int configs_timed;
} gcmfgh_tuning;
gcmfgh_status gcmfgh_autotune_joined(gcmfgh_ctx* ctx, const gcmfgh_layer* base, const gcmfgh_layer* overlay,
                                     gcmfgh_tuning* out);
/* the thresholds a clip of n_pairs on these layers would use now (recorded or default) */
gcmfgh_status gcmfgh_tuning_for(gcmfgh_ctx* ctx, const gcmfgh_layer* base, const gcmfgh_layer* overlay,
                                int64_t n_pairs, gcmfgh_tuning* out);
/* device error word of the last call (0 none, 1 capacity, 2 trace budget, 4 wait limit) */
int gcmfgh_last_device_error(gcmfgh_ctx* ctx);
/* Stage timing, replacing the reference's StartTimer/StopTimer pairs around each stage
 * (GPU_Manage.h:4-19, spatialJoin3.cu:197-375) and its DEBUG_TIMING kernel events
 * (gppolyclip_mDIV512.cu:1319-1669): when on, CUDA events are recorded on the stream
 * between stages.  gcmfgh_get_timing(which = 0 join, 1 clip) fills ms[i] / names[i]
 * (stage ending at mark i+1) for the last call and returns the number of stages. */
gcmfgh_status gcmfgh_set_timing(gcmfgh_ctx* ctx, int on);
int gcmfgh_get_timing(gcmfgh_ctx* ctx, int which, float* ms, const char** names, int cap);
/* number of kernels this library has launched in the process so far */
unsigned long long gcmfgh_launch_count(void);

/* ---- join: replaces the stage sequence of spatialJoin (spatialJoin3.cu:197-363) */
gcmfgh_status gcmf_join(gcmfgh_ctx* ctx, const gcmfgh_layer* base, const gcmfgh_layer* overlay,
                        gcmfgh_join_info* info);
/* copy a join field to dst (host if dst_on_device == 0); cap = dst size in bytes;
 * *bytes receives the field's size (size query: dst NULL) */
gcmfgh_status gcmf_join_get(gcmfgh_ctx* ctx, int field, void* dst, int64_t cap, int dst_on_device,
                            int64_t* bytes);
gcmfgh_status gcmf_join_ptr(gcmfgh_ctx* ctx, int field, const void** dev_ptr, int64_t* count);

/* ---- clip: replaces ghcuda (ghcuda.cpp:385) for a whole batch of pairs.
 * pid/qid: device int32 [n_pairs] base / overlay polygon ids. */
gcmfgh_status gh_clip_batch(gcmfgh_ctx* ctx, const gcmfgh_layer* base, const gcmfgh_layer* overlay,
                            const int32_t* pid, const int32_t* qid, int64_t n_pairs,
                            gcmfgh_clip_info* info);
/* as gh_clip_batch with the pair ids in HOST memory (copied in) */
gcmfgh_status gh_clip_batch_host_ids(gcmfgh_ctx* ctx, const gcmfgh_layer* base, const gcmfgh_layer* overlay,
                                     const int32_t* pid, const int32_t* qid, int64_t n_pairs,
                                     gcmfgh_clip_info* info);
/* clip the clip set of the last gcmf_join on the same layers (no host round trip) */
gcmfgh_status gh_clip_joined(gcmfgh_ctx* ctx, const gcmfgh_layer* base, const gcmfgh_layer* overlay,
                             gcmfgh_clip_info* info);
gcmfgh_status gh_clip_get(gcmfgh_ctx* ctx, int field, void* dst, int64_t cap, int dst_on_device,
                          int64_t* bytes);
gcmfgh_status gh_clip_ptr(gcmfgh_ctx* ctx, int field, const void** dev_ptr, int64_t* count);

/* ---- one pair: replaces the per-pair GH_CUDA (ghcuda.cpp:341).  P, Q: host open rings
 * (no closing vertex) of nP, nQ vertices; P is clipped against Q as given (no swap). */
gcmfgh_status gh_clip_pair(gcmfgh_ctx* ctx, const double* P, int32_t nP, const double* Q, int32_t nQ,
                           gcmfgh_clip_info* info);

/* ---- one pair of multi-component polygons (outer rings and holes, even-odd; the
 * reference's CPU clipper over component lists, GH-CUDA/lib/polyclip.h, whose GPU form
 * calculateIntersectionsMultipleComponents is declared in ghcuda.h:15 and never defined).
 * P, Q: host rings, interleaved and open (no closing vertex), ring c of p_sizes[c] (or
 * q_sizes[c]) >= 3 vertices, one after the other.  P is clipped against Q as given.
 * Every (P ring, Q ring) pair gets the GPU path's filters and P/Q count check; one failing
 * ring pair makes the pair invalid (status 1).  The result is read like one pair of
 * gh_clip_batch (gh_clip_get / gh_clip_ptr). */
gcmfgh_status gh_clip_multi(gcmfgh_ctx* ctx, const double* P, const int32_t* p_sizes, int32_t p_rings,
                            const double* Q, const int32_t* q_sizes, int32_t q_rings, gcmfgh_clip_info* info);
/* ---- n_pairs such pairs in one batch.  Pair i's P has p_rings[i] rings, taken in order
 * from p_sizes / P (every pair's rings one after the other), and the same for Q.  The
 * intersection records of all ring pairs come from one run of the batched stages; the
 * labelling and tracing run one GPU thread per pair.  Read the result like gh_clip_batch's. */
gcmfgh_status gh_clip_multi_batch(gcmfgh_ctx* ctx, int64_t n_pairs, const double* P, const int32_t* p_sizes,
                                  const int32_t* p_rings, const double* Q, const int32_t* q_sizes,
                                  const int32_t* q_rings, gcmfgh_clip_info* info);

/* ---- the intersection phase of one pair: replaces calculateIntersections
 * (ghcuda.h:6-14, gppolyclip_mDIV512.cu:1298-1640), which hands the merged rings to the
 * host list builder (ghcuda.cpp:239-322).  Arrays are host malloc'ed, freed by
 * gh_free_intersections; they are NULL when the pair is invalid. */
typedef struct {
  int64_t n_p, n_q;        /* countNonDegenIntP / Q: ring vertices plus inserted vertices */
  int32_t invalid;         /* 1 when the P-side and Q-side intersection counts differ (:1460-1476) */
  double* xy_p;            /* merged rings in ring order, interleaved x,y (intersectionsP / Q) */
  double* xy_q;
  int32_t* alpha_p;        /* (int)(1e7 * alpha) where the vertex carries an intersection, -100
                              at plain vertices (alphaValuesP / Q) */
  int32_t* alpha_q;
  int32_t* label_p;        /* initial label (IntersectionLabel, polygon.h:21-32) at P vertices
                              with a key and at their Q neighbours, -100 elsewhere, -102 where
                              the two positions name no label (initLabelsP / Q) */
  int32_t* label_q;
  int32_t* neighbor_p;     /* 1-based index of the linked vertex in the other ring, 0 = none */
  int32_t* neighbor_q;
} gcmfgh_intersections;

/* P = polygon p_id of p_layer, Q = polygon q_id of q_layer (device layers in the reference
 * layout, as spatialJoin hands them out); P is not swapped with Q.  The common MBR is the
 * intersection of the two polygons' MBRs, as the caller computes it (ghcuda.cpp:94-125).
 * Differences from the reference: the per-edge vertex order is by exact FP64 parameter (the
 * reference sorts the integer keys), ties on the Q side's source-vertex keys go to the
 * largest P edge (a race in the reference), neighbour entries of plain vertices are 0 (left
 * uninitialised there), and for an invalid pair n_q counts the Q vertices inserted by the
 * P-side records (the reference counts its Q-side pass). */
gcmfgh_status gh_calculate_intersections(gcmfgh_ctx* ctx, const gcmfgh_layer* p_layer, int32_t p_id,
                                         const gcmfgh_layer* q_layer, int32_t q_id, gcmfgh_intersections* out);
void gh_free_intersections(gcmfgh_intersections* x);

/* ---- the device primitives the path is built on.  Replace PrefixSum (GPU_Utility.h:128,
 * a multi-pass inclusive scan, GPU_PrefixSum.h:355) and RadixSort (GPU_Utility.h:242, a
 * 16-digit decimal LSD sort, GPU_RadixSort.h:27-148).  d_* are device pointers.
 * exclusive scan: d_out[i] = sum(d_in[0..i-1]); *total (host, may be NULL) = sum(d_in).
 * radix sort: stable ascending by the low key_bits bits of d_keys, d_vals permuted along. */
gcmfgh_status gcmfgh_exclusive_scan_i32(gcmfgh_ctx* ctx, const int32_t* d_in, int64_t* d_out, int64_t n,
                                        int64_t* total);
gcmfgh_status gcmfgh_radix_sort_u64(gcmfgh_ctx* ctx, uint64_t* d_keys, uint32_t* d_vals, int64_t n,
                                    int key_bits);

/* ---- allocation-free exclusive scan.  No counterpart in the reference.
 * For callers that cannot let a library allocate device memory: engines that account for
 * every device byte through their own pool, or latency-sensitive loops that must not hit
 * cudaMalloc's implicit synchronisation.  Same result as gcmfgh_exclusive_scan_i32, but
 * needs no context and calls no cudaMalloc/cudaFree: its scratch is a fixed device array
 * inside the library (about 66 KB, held on every GPU that loads the library until the
 * process exits), so n is limited to GCMFGH_NOALLOC_SCAN_MAX_ELEMENTS; larger n returns
 * GCMFGH_INVALID_ARGUMENT.  d_in, d_out, d_total (may be NULL) are device pointers on the
 * current device; stream is a cudaStream_t (NULL = legacy default stream).  The call
 * returns when the result is ready.  The first call on a device looks the scratch array's
 * address up (cudaGetSymbolAddress), so make that first call before any stream capture.
 * The looked-up address is kept for the life of the process, so cudaDeviceReset on a
 * device after its first call here is not supported.  Input values may be negative.
 * All calls share the one array: calls that overlap on the GPU (other threads, other
 * streams of the same device) race and must be serialised by the caller. */
#define GCMFGH_NOALLOC_SCAN_MAX_ELEMENTS (1LL << 24)
gcmfgh_status gcmfgh_exclusive_scan_i32_noalloc(const int32_t* d_in, int64_t* d_out, int64_t n,
                                                int64_t* d_total, void* stream);

/* ---- host-resident layers: H2D copies, join, clip of the clip set; results stay on the
 * device for the *_get calls.  This is the end-to-end path of the reference's main()
 * (main.cpp:15-29). */
gcmfgh_status gcmfgh_join_clip_host(gcmfgh_ctx* ctx, const gcmfgh_layer* base_host,
                                    const gcmfgh_layer* overlay_host, gcmfgh_join_info* jinfo,
                                    gcmfgh_clip_info* cinfo);

/* ---- the GCMF text layer format (dataConverter.py:95-111; reader
 * ReadTextFormatPolygon2WithVector, SEQ_Overlay.h:285-390): a header line, then per
 * polygon "id minx miny maxx maxy x0 y0 ... x0 y0".  gcmfgh_read_text_layer parses it on
 * `threads` host threads (<= 0: all cores) with the reference reader's rules (tokens of
 * 0-9 . -, MBR over every pair read, zero-width MBR polygons skipped) into malloc'ed
 * host arrays in the layer layout above; ids holds each stored polygon's file id.
 * gcmfgh_write_text_layer writes a host layer in the format, 17 significant digits in
 * fixed-point notation (the reference tokenizer has no exponents). */
typedef struct {
  double* coords;
  int32_t* vnum;
  int64_t* vps;
  int64_t* ids;
  int64_t n_polys;
  int64_t n_vertices;
} gcmfgh_text_layer;
gcmfgh_status gcmfgh_read_text_layer(const char* path, int threads, gcmfgh_text_layer* out);
void gcmfgh_free_text_layer(gcmfgh_text_layer* layer);
gcmfgh_status gcmfgh_write_text_layer(const char* path, const gcmfgh_layer* host_layer);

/* copy a host layer to the device; the copy belongs to the context and lives until
 * gcmfgh_destroy.  dev_out receives the device view. */
gcmfgh_status gcmfgh_upload_layer(gcmfgh_ctx* ctx, const gcmfgh_layer* host_layer, gcmfgh_layer* dev_out);

/* ---- serving: continuous batching of join+clip queries against a resident layer.
 * No counterpart in the reference (its main() runs one join and one clip over two whole
 * layers, main.cpp:15-29).  The resident layer is copied to the device once and indexed
 * by an MBR grid.  Each submitted query polygon is joined against it (the same MBR
 * candidate predicate, containment, common-MBR and segment filters as gcmf_join, with the
 * query as base polygon) and clipped against every hit (as gh_clip_batch, swap rule
 * included).  Worker threads, each with its own stream and device workspace, take the
 * queries waiting at that moment as one batch: FIFO, at most max_batch_queries queries and
 * max_batch_vertices query vertices, and no more vertices than
 * (free device memory - reserve_bytes) / bytes_per_vertex (at least one query).  While one
 * batch is on the GPU the next worker admits what arrived meanwhile.  A query's result
 * does not depend on the other queries of its batch.  workers = 1 with
 * max_batch_queries = 1 is the plain one-query-per-launch form. */
typedef struct gcmfgh_server gcmfgh_server;
typedef struct {
  int device;
  int workers;                 /* batches in flight at once (default 2) */
  int64_t max_batch_queries;   /* default 4096 */
  int64_t max_batch_vertices;  /* default 2^22 */
  int64_t reserve_bytes;       /* device memory left free when admitting (default 2 GiB) */
  int64_t bytes_per_vertex;    /* working-set estimate per query vertex (default 4096) */
  double eps, eps_clean;       /* as gcmfgh_set_params */
  int union_mode;
  int exact;                   /* GCMFGH_PRECISION_EXACT semantics when nonzero */
} gcmfgh_serve_options;
typedef struct {
  int32_t status;              /* gcmfgh_status of the query's batch */
  int64_t n_hits;              /* clipped pairs (resident polygons in the clip set) */
  int64_t n_components;
  int64_t n_vertices;
  int64_t n_candidates;        /* MBR candidates */
  int64_t arrival_ns;          /* CLOCK_MONOTONIC nanoseconds */
  int64_t admitted_ns;         /* taken into a batch */
  int64_t done_ns;             /* results on the host */
  int64_t batch_id;
  int64_t batch_queries;       /* queries in that batch */
} gcmfgh_serve_result;
gcmfgh_status gcmfgh_serve_default_options(gcmfgh_serve_options* opt);
/* resident: HOST layer in the layout above; opt may be NULL (defaults) */
gcmfgh_status gcmfgh_serve_open(const gcmfgh_layer* resident, const gcmfgh_serve_options* opt,
                                gcmfgh_server** out);
/* one query: host open ring (no closing vertex) of n vertices, copied before returning;
 * arrival_ns: when the request arrived (CLOCK_MONOTONIC ns; <= 0 = now).  Thread-safe. */
gcmfgh_status gcmfgh_serve_submit(gcmfgh_server* srv, const double* xy, int32_t n, int64_t arrival_ns,
                                  uint64_t* ticket);
/* GCMFGH_NOT_READY until the query's batch has completed, then fills *info */
gcmfgh_status gcmfgh_serve_poll(gcmfgh_server* srv, uint64_t ticket, gcmfgh_serve_result* info);
/* blocks until completed or timeout_ms elapsed (< 0: no limit) */
gcmfgh_status gcmfgh_serve_wait(gcmfgh_server* srv, uint64_t ticket, int64_t timeout_ms,
                                gcmfgh_serve_result* info);
/* copies a completed result and releases the ticket: per hit its resident polygon id,
 * clip status and component count [n_hits]; component sizes [n_components]; vertices
 * [2 n_vertices].  Hits are in ascending resident id; NULL skips a field. */
gcmfgh_status gcmfgh_serve_take(gcmfgh_server* srv, uint64_t ticket, int32_t* hit_ids, int32_t* hit_status,
                                int32_t* hit_ncomp, int32_t* comp_size, double* xy);
gcmfgh_status gcmfgh_serve_stats(gcmfgh_server* srv, int64_t* batches, int64_t* queries, int64_t* peak_batch);
/* Where serving time goes, summed over all batches so far (batches of different workers
 * overlap on the GPU, so these are shares, not wall time).  ms[7]: host staging, H2D,
 * MBR candidates (grid index + sort), join stages J3-J6, clip, D2H (GPU times from CUDA
 * events on the worker's stream), and the host split of the results.  work[4]: query
 * vertices, clipped pairs, merged-ring vertices, result vertices.  No counterpart in the
 * reference (it has no serving loop). */
gcmfgh_status gcmfgh_serve_phases(gcmfgh_server* srv, double* ms, int64_t* work);
/* finishes the queued queries, stops the workers and frees the device state */
gcmfgh_status gcmfgh_serve_close(gcmfgh_server* srv);

#ifdef __cplusplus
}
#endif

#endif /* GCMFGH_H */
