// api.cu -- the C ABI (include/gcmfgh.h): contexts, device arenas, argument checks and
// result export.  The reference's entry points exit the process on errors
// (GPU_Manage.h:25-44, ghcuda.cpp:109-116); these return a status instead.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>
#include <vector>
#include "common.cuh"
#include "engine.cuh"
#include "prims.cuh"
#include "../../include/gcmfgh.h"

namespace gcmfgh {

cudaStream_t create_priority_stream() {
  int lo = 0, hi = 0;
  cudaDeviceGetStreamPriorityRange(&lo, &hi);
  cudaStream_t s = nullptr;
  if (cudaStreamCreateWithPriority(&s, cudaStreamNonBlocking, hi) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  return s;
}

std::atomic<unsigned long long>& launch_counter() {
  static std::atomic<unsigned long long> n{0};
  return n;
}

void* Arena::take(size_t bytes) {
  bytes = (bytes + 255) & ~size_t(255);
  for (auto& c : chunks_) {                       // first fit: earlier chunks' leftover room too
    if (c.off + bytes <= c.cap) {
      void* p = c.base + c.off;
      c.off += bytes;
      return p;
    }
  }
  size_t last = 0;
  for (auto& c : chunks_) last = c.cap > last ? c.cap : last;
  size_t cap = bytes > 2 * last ? bytes : 2 * last;
  if (cap < (size_t(64) << 20)) cap = size_t(64) << 20;
  char* p = nullptr;
  if (cudaMalloc(&p, cap) != cudaSuccess) {
    cudaGetLastError();
    // Chunks not touched since the last reset() hold nothing: give them back (cudaFree
    // waits for the device), then retry with the exact size.
    for (size_t i = 0; i < chunks_.size();) {
      if (chunks_[i].off == 0) {
        cudaFree(chunks_[i].base);
        chunks_.erase(chunks_.begin() + (std::ptrdiff_t)i);
      } else {
        ++i;
      }
    }
    cap = bytes;
    if (cudaMalloc(&p, cap) != cudaSuccess) { cudaGetLastError(); return nullptr; }
  }
  chunks_.push_back({p, cap, bytes});
  return p;
}

void Arena::release() {
  for (auto& c : chunks_) cudaFree(c.base);
  chunks_.clear();
}

namespace {

constexpr int kThreads = 256;

__global__ void clip_stats_kernel(const int32_t* __restrict__ status, int64_t n, unsigned long long* out) {
  int64_t i = (int64_t)blockIdx.x * kThreads + threadIdx.x;
  unsigned long long c[3] = {0, 0, 0};
  if (i < n) {
    int s = status[i];
    if (s == 1) c[0] = 1;
    if (s == 2) c[1] = 1;
    if (s == 3) c[2] = 1;
  }
  for (int j = 0; j < 3; ++j) {
    unsigned long long v = warp_sum(c[j]);
    if (lane_id() == 0 && v) atomicAdd(&out[j], v);
  }
}

}  // namespace
}  // namespace gcmfgh

using namespace gcmfgh;

// One record of the autotuner: the thresholds chosen for a workload signature.
struct TuneRecord {
  std::string gpu;
  int pairs_log2 = 0, verts_log2 = 0, exact = 0;
  int64_t bin_grid = 0, tile_label = 0, mid_label = 0, big_label = 0, wide_label = 0;
  double ms_default = 0, ms_tuned = 0;
};

struct gcmfgh_ctx {
  int device = 0;
  std::string gpu_name;
  bool tuning_explicit = false;   // gcmfgh_set_tuning was called: recorded tunings are not applied
  int join_f32 = 5;               // join options: FP32 prefilters (bit 0 MBR y test, bit 1 edge test),
                                  // bit 2 the sort-sweep MBR filter instead of the grid probe,
                                  // bit 3 the sweep as count and emit passes
  bool hint_explicit = false;     // gcmfgh_set_tuning fixed the record capacity hint
  int64_t cand_hint = 0;          // MBR candidates of the last join (the one-pass sweep's capacity)
  int64_t list_hint[2] = {0, 0};  // common-MBR edge list entries of the last join (the one-pass filter's)
  std::vector<TuneRecord> tunings;
  cudaStream_t own = nullptr;
  cudaStream_t stream = nullptr;
  cudaStream_t aux = nullptr;     // high-priority stream for the long pairs' labelling
  cudaStream_t aux2 = nullptr;    // third stream: the warp-per-pair labelling beside the tiles
  Arena join_arena, clip_arena, layer_arena, pair_arena;
  int* d_err = nullptr;
  int64_t* h_scratch = nullptr;   // pinned
  unsigned long long* d_stats = nullptr;
  JoinDev join;
  bool have_join = false;
  ClipDev clip;
  bool have_clip = false;
  ClipParams prm;
  int last_err = 0;
  const double* join_b = nullptr;
  const double* join_o = nullptr;
  int64_t join_nb = 0, join_no = 0;
  Marks marks[2];                 // stage timing of the last join / clip
  std::vector<void*> uploads;     // gcmfgh_upload_layer copies, freed by gcmfgh_destroy
};

namespace {

gcmfgh_status to_status(int st) { return static_cast<gcmfgh_status>(st); }

bool layer_ok(const gcmfgh_layer* L) {
  if (!L || L->n_polys < 0) return false;
  if (L->n_polys == 0) return true;
  if (!L->coords || !L->vnum || !L->vps) return false;
  if (reinterpret_cast<uintptr_t>(L->coords) % 16 != 0) return false;   // 128-bit vertex loads
  return true;
}

LayerDev to_dev(const gcmfgh_layer* L) { return LayerDev{L->coords, L->vnum, L->vps, L->n_polys, L->n_vertices}; }

gcmfgh_status finish(gcmfgh_ctx* c, int st) {
  if (st != ST_OK) {
    cudaStreamSynchronize(c->stream);
    cudaError_t e = cudaGetLastError();
    (void)e;
    return to_status(st);
  }
  if (cudaMemcpyAsync(c->h_scratch + 60, c->d_err, sizeof(int), cudaMemcpyDeviceToHost, c->stream) != cudaSuccess)
    return GCMFGH_CUDA_ERROR;
  if (cudaStreamSynchronize(c->stream) != cudaSuccess) return GCMFGH_CUDA_ERROR;
  if (cudaGetLastError() != cudaSuccess) return GCMFGH_CUDA_ERROR;
  int e = *reinterpret_cast<int*>(c->h_scratch + 60);
  c->last_err = e;
  if (e == DEV_TIMEOUT) return GCMFGH_DEVICE_ERROR;
  return GCMFGH_OK;
}

gcmfgh_status clip_info(gcmfgh_ctx* c, gcmfgh_clip_info* info) {
  if (!info) return GCMFGH_OK;
  info->n_pairs = c->clip.n_pairs;
  info->n_components = c->clip.n_components;
  info->n_vertices = c->clip.n_vertices;
  info->n_records = c->clip.n_records;
  info->n_ring_vertices = c->clip.n_ring_vertices;
  info->n_invalid = info->n_disjoint = info->n_error = 0;
  if (c->clip.n_pairs > 0) {
    cudaMemsetAsync(c->d_stats, 0, 3 * sizeof(unsigned long long), c->stream);
    { clip_stats_kernel<<<(unsigned)((c->clip.n_pairs + kThreads - 1) / kThreads), kThreads, 0, c->stream>>>(
        c->clip.status, c->clip.n_pairs, c->d_stats); note_launch(); }
    cudaMemcpyAsync(c->h_scratch, c->d_stats, 3 * sizeof(int64_t), cudaMemcpyDeviceToHost, c->stream);
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) return GCMFGH_CUDA_ERROR;
    info->n_invalid = c->h_scratch[0];
    info->n_disjoint = c->h_scratch[1];
    info->n_error = c->h_scratch[2];
  }
  return GCMFGH_OK;
}

int floor_log2(double v) { return v >= 1.0 ? (int)std::floor(std::log2(v)) : 0; }

int mean_verts_log2(const gcmfgh_layer* b, const gcmfgh_layer* o) {
  const int64_t np = b->n_polys + o->n_polys;
  return np > 0 ? floor_log2((double)(b->n_vertices + o->n_vertices) / (double)np) : 0;
}

// the recorded thresholds for this workload's signature, if any
const TuneRecord* find_tuning(const gcmfgh_ctx* c, int pl, int vl, int exact) {
  for (const auto& t : c->tunings)
    if (t.gpu == c->gpu_name && t.pairs_log2 == pl && t.verts_log2 == vl && t.exact == exact) return &t;
  return nullptr;
}

void apply_tuning(ClipParams& p, const TuneRecord& t) {
  p.bin_grid = t.bin_grid;
  p.tile_label_max = t.tile_label;
  p.mid_label_min = t.mid_label;
  p.big_label_min = t.big_label;
  p.wide_label_min = t.wide_label;
}

// the parameters a clip of n pairs on these layers runs with
ClipParams clip_params(const gcmfgh_ctx* c, const gcmfgh_layer* b, const gcmfgh_layer* o, int64_t n) {
  ClipParams p = c->prm;
  if (!c->tuning_explicit) {
    const TuneRecord* t = find_tuning(c, floor_log2((double)std::max<int64_t>(n, 1)), mean_verts_log2(b, o), p.exact);
    if (t) apply_tuning(p, *t);
  }
  return p;
}

// the last join's edge lists, for a clip of its clip set
JoinEdges join_edges(const gcmfgh_ctx* c) {
  JoinEdges e;
  const JoinDev& J = c->join;
  if (!J.clip_cand || !J.bOff) return e;
  e.cand = J.clip_cand; e.flag = J.join_flag; e.bE = J.bE; e.oE = J.oE;
  e.bOff = J.bOff; e.oOff = J.oOff; e.bList = J.bList; e.oList = J.oList;
  return e;
}

gcmfgh_status run_clip_ctx(gcmfgh_ctx* c, const gcmfgh_layer* b, const gcmfgh_layer* o,
                           const int32_t* pid, const int32_t* qid, int64_t n, gcmfgh_clip_info* info,
                           const double* mbrB = nullptr, const double* mbrO = nullptr,
                           const ClipParams* force = nullptr, const JoinEdges* je = nullptr) {
  c->clip_arena.reset();
  c->have_clip = false;
  c->marks[1].n = 0;
  cudaMemsetAsync(c->d_err, 0, sizeof(int), c->stream);
  const ClipParams prm = force ? *force : clip_params(c, b, o, n);
  int st = run_clip(to_dev(b), to_dev(o), pid, qid, n, prm, c->clip_arena, c->clip, c->d_err,
                    c->h_scratch, c->stream, &c->marks[1], c->aux, nullptr, c->aux2, mbrB, mbrO, je);
  gcmfgh_status r = finish(c, st);
  if (r != GCMFGH_OK) return r;
  c->have_clip = true;
  if (!c->hint_explicit) c->prm.rec_hint = c->clip.n_records;   // the next clip's record capacity
  return clip_info(c, info);
}

// ---- tuning records on disk: one JSON object per line
bool json_str(const std::string& line, const char* key, std::string& out) {
  std::string k = std::string("\"") + key + "\": \"";
  size_t a = line.find(k);
  if (a == std::string::npos) return false;
  a += k.size();
  size_t e = line.find('"', a);
  if (e == std::string::npos) return false;
  out = line.substr(a, e - a);
  return true;
}

bool json_num(const std::string& line, const char* key, double& out) {
  std::string k = std::string("\"") + key + "\": ";
  size_t a = line.find(k);
  if (a == std::string::npos) return false;
  out = std::strtod(line.c_str() + a + k.size(), nullptr);
  return true;
}

bool json_int(const std::string& line, const char* key, int64_t& out) {
  std::string k = std::string("\"") + key + "\": ";
  size_t a = line.find(k);
  if (a == std::string::npos) return false;
  out = (int64_t)std::strtoll(line.c_str() + a + k.size(), nullptr, 10);
  return true;
}

void load_tunings(const char* path, std::vector<TuneRecord>& out) {
  FILE* f = std::fopen(path, "r");
  if (!f) return;
  char buf[1024];
  while (std::fgets(buf, sizeof(buf), f)) {
    std::string line(buf);
    TuneRecord t;
    int64_t v[8];
    const char* keys[8] = {"pairs_log2", "verts_log2", "exact", "bin_grid", "tile_label", "mid_label",
                           "big_label", "wide_label"};
    bool ok = json_str(line, "gpu", t.gpu);
    for (int i = 0; i < 8 && ok; ++i) ok = json_int(line, keys[i], v[i]);
    ok = ok && json_num(line, "ms_default", t.ms_default) && json_num(line, "ms_tuned", t.ms_tuned);
    if (!ok) continue;
    t.pairs_log2 = (int)v[0]; t.verts_log2 = (int)v[1]; t.exact = (int)v[2];
    t.bin_grid = v[3]; t.tile_label = v[4]; t.mid_label = v[5]; t.big_label = v[6]; t.wide_label = v[7];
    out.push_back(t);
  }
  std::fclose(f);
}

void save_tunings(const char* path, const std::vector<TuneRecord>& recs) {
  FILE* f = std::fopen(path, "w");
  if (!f) return;
  for (const auto& t : recs)
    std::fprintf(f,
                 "{\"gpu\": \"%s\", \"pairs_log2\": %d, \"verts_log2\": %d, \"exact\": %d, \"bin_grid\": %lld, "
                 "\"tile_label\": %lld, \"mid_label\": %lld, \"big_label\": %lld, \"wide_label\": %lld, "
                 "\"ms_default\": %.6f, \"ms_tuned\": %.6f}\n",
                 t.gpu.c_str(), t.pairs_log2, t.verts_log2, t.exact, (long long)t.bin_grid, (long long)t.tile_label,
                 (long long)t.mid_label, (long long)t.big_label, (long long)t.wide_label, t.ms_default, t.ms_tuned);
  std::fclose(f);
}

TuneRecord record_of(const ClipParams& p) {
  TuneRecord t;
  t.bin_grid = p.bin_grid; t.tile_label = p.tile_label_max; t.mid_label = p.mid_label_min;
  t.big_label = p.big_label_min; t.wide_label = p.wide_label_min;
  return t;
}

void to_public(const TuneRecord& t, gcmfgh_tuning* out) {
  out->bin_grid = t.bin_grid; out->tile_label = t.tile_label; out->mid_label = t.mid_label;
  out->big_label = t.big_label; out->wide_label = t.wide_label;
  out->pairs_log2 = t.pairs_log2; out->verts_log2 = t.verts_log2; out->exact = t.exact;
  out->ms_default = t.ms_default; out->ms_tuned = t.ms_tuned;
}

struct FieldRef { const void* p; int64_t count; int esize; };

FieldRef join_field(const gcmfgh_ctx* c, int f) {
  const JoinDev& J = c->join;
  int64_t K = J.n_pairs;
  switch (f) {
    case GCMF_PAIR_BASE: return {J.b, K, 4};
    case GCMF_PAIR_OVERLAY: return {J.o, K, 4};
    case GCMF_CMBR: return {J.cmbr, 4 * K, 8};
    case GCMF_PIP_TYPE: return {J.pip_type, K, 1};
    case GCMF_PIP_FLAG: return {J.pip_flag, K, 1};
    case GCMF_JOIN_FLAG: return {J.join_flag, K, 1};
    case GCMF_BASE_EDGES: return {J.bE, K, 4};
    case GCMF_OVERLAY_EDGES: return {J.oE, K, 4};
    case GCMF_SEG_FLAG: return {J.seg_flag, K, 1};
    case GCMF_CLIP_FLAG: return {J.clip, K, 1};
    case GCMF_CLIP_BASE: return {J.clip_b, J.n_clip, 4};
    case GCMF_CLIP_OVERLAY: return {J.clip_o, J.n_clip, 4};
    case GCMF_MBR_BASE: return {J.mbr_b, J.mbr_b ? 4 * c->join_nb : 0, 8};
    case GCMF_MBR_OVERLAY: return {J.mbr_o, J.mbr_o ? 4 * c->join_no : 0, 8};
    case GCMF_VALID_BASE: return {J.valid_b, J.valid_b ? c->join_nb : 0, 1};
    case GCMF_VALID_OVERLAY: return {J.valid_o, J.valid_o ? c->join_no : 0, 1};
  }
  return {nullptr, -1, 0};
}

FieldRef clip_field(const gcmfgh_ctx* c, int f) {
  const ClipDev& C = c->clip;
  switch (f) {
    case GH_STATUS: return {C.status, C.n_pairs, 4};
    case GH_NCOMP: return {C.ncomp, C.n_pairs, 4};
    case GH_COMP_OFFSET: return {C.comp_off, C.n_pairs, 8};
    case GH_COUNT1: return {C.count1, C.n_pairs, 8};
    case GH_COMP_SIZE: return {C.comp_size, C.n_components, 4};
    case GH_VERT_OFFSET: return {C.vert_off, C.n_pairs, 8};
    case GH_XY: return {C.xy, 2 * C.n_vertices, 8};
    case GH_SWAPPED: return {C.swapped, C.n_pairs, 4};
  }
  return {nullptr, -1, 0};
}

gcmfgh_status copy_field(gcmfgh_ctx* c, FieldRef r, void* dst, int64_t cap, int on_dev, int64_t* bytes) {
  if (r.count < 0) return GCMFGH_INVALID_ARGUMENT;
  int64_t nb = r.count * r.esize;
  if (bytes) *bytes = nb;
  if (!dst) return GCMFGH_OK;
  if (cap < nb) return GCMFGH_CAPACITY;
  if (nb == 0) return GCMFGH_OK;
  if (!r.p) return GCMFGH_NOT_READY;
  cudaError_t e = cudaMemcpyAsync(dst, r.p, (size_t)nb, on_dev ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                                  c->stream);
  if (e != cudaSuccess) return GCMFGH_CUDA_ERROR;
  if (cudaStreamSynchronize(c->stream) != cudaSuccess) return GCMFGH_CUDA_ERROR;
  return GCMFGH_OK;
}

}  // namespace

extern "C" {

const char* gcmfgh_status_string(gcmfgh_status s) {
  switch (s) {
    case GCMFGH_OK: return "ok";
    case GCMFGH_INVALID_ARGUMENT: return "invalid argument";
    case GCMFGH_CUDA_ERROR: return "CUDA error";
    case GCMFGH_OUT_OF_MEMORY: return "out of device memory";
    case GCMFGH_DEVICE_ERROR: return "device-side error";
    case GCMFGH_NOT_READY: return "no result yet";
    case GCMFGH_CAPACITY: return "destination too small";
    case GCMFGH_NO_DEVICE: return "no CUDA device";
  }
  return "unknown status";
}

gcmfgh_status gcmfgh_create(int device, gcmfgh_ctx** out) {
  if (!out) return GCMFGH_INVALID_ARGUMENT;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) { cudaGetLastError(); return GCMFGH_NO_DEVICE; }
  if (device < 0 || device >= n) return GCMFGH_INVALID_ARGUMENT;
  if (cudaSetDevice(device) != cudaSuccess) return GCMFGH_CUDA_ERROR;
  gcmfgh_ctx* c = new (std::nothrow) gcmfgh_ctx();
  if (!c) return GCMFGH_OUT_OF_MEMORY;
  c->device = device;
  if (cudaStreamCreateWithFlags(&c->own, cudaStreamNonBlocking) != cudaSuccess ||
      cudaMalloc(&c->d_err, 64) != cudaSuccess ||
      cudaMalloc(&c->d_stats, 64) != cudaSuccess ||
      cudaMallocHost(&c->h_scratch, 64 * sizeof(int64_t)) != cudaSuccess) {
    gcmfgh_destroy(c);
    return GCMFGH_CUDA_ERROR;
  }
  c->stream = c->own;
  c->aux = create_priority_stream();
  if (cudaStreamCreateWithFlags(&c->aux2, cudaStreamNonBlocking) != cudaSuccess) {
    cudaGetLastError();
    c->aux2 = nullptr;
  }
  cudaMemset(c->d_err, 0, 64);
  for (auto& m : c->marks)
    for (int i = 0; i < Marks::kMax; ++i) cudaEventCreate(&m.ev[i]);
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) == cudaSuccess) c->gpu_name = prop.name;
  else cudaGetLastError();
  if (const char* f = std::getenv("GCMFGH_TUNING_FILE")) load_tunings(f, c->tunings);
  *out = c;
  return GCMFGH_OK;
}

gcmfgh_status gcmfgh_set_timing(gcmfgh_ctx* c, int on) {
  if (!c) return GCMFGH_INVALID_ARGUMENT;
  c->marks[0].on = c->marks[1].on = (on != 0);
  return GCMFGH_OK;
}

int gcmfgh_get_timing(gcmfgh_ctx* c, int which, float* ms, const char** names, int cap) {
  if (!c || which < 0 || which > 1) return -1;
  Marks& m = c->marks[which];
  int n = m.n > 1 ? m.n - 1 : 0;
  for (int i = 0; i < n && i < cap; ++i) {
    float t = 0;
    cudaEventElapsedTime(&t, m.ev[i], m.ev[i + 1]);
    if (ms) ms[i] = t;
    if (names) names[i] = m.name[i + 1];
  }
  return n;
}

gcmfgh_status gcmfgh_destroy(gcmfgh_ctx* c) {
  if (!c) return GCMFGH_OK;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  c->join_arena.release();
  c->clip_arena.release();
  c->layer_arena.release();
  c->pair_arena.release();
  for (void* p : c->uploads) cudaFree(p);
  if (c->d_err) cudaFree(c->d_err);
  if (c->d_stats) cudaFree(c->d_stats);
  if (c->h_scratch) cudaFreeHost(c->h_scratch);
  if (c->own) cudaStreamDestroy(c->own);
  if (c->aux) cudaStreamDestroy(c->aux);
  if (c->aux2) cudaStreamDestroy(c->aux2);
  for (auto& m : c->marks)
    for (int i = 0; i < Marks::kMax; ++i)
      if (m.ev[i]) cudaEventDestroy(m.ev[i]);
  delete c;
  return GCMFGH_OK;
}

gcmfgh_status gcmfgh_set_stream(gcmfgh_ctx* c, void* stream) {
  if (!c) return GCMFGH_INVALID_ARGUMENT;
  c->stream = stream ? static_cast<cudaStream_t>(stream) : c->own;
  return GCMFGH_OK;
}

gcmfgh_status gcmfgh_set_params(gcmfgh_ctx* c, double eps, double eps_clean, int union_mode) {
  if (!c || !(eps >= 0) || !(eps_clean >= 0)) return GCMFGH_INVALID_ARGUMENT;
  c->prm.eps = eps;
  c->prm.eps_clean = eps_clean;
  c->prm.union_mode = union_mode ? 1 : 0;
  return GCMFGH_OK;
}

gcmfgh_status gcmfgh_upload_layer(gcmfgh_ctx* c, const gcmfgh_layer* h, gcmfgh_layer* d) {
  if (!c || !h || !d || h->n_polys < 0) return GCMFGH_INVALID_ARGUMENT;
  if (h->n_polys > 0 && (!h->coords || !h->vnum || !h->vps)) return GCMFGH_INVALID_ARGUMENT;
  cudaSetDevice(c->device);
  const int64_t n = h->n_polys;
  const int64_t nv = n > 0 ? (h->n_vertices > 0 ? h->n_vertices : h->vps[n - 1]) : 0;
  const size_t bxy = ((sizeof(double) * 2 * nv + 255) / 256) * 256;
  const size_t bvn = ((sizeof(int32_t) * n + 255) / 256) * 256;
  char* p = nullptr;
  if (cudaMalloc(&p, bxy + bvn + sizeof(int64_t) * n + 256) != cudaSuccess) { cudaGetLastError(); return GCMFGH_OUT_OF_MEMORY; }
  c->uploads.push_back(p);
  cudaMemcpyAsync(p, h->coords, sizeof(double) * 2 * nv, cudaMemcpyHostToDevice, c->stream);
  cudaMemcpyAsync(p + bxy, h->vnum, sizeof(int32_t) * n, cudaMemcpyHostToDevice, c->stream);
  cudaMemcpyAsync(p + bxy + bvn, h->vps, sizeof(int64_t) * n, cudaMemcpyHostToDevice, c->stream);
  if (cudaStreamSynchronize(c->stream) != cudaSuccess) return GCMFGH_CUDA_ERROR;
  d->coords = reinterpret_cast<const double*>(p);
  d->vnum = reinterpret_cast<const int32_t*>(p + bxy);
  d->vps = reinterpret_cast<const int64_t*>(p + bxy + bvn);
  d->n_polys = n;
  d->n_vertices = nv;
  return GCMFGH_OK;
}

gcmfgh_status gcmfgh_set_precision(gcmfgh_ctx* c, int mode) {
  if (!c || (mode != GCMFGH_PRECISION_REFERENCE && mode != GCMFGH_PRECISION_EXACT)) return GCMFGH_INVALID_ARGUMENT;
  c->prm.exact = mode == GCMFGH_PRECISION_EXACT;
  return GCMFGH_OK;
}

gcmfgh_status gcmfgh_set_tuning(gcmfgh_ctx* c, int key, int64_t value) {
  if (!c || value < 0) return GCMFGH_INVALID_ARGUMENT;
  if (key == GCMFGH_TUNE_F32_FILTER) {
    c->join_f32 = (c->join_f32 & 12) | (int)(value & 3);
    return GCMFGH_OK;
  }
  if (key == GCMFGH_TUNE_SWEEP_TWO_PASS) {
    c->join_f32 = (c->join_f32 & 7) | (value ? 8 : 0);
    return GCMFGH_OK;
  }
  if (key == GCMFGH_TUNE_JOIN_SWEEP) {
    c->join_f32 = (c->join_f32 & 11) | (value ? 4 : 0);
    return GCMFGH_OK;
  }
  if (key == GCMFGH_TUNE_FUSED_EMIT) {
    if (value > 2) return GCMFGH_INVALID_ARGUMENT;
    c->prm.fused_emit = (int)value;
    return GCMFGH_OK;
  }
  if (key == GCMFGH_TUNE_RECORD_HINT) {
    c->prm.rec_hint = value;
    c->hint_explicit = value > 0;
    return GCMFGH_OK;
  }
  c->tuning_explicit = true;
  if (key == GCMFGH_TUNE_BIN_GRID) c->prm.bin_grid = value;
  else if (key == GCMFGH_TUNE_BIG_LABEL) c->prm.big_label_min = value;
  else if (key == GCMFGH_TUNE_MID_LABEL) c->prm.mid_label_min = value;
  else if (key == GCMFGH_TUNE_TILE_LABEL) c->prm.tile_label_max = value;
  else if (key == GCMFGH_TUNE_WIDE_LABEL) c->prm.wide_label_min = value;
  else return GCMFGH_INVALID_ARGUMENT;
  return GCMFGH_OK;
}

int gcmfgh_last_device_error(gcmfgh_ctx* c) { return c ? c->last_err : -1; }

unsigned long long gcmfgh_launch_count(void) { return launch_counter(); }

}  // extern "C"

// gcmf_join; ovl_ready (may be null): an event recorded after the overlay's upload
static gcmfgh_status join_impl(gcmfgh_ctx* c, const gcmfgh_layer* b, const gcmfgh_layer* o, gcmfgh_join_info* info,
                               cudaEvent_t ovl_ready) {
  if (!c || !layer_ok(b) || !layer_ok(o)) return GCMFGH_INVALID_ARGUMENT;
  cudaSetDevice(c->device);
  c->join_arena.reset();
  c->have_join = false;
  c->marks[0].n = 0;
  cudaMemsetAsync(c->d_err, 0, sizeof(int), c->stream);
  int st = run_join(to_dev(b), to_dev(o), c->join_arena, c->join, c->d_err, c->h_scratch, c->stream,
                    &c->marks[0], c->aux, c->join_f32, ovl_ready, c->cand_hint, c->list_hint[0],
                    c->list_hint[1]);
  gcmfgh_status r = finish(c, st);
  if (r != GCMFGH_OK) return r;
  c->have_join = true;
  c->cand_hint = c->join.n_pairs;                  // the next join's key and list capacities
  c->list_hint[0] = c->join.n_blist;
  c->list_hint[1] = c->join.n_olist;
  c->join_b = b->coords;
  c->join_o = o->coords;
  c->join_nb = b->n_polys;
  c->join_no = o->n_polys;
  if (info) {
    info->n_pairs = c->join.n_pairs;
    info->n_pip_candidates = c->join.n_pip_candidates;
    info->n_within = c->join.n_within;
    info->n_cmf = c->join.n_cmf;
    info->n_seg = c->join.n_seg;
    info->n_clip = c->join.n_clip;
  }
  return GCMFGH_OK;
}

extern "C" {

gcmfgh_status gcmf_join(gcmfgh_ctx* c, const gcmfgh_layer* b, const gcmfgh_layer* o, gcmfgh_join_info* info) {
  return join_impl(c, b, o, info, nullptr);
}

gcmfgh_status gcmf_join_get(gcmfgh_ctx* c, int f, void* dst, int64_t cap, int on_dev, int64_t* bytes) {
  if (!c) return GCMFGH_INVALID_ARGUMENT;
  if (!c->have_join) return GCMFGH_NOT_READY;
  return copy_field(c, join_field(c, f), dst, cap, on_dev, bytes);
}

gcmfgh_status gcmf_join_ptr(gcmfgh_ctx* c, int f, const void** p, int64_t* count) {
  if (!c || !p) return GCMFGH_INVALID_ARGUMENT;
  if (!c->have_join) return GCMFGH_NOT_READY;
  FieldRef r = join_field(c, f);
  if (r.count < 0) return GCMFGH_INVALID_ARGUMENT;
  *p = r.p;
  if (count) *count = r.count;
  return GCMFGH_OK;
}

gcmfgh_status gh_clip_batch(gcmfgh_ctx* c, const gcmfgh_layer* b, const gcmfgh_layer* o, const int32_t* pid,
                            const int32_t* qid, int64_t n, gcmfgh_clip_info* info) {
  if (!c || !layer_ok(b) || !layer_ok(o) || n < 0 || (n > 0 && (!pid || !qid))) return GCMFGH_INVALID_ARGUMENT;
  cudaSetDevice(c->device);
  c->prm.no_swap = 0;
  return run_clip_ctx(c, b, o, pid, qid, n, info);
}

gcmfgh_status gh_clip_batch_host_ids(gcmfgh_ctx* c, const gcmfgh_layer* b, const gcmfgh_layer* o,
                                     const int32_t* pid, const int32_t* qid, int64_t n, gcmfgh_clip_info* info) {
  if (!c || !layer_ok(b) || !layer_ok(o) || n < 0 || (n > 0 && (!pid || !qid))) return GCMFGH_INVALID_ARGUMENT;
  cudaSetDevice(c->device);
  c->pair_arena.reset();
  int32_t* d = c->pair_arena.take_n<int32_t>(2 * std::max<int64_t>(n, 1));
  if (!d) return GCMFGH_OUT_OF_MEMORY;
  if (n > 0) {
    cudaMemcpyAsync(d, pid, sizeof(int32_t) * n, cudaMemcpyHostToDevice, c->stream);
    cudaMemcpyAsync(d + n, qid, sizeof(int32_t) * n, cudaMemcpyHostToDevice, c->stream);
  }
  c->prm.no_swap = 0;
  return run_clip_ctx(c, b, o, d, d + n, n, info);
}

gcmfgh_status gh_clip_joined(gcmfgh_ctx* c, const gcmfgh_layer* b, const gcmfgh_layer* o, gcmfgh_clip_info* info) {
  if (!c || !layer_ok(b) || !layer_ok(o)) return GCMFGH_INVALID_ARGUMENT;
  if (!c->have_join) return GCMFGH_NOT_READY;
  if (b->coords != c->join_b || o->coords != c->join_o) return GCMFGH_INVALID_ARGUMENT;
  cudaSetDevice(c->device);
  c->prm.no_swap = 0;
  // the join's polygon MBRs of the same layers (mbr_kernel computes what the clip would)
  const JoinEdges je = join_edges(c);
  return run_clip_ctx(c, b, o, c->join.clip_b, c->join.clip_o, c->join.n_clip, info, c->join.mbr_b,
                      c->join.mbr_o, nullptr, &je);
}

gcmfgh_status gcmfgh_tuning_for(gcmfgh_ctx* c, const gcmfgh_layer* b, const gcmfgh_layer* o, int64_t n,
                                gcmfgh_tuning* out) {
  if (!c || !layer_ok(b) || !layer_ok(o) || n < 0 || !out) return GCMFGH_INVALID_ARGUMENT;
  TuneRecord t = record_of(clip_params(c, b, o, n));
  t.pairs_log2 = floor_log2((double)std::max<int64_t>(n, 1));
  t.verts_log2 = mean_verts_log2(b, o);
  t.exact = c->prm.exact;
  if (const TuneRecord* r = c->tuning_explicit ? nullptr : find_tuning(c, t.pairs_log2, t.verts_log2, t.exact)) {
    t.ms_default = r->ms_default;
    t.ms_tuned = r->ms_tuned;
  }
  std::memset(out, 0, sizeof(*out));
  to_public(t, out);
  return GCMFGH_OK;
}

gcmfgh_status gcmfgh_autotune_joined(gcmfgh_ctx* c, const gcmfgh_layer* b, const gcmfgh_layer* o,
                                     gcmfgh_tuning* out) {
  if (!c || !layer_ok(b) || !layer_ok(o) || !out) return GCMFGH_INVALID_ARGUMENT;
  if (!c->have_join) return GCMFGH_NOT_READY;
  if (b->coords != c->join_b || o->coords != c->join_o) return GCMFGH_INVALID_ARGUMENT;
  cudaSetDevice(c->device);
  c->prm.no_swap = 0;
  const int64_t n = c->join.n_clip;
  const JoinEdges je = join_edges(c);
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) return GCMFGH_CUDA_ERROR;
  int timed = 0;
  // median of three clips of the join's clip set under parameters p (ms), < 0 on failure
  auto time_with = [&](const ClipParams& p) -> float {
    float t[3];
    gcmfgh_clip_info info;
    for (int r = 0; r < 3; ++r) {
      cudaEventRecord(e0, c->stream);
      if (run_clip_ctx(c, b, o, c->join.clip_b, c->join.clip_o, n, &info, c->join.mbr_b, c->join.mbr_o, &p, &je) !=
          GCMFGH_OK)
        return -1.0f;
      cudaEventRecord(e1, c->stream);
      cudaEventSynchronize(e1);
      cudaEventElapsedTime(&t[r], e0, e1);
    }
    ++timed;
    std::sort(t, t + 3);
    return t[1];
  };
  ClipParams cur = clip_params(c, b, o, n);
  gcmfgh_clip_info warm;
  run_clip_ctx(c, b, o, c->join.clip_b, c->join.clip_o, n, &warm, c->join.mbr_b, c->join.mbr_o, &cur, &je);
  const float ms0 = time_with(cur);
  if (ms0 < 0) { cudaEventDestroy(e0); cudaEventDestroy(e1); return GCMFGH_CUDA_ERROR; }
  float best = ms0;
  // one pass of coordinate descent; the candidates span the useful range of each limit
  const int64_t kNever = INT64_MAX / 4;
  using Field = int64_t ClipParams::*;
  struct Knob { Field f; std::vector<int64_t> vals; };
  const Knob knobs[] = {
      {&ClipParams::bin_grid, {1ll << 10, 1ll << 12, 1ll << 14, 1ll << 16, 1ll << 20, 1ll << 24}},
      {&ClipParams::tile_label_max, {0, 32, 64, 96, 128, 192, 256}},
      {&ClipParams::mid_label_min, {256, 512, 1024, 2048, 4096}},
      {&ClipParams::big_label_min, {1ll << 15, 1ll << 16, 1ll << 17, 1ll << 18, 1ll << 19}},
      {&ClipParams::wide_label_min, {0, 1ll << 16, kNever}},
  };
  for (const Knob& k : knobs) {
    const int64_t keep = cur.*(k.f);
    int64_t chosen = keep;
    for (int64_t v : k.vals) {
      if (v == keep) continue;
      ClipParams p = cur;
      p.*(k.f) = v;
      const float ms = time_with(p);
      if (ms >= 0 && ms < best) { best = ms; chosen = v; }
    }
    cur.*(k.f) = chosen;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  TuneRecord t = record_of(cur);
  t.gpu = c->gpu_name;
  t.pairs_log2 = floor_log2((double)std::max<int64_t>(n, 1));
  t.verts_log2 = mean_verts_log2(b, o);
  t.exact = cur.exact;
  t.ms_default = ms0;
  t.ms_tuned = best;
  bool replaced = false;
  for (auto& r : c->tunings)
    if (r.gpu == t.gpu && r.pairs_log2 == t.pairs_log2 && r.verts_log2 == t.verts_log2 && r.exact == t.exact) {
      r = t;
      replaced = true;
    }
  if (!replaced) c->tunings.push_back(t);
  c->tuning_explicit = false;
  if (const char* f = std::getenv("GCMFGH_TUNING_FILE")) save_tunings(f, c->tunings);
  std::memset(out, 0, sizeof(*out));
  to_public(t, out);
  out->configs_timed = timed;
  // leave the clip result of the chosen thresholds in place
  gcmfgh_clip_info info;
  return run_clip_ctx(c, b, o, c->join.clip_b, c->join.clip_o, n, &info, c->join.mbr_b, c->join.mbr_o, &cur, &je);
}

gcmfgh_status gh_clip_get(gcmfgh_ctx* c, int f, void* dst, int64_t cap, int on_dev, int64_t* bytes) {
  if (!c) return GCMFGH_INVALID_ARGUMENT;
  if (!c->have_clip) return GCMFGH_NOT_READY;
  return copy_field(c, clip_field(c, f), dst, cap, on_dev, bytes);
}

gcmfgh_status gh_clip_ptr(gcmfgh_ctx* c, int f, const void** p, int64_t* count) {
  if (!c || !p) return GCMFGH_INVALID_ARGUMENT;
  if (!c->have_clip) return GCMFGH_NOT_READY;
  FieldRef r = clip_field(c, f);
  if (r.count < 0) return GCMFGH_INVALID_ARGUMENT;
  *p = r.p;
  if (count) *count = r.count;
  return GCMFGH_OK;
}

gcmfgh_status gh_clip_pair(gcmfgh_ctx* c, const double* P, int32_t nP, const double* Q, int32_t nQ,
                           gcmfgh_clip_info* info) {
  if (!c || !P || !Q || nP < 1 || nQ < 1) return GCMFGH_INVALID_ARGUMENT;
  cudaSetDevice(c->device);
  c->pair_arena.reset();
  // two one-polygon layers in the reference layout (closing vertex appended)
  int64_t nv = (int64_t)nP + 1 + nQ + 1;
  double* xy = c->pair_arena.take_n<double>(2 * nv);
  int32_t* vn = c->pair_arena.take_n<int32_t>(4);
  int64_t* vp = c->pair_arena.take_n<int64_t>(4);
  int32_t* ids = c->pair_arena.take_n<int32_t>(2);
  if (!xy || !vn || !vp || !ids) return GCMFGH_OUT_OF_MEMORY;
  double* hxy = static_cast<double*>(malloc(sizeof(double) * 2 * nv));
  if (!hxy) return GCMFGH_OUT_OF_MEMORY;
  memcpy(hxy, P, sizeof(double) * 2 * nP);
  hxy[2 * nP] = P[0]; hxy[2 * nP + 1] = P[1];
  memcpy(hxy + 2 * (nP + 1), Q, sizeof(double) * 2 * nQ);
  hxy[2 * (nP + 1 + nQ)] = Q[0]; hxy[2 * (nP + 1 + nQ) + 1] = Q[1];
  int32_t hvn[2] = {nP + 1, nQ + 1};
  int64_t hvp[2] = {(int64_t)nP + 1, (int64_t)nQ + 1};
  int32_t hid[2] = {0, 0};
  cudaMemcpyAsync(xy, hxy, sizeof(double) * 2 * nv, cudaMemcpyHostToDevice, c->stream);
  cudaMemcpyAsync(vn, hvn, sizeof(hvn), cudaMemcpyHostToDevice, c->stream);
  cudaMemcpyAsync(vp, hvp, sizeof(hvp), cudaMemcpyHostToDevice, c->stream);
  cudaMemcpyAsync(ids, hid, sizeof(hid), cudaMemcpyHostToDevice, c->stream);
  cudaStreamSynchronize(c->stream);
  free(hxy);
  gcmfgh_layer lb{xy, vn, vp, 1, (int64_t)nP + 1};
  gcmfgh_layer lo{xy + 2 * (nP + 1), vn + 1, vp + 1, 1, (int64_t)nQ + 1};
  c->prm.no_swap = 1;
  gcmfgh_status r = run_clip_ctx(c, &lb, &lo, ids, ids + 1, 1, info);
  c->prm.no_swap = 0;
  return r;
}

gcmfgh_status gh_clip_multi(gcmfgh_ctx* c, const double* P, const int32_t* p_sizes, int32_t p_rings,
                            const double* Q, const int32_t* q_sizes, int32_t q_rings, gcmfgh_clip_info* info) {
  if (!c || !P || !Q || !p_sizes || !q_sizes || p_rings < 1 || q_rings < 1) return GCMFGH_INVALID_ARGUMENT;
  for (int32_t i = 0; i < p_rings; ++i) if (p_sizes[i] < 3) return GCMFGH_INVALID_ARGUMENT;
  for (int32_t i = 0; i < q_rings; ++i) if (q_sizes[i] < 3) return GCMFGH_INVALID_ARGUMENT;
  cudaSetDevice(c->device);
  c->clip_arena.reset();
  c->have_clip = false;
  c->marks[1].n = 0;
  cudaMemsetAsync(c->d_err, 0, sizeof(int), c->stream);
  int st = run_clip_multi(P, p_sizes, p_rings, Q, q_sizes, q_rings, c->prm, c->clip_arena, c->clip, c->d_err,
                          c->h_scratch, c->stream);
  gcmfgh_status r = finish(c, st);
  if (r != GCMFGH_OK) return r;
  c->have_clip = true;
  return clip_info(c, info);
}

gcmfgh_status gh_clip_multi_batch(gcmfgh_ctx* c, int64_t n, const double* P, const int32_t* p_sizes,
                                  const int32_t* p_rings, const double* Q, const int32_t* q_sizes,
                                  const int32_t* q_rings, gcmfgh_clip_info* info) {
  if (!c || n < 1 || !P || !Q || !p_sizes || !q_sizes || !p_rings || !q_rings) return GCMFGH_INVALID_ARGUMENT;
  cudaSetDevice(c->device);
  c->clip_arena.reset();
  c->have_clip = false;
  c->marks[1].n = 0;
  cudaMemsetAsync(c->d_err, 0, sizeof(int), c->stream);
  int st = run_clip_multi_batch(n, P, p_sizes, p_rings, Q, q_sizes, q_rings, c->prm, c->clip_arena, c->clip,
                                c->d_err, c->h_scratch, c->stream);
  gcmfgh_status r = finish(c, st);
  if (r != GCMFGH_OK) return r;
  c->have_clip = true;
  return clip_info(c, info);
}

gcmfgh_status gh_calculate_intersections(gcmfgh_ctx* c, const gcmfgh_layer* pl, int32_t p_id,
                                         const gcmfgh_layer* ql, int32_t q_id, gcmfgh_intersections* out) {
  if (!out) return GCMFGH_INVALID_ARGUMENT;
  std::memset(out, 0, sizeof(*out));
  if (!c || !layer_ok(pl) || !layer_ok(ql) || p_id < 0 || q_id < 0 || p_id >= pl->n_polys || q_id >= ql->n_polys)
    return GCMFGH_INVALID_ARGUMENT;
  cudaSetDevice(c->device);
  c->pair_arena.reset();
  int32_t* ids = c->pair_arena.take_n<int32_t>(2);
  if (!ids) return GCMFGH_OUT_OF_MEMORY;
  const int32_t hid[2] = {p_id, q_id};
  if (cudaMemcpy(ids, hid, sizeof(hid), cudaMemcpyHostToDevice) != cudaSuccess) return GCMFGH_CUDA_ERROR;
  c->clip_arena.reset();
  c->have_clip = false;
  c->marks[1].n = 0;
  cudaMemsetAsync(c->d_err, 0, sizeof(int), c->stream);
  ClipParams prm = c->prm;
  prm.no_swap = 1;
  RingExport ex;
  int st = run_clip(to_dev(pl), to_dev(ql), ids, ids + 1, 1, prm, c->clip_arena, c->clip, c->d_err, c->h_scratch,
                    c->stream, nullptr, nullptr, &ex);
  gcmfgh_status r = finish(c, st);
  if (r != GCMFGH_OK) return r;
  out->n_p = ex.n_p;
  out->n_q = ex.n_q;
  out->invalid = ex.status == 1 ? 1 : 0;
  if (ex.status == 1) return GCMFGH_OK;
  if (ex.status == 2) {
    // disjoint MBRs: no edge meets the (empty) common MBR, so the rings come back as they
    // are, every vertex plain
    const gcmfgh_layer* L[2] = {pl, ql};
    const int32_t id[2] = {p_id, q_id};
    std::vector<double>* dst[2] = {&ex.xy_p, &ex.xy_q};
    int64_t n[2];
    for (int side = 0; side < 2; ++side) {
      int32_t vn = 0;
      int64_t vp = 0;
      if (cudaMemcpy(&vn, L[side]->vnum + id[side], sizeof(vn), cudaMemcpyDeviceToHost) != cudaSuccess ||
          cudaMemcpy(&vp, L[side]->vps + id[side], sizeof(vp), cudaMemcpyDeviceToHost) != cudaSuccess)
        return GCMFGH_CUDA_ERROR;
      n[side] = std::max<int64_t>(vn - 1, 0);
      dst[side]->resize(2 * n[side]);
      if (n[side] > 0 && cudaMemcpy(dst[side]->data(), L[side]->coords + 2 * (vp - vn),
                                    2 * n[side] * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
        return GCMFGH_CUDA_ERROR;
    }
    out->n_p = n[0];
    out->n_q = n[1];
    ex.alpha_p.assign(n[0], -100); ex.label_p.assign(n[0], -100); ex.nb_p.assign(n[0], 0);
    ex.alpha_q.assign(n[1], -100); ex.label_q.assign(n[1], -100); ex.nb_q.assign(n[1], 0);
  } else if (ex.status != 0) {
    return GCMFGH_DEVICE_ERROR;
  }
  const int64_t np = out->n_p, nq = out->n_q;
  out->xy_p = static_cast<double*>(malloc(sizeof(double) * 2 * std::max<int64_t>(np, 1)));
  out->xy_q = static_cast<double*>(malloc(sizeof(double) * 2 * std::max<int64_t>(nq, 1)));
  int32_t** arr[6] = {&out->alpha_p, &out->label_p, &out->neighbor_p, &out->alpha_q, &out->label_q, &out->neighbor_q};
  const std::vector<int32_t>* src[6] = {&ex.alpha_p, &ex.label_p, &ex.nb_p, &ex.alpha_q, &ex.label_q, &ex.nb_q};
  bool ok = out->xy_p && out->xy_q;
  for (int i = 0; i < 6; ++i) {
    const int64_t n = i < 3 ? np : nq;
    *arr[i] = static_cast<int32_t*>(malloc(sizeof(int32_t) * std::max<int64_t>(n, 1)));
    ok = ok && *arr[i];
    if (*arr[i] && n > 0) memcpy(*arr[i], src[i]->data(), sizeof(int32_t) * n);
  }
  if (!ok) {
    gh_free_intersections(out);
    return GCMFGH_OUT_OF_MEMORY;
  }
  if (np > 0) memcpy(out->xy_p, ex.xy_p.data(), sizeof(double) * 2 * np);
  if (nq > 0) memcpy(out->xy_q, ex.xy_q.data(), sizeof(double) * 2 * nq);
  return GCMFGH_OK;
}

void gh_free_intersections(gcmfgh_intersections* x) {
  if (!x) return;
  free(x->xy_p); free(x->xy_q);
  free(x->alpha_p); free(x->alpha_q);
  free(x->label_p); free(x->label_q);
  free(x->neighbor_p); free(x->neighbor_q);
  const int64_t np = x->n_p, nq = x->n_q;
  const int32_t inv = x->invalid;
  std::memset(x, 0, sizeof(*x));
  x->n_p = np; x->n_q = nq; x->invalid = inv;
}

gcmfgh_status gcmfgh_exclusive_scan_i32(gcmfgh_ctx* c, const int32_t* d_in, int64_t* d_out, int64_t n,
                                        int64_t* total) {
  if (!c || n < 0 || (n > 0 && (!d_in || !d_out))) return GCMFGH_INVALID_ARGUMENT;
  cudaSetDevice(c->device);
  c->pair_arena.reset();
  void* tmp = c->pair_arena.take(scan_temp_bytes(n > 0 ? n : 1));
  int64_t* d_tot = c->pair_arena.take_n<int64_t>(1);
  if (!tmp || !d_tot) return GCMFGH_OUT_OF_MEMORY;
  cudaMemsetAsync(c->d_err, 0, sizeof(int), c->stream);
  exclusive_scan_i32(d_in, d_out, n, d_tot, tmp, c->d_err, c->stream);
  cudaMemcpyAsync(c->h_scratch + 32, d_tot, sizeof(int64_t), cudaMemcpyDeviceToHost, c->stream);
  gcmfgh_status r = finish(c, ST_OK);
  if (r == GCMFGH_OK && total) *total = c->h_scratch[32];
  return r;
}

gcmfgh_status gcmfgh_radix_sort_u64(gcmfgh_ctx* c, uint64_t* d_keys, uint32_t* d_vals, int64_t n, int key_bits) {
  if (!c || n < 0 || (n > 0 && (!d_keys || !d_vals)) || key_bits < 0 || key_bits > 64)
    return GCMFGH_INVALID_ARGUMENT;
  cudaSetDevice(c->device);
  c->pair_arena.reset();
  uint64_t* ka = c->pair_arena.take_n<uint64_t>(n);
  uint32_t* va = c->pair_arena.take_n<uint32_t>(n);
  void* tmp = c->pair_arena.take(radix_temp_bytes(n > 0 ? n : 1));
  if (!ka || !va || !tmp) return GCMFGH_OUT_OF_MEMORY;
  cudaMemsetAsync(c->d_err, 0, sizeof(int), c->stream);
  radix_sort_pairs(d_keys, d_vals, ka, va, n, ((key_bits + 7) / 8) * 8, tmp, c->d_err, c->stream);
  return finish(c, ST_OK);
}

gcmfgh_status gcmfgh_join_clip_host(gcmfgh_ctx* c, const gcmfgh_layer* bh, const gcmfgh_layer* oh,
                                    gcmfgh_join_info* jinfo, gcmfgh_clip_info* cinfo) {
  if (!c || !bh || !oh || bh->n_polys < 0 || oh->n_polys < 0) return GCMFGH_INVALID_ARGUMENT;
  cudaSetDevice(c->device);
  c->layer_arena.reset();
  gcmfgh_layer dl[2];
  const gcmfgh_layer* hl[2] = {bh, oh};
  // The overlay goes up on the auxiliary stream, where the join processes it: the base
  // layer's MBRs and sort on the main stream overlap the overlay's copy.
  cudaEvent_t ovl_done = nullptr;
  cudaStream_t ovl_stream = c->stream;
  if (c->aux && cudaEventCreateWithFlags(&ovl_done, cudaEventDisableTiming) == cudaSuccess) ovl_stream = c->aux;
  struct EvGuard { cudaEvent_t e; ~EvGuard() { if (e) { cudaEventSynchronize(e); cudaEventDestroy(e); } } } guard{ovl_done};
  for (int i = 0; i < 2; ++i) {
    const gcmfgh_layer* h = hl[i];
    cudaStream_t cs = i == 0 ? c->stream : ovl_stream;
    double* xy = c->layer_arena.take_n<double>(2 * h->n_vertices);
    int32_t* vn = c->layer_arena.take_n<int32_t>(h->n_polys);
    int64_t* vp = c->layer_arena.take_n<int64_t>(h->n_polys);
    if (!xy || !vn || !vp) return GCMFGH_OUT_OF_MEMORY;
    if (h->n_polys > 0) {
      if (!h->coords || !h->vnum || !h->vps) return GCMFGH_INVALID_ARGUMENT;
      if (cudaMemcpyAsync(xy, h->coords, sizeof(double) * 2 * h->n_vertices, cudaMemcpyHostToDevice, cs) !=
              cudaSuccess ||
          cudaMemcpyAsync(vn, h->vnum, sizeof(int32_t) * h->n_polys, cudaMemcpyHostToDevice, cs) != cudaSuccess ||
          cudaMemcpyAsync(vp, h->vps, sizeof(int64_t) * h->n_polys, cudaMemcpyHostToDevice, cs) != cudaSuccess)
        return GCMFGH_CUDA_ERROR;
    }
    dl[i] = gcmfgh_layer{xy, vn, vp, h->n_polys, h->n_vertices};
  }
  if (ovl_done) cudaEventRecord(ovl_done, ovl_stream);
  gcmfgh_status r = join_impl(c, &dl[0], &dl[1], jinfo, ovl_done);
  if (r != GCMFGH_OK) return r;
  return gh_clip_joined(c, &dl[0], &dl[1], cinfo);
}

}  // extern "C"
