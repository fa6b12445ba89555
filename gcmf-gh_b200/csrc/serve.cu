// serve.cu -- continuous-batching server for join+clip queries against a resident layer.
//
// No counterpart in the reference: its main() (main.cpp:15-29) runs one join and one
// clip over two whole layers.  Here a layer stays resident in HBM with an MBR grid index;
// query polygons are submitted one at a time from any host thread, and worker threads
// (each with its own stream and device arenas) take the queries waiting at that moment
// as one batch, sized by a vertex budget and by the device memory that is free, run
// MBR candidates -> stages J3-J6 -> clip on it, and copy the results back.  While one
// worker's batch is on the GPU the next worker admits the requests that arrived
// meanwhile, so batches overlap on the device.
//
// A batch's result for a query does not depend on which other queries share the batch:
// the MBR candidates of a query are the pairs the join's sweep would form between the
// query and the resident layer (same predicate, see sweep_kernel in join.cu), and every
// later stage works per pair.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>
#include "common.cuh"
#include "engine.cuh"
#include "grid.cuh"
#include "prims.cuh"
#include "../../include/gcmfgh.h"

namespace gcmfgh {
namespace {

constexpr int kThreads = 256;
constexpr int kWarpsPerBlock = kThreads / 32;
inline unsigned blocks_for_warps(int64_t warps) { return (unsigned)((warps + kWarpsPerBlock - 1) / kWarpsPerBlock); }
inline unsigned blocks_for(int64_t n) { return (unsigned)((n + kThreads - 1) / kThreads); }

int key_bits_for(int64_t n) {
  int b = 1;
  while ((1ll << b) < n) ++b;
  return b;
}

int64_t now_ns() {
  return std::chrono::duration_cast<std::chrono::nanoseconds>(
             std::chrono::steady_clock::now().time_since_epoch()).count();
}

// Polygon MBR over every stored vertex and the join's validity rule (mbr_kernel in
// join.cu: at least two stored vertices, nonzero width and height).
__global__ void serve_mbr_kernel(LayerDev L, double* __restrict__ mbr, uint8_t* __restrict__ valid) {
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
  if (lane_id() == 0) {
    reinterpret_cast<double4*>(mbr)[w] = make_double4(x1, y1, x2, y2);
    valid[w] = (nv >= 2 && x1 != x2 && y1 != y2) ? 1 : 0;
  }
}

// Pinned host blocks for the batches' results, recycled: a batch's results are copied from
// the device into one block, its requests read their ranges from it, and the block goes
// back to the pool when the last of them has been taken.
class PinnedPool {
 public:
  struct Block { char* p = nullptr; size_t cap = 0; };
  ~PinnedPool() { for (auto& b : free_) cudaFreeHost(b.p); }
  Block get(size_t n) {
    {
      std::lock_guard<std::mutex> lk(mu_);
      size_t best = free_.size();
      for (size_t i = 0; i < free_.size(); ++i)
        if (free_[i].cap >= n && (best == free_.size() || free_[i].cap < free_[best].cap)) best = i;
      if (best < free_.size()) {
        Block b = free_[best];
        free_.erase(free_.begin() + (std::ptrdiff_t)best);
        return b;
      }
    }
    Block b;
    const size_t cap = std::max<size_t>(n + n / 4, size_t(16) << 20);
    if (cudaMallocHost(&b.p, cap) != cudaSuccess) { cudaGetLastError(); return Block{}; }
    b.cap = cap;
    return b;
  }
  void put(Block b) {
    if (!b.p) return;
    std::lock_guard<std::mutex> lk(mu_);
    free_.push_back(b);
  }
 private:
  std::mutex mu_;
  std::vector<Block> free_;
};

// A batch's results on the host, shared by its requests: pairs sorted by (query, resident
// id), then their components and vertices in the same order, so each request's part is
// one range of each array.
struct BatchOut {
  PinnedPool* pool = nullptr;
  PinnedPool::Block blk;
  size_t o_b = 0, o_o = 0, o_st = 0, o_nc = 0, o_cs = 0, o_xy = 0;
  ~BatchOut() { if (pool) pool->put(blk); }
  const int32_t* i32(size_t o) const { return reinterpret_cast<const int32_t*>(blk.p + o); }
  const double* xy() const { return reinterpret_cast<const double*>(blk.p + o_xy); }
};

struct Request {
  std::vector<double> ring;      // open ring, interleaved x,y
  int32_t n = 0;
  int64_t arrival_ns = 0, admitted_ns = 0, done_ns = 0;
  int64_t batch_id = -1, batch_queries = 0;
  int status = GCMFGH_OK;
  bool done = false;
  int64_t n_candidates = 0;
  std::shared_ptr<const BatchOut> out;    // results: pairs [p0, p1), components [c0, c1), vertices [v0, v1)
  int64_t p0 = 0, p1 = 0, c0 = 0, c1 = 0, v0 = 0, v1 = 0;
};

template <class T>
struct Pinned {
  T* p = nullptr;
  size_t cap = 0;
  ~Pinned() { if (p) cudaFreeHost(p); }
  bool reserve(size_t n) {
    if (n <= cap) return true;
    if (p) cudaFreeHost(p);
    p = nullptr;
    cap = 0;
    size_t c = std::max<size_t>(n, 1024);
    c = std::max(c, size_t(1.5 * (double)n));
    if (cudaMallocHost(&p, c * sizeof(T)) != cudaSuccess) { cudaGetLastError(); return false; }
    cap = c;
    return true;
  }
};

}  // namespace
}  // namespace gcmfgh

using namespace gcmfgh;

struct gcmfgh_server {
  gcmfgh_serve_options opt{};
  int device = 0;
  // resident layer + index (device)
  double* r_xy = nullptr;
  int32_t* r_vnum = nullptr;
  int64_t* r_vps = nullptr;
  int64_t r_n = 0;
  double* r_mbr = nullptr;
  uint8_t* r_valid = nullptr;
  int64_t* r_cellOff = nullptr;
  int32_t* r_cellList = nullptr;
  GridIndex grid{};
  // requests
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<uint64_t> queue;
  PinnedPool out_pool;           // declared before the requests, so it outlives their results
  std::unordered_map<uint64_t, std::shared_ptr<Request>> reqs;
  uint64_t next_ticket = 1;
  bool stopping = false;
  std::vector<std::thread> workers;
  std::atomic<int64_t> batches{0}, batched_queries{0}, peak_batch{0};
  int64_t next_batch = 0;
  // per-phase time summed over batches (batches of different workers overlap on the GPU,
  // so the sums show shares, not wall time): host staging, H2D, MBR candidates, join
  // stages J3-J6, clip, D2H, host split; and totals of the work those phases did
  std::mutex stats_mu;
  double phase_ms[7] = {0, 0, 0, 0, 0, 0, 0};
  int64_t work[4] = {0, 0, 0, 0};     // query vertices, clipped pairs, merged-ring vertices, result vertices

  LayerDev resident() const { return LayerDev{r_xy, r_vnum, r_vps, r_n}; }
  void worker_main(int wid);
  int run_batch(std::vector<std::shared_ptr<Request>>& batch, int64_t batch_id, cudaStream_t s, cudaStream_t aux,
                Arena& A,
                Arena& C, int* d_err, int64_t* h_scratch, Pinned<char>& hin, cudaEvent_t* ev);
};

namespace {

size_t align16(size_t b) { return (b + 15) & ~size_t(15); }

}  // namespace

// One batch: queries -> device layer, MBR candidates from the grid index, join stages
// J3-J6, clip of the clip set, results back to the host and split per query.
int gcmfgh_server::run_batch(std::vector<std::shared_ptr<Request>>& batch, int64_t batch_id, cudaStream_t s,
                             cudaStream_t aux,
                             Arena& A, Arena& C, int* d_err, int64_t* h_scratch, Pinned<char>& hin,
                             cudaEvent_t* ev) {
  A.reset();
  C.reset();
  const int64_t t_stage0 = now_ns();
  const int64_t nq = (int64_t)batch.size();
  int64_t nv = 0;
  for (auto& r : batch) nv += r->n + 1;
  // ---- host staging (layer layout: closing vertex stored, inclusive prefix)
  const size_t bxy = align16(sizeof(double) * 2 * nv), bvn = align16(sizeof(int32_t) * nq),
               bvp = align16(sizeof(int64_t) * nq);
  if (!hin.reserve(bxy + bvn + bvp)) return ST_OUT_OF_MEMORY;
  double* hxy = reinterpret_cast<double*>(hin.p);
  int32_t* hvn = reinterpret_cast<int32_t*>(hin.p + bxy);
  int64_t* hvp = reinterpret_cast<int64_t*>(hin.p + bxy + bvn);
  int64_t at = 0;
  for (int64_t i = 0; i < nq; ++i) {
    const Request& r = *batch[i];
    std::memcpy(hxy + 2 * at, r.ring.data(), sizeof(double) * 2 * r.n);
    hxy[2 * (at + r.n)] = r.ring[0];
    hxy[2 * (at + r.n) + 1] = r.ring[1];
    at += r.n + 1;
    hvn[i] = r.n + 1;
    hvp[i] = at;
  }
  char* dq = static_cast<char*>(A.take(bxy + bvn + bvp));
  double* qmbr = A.take_n<double>(4 * nq);
  uint8_t* qvalid = A.take_n<uint8_t>(nq);
  int32_t* qcnt = A.take_n<int32_t>(nq);
  int64_t* qoff = A.take_n<int64_t>(nq);
  int64_t* d_total = A.take_n<int64_t>(8);
  unsigned long long* d_cnt = A.take_n<unsigned long long>(8);
  void* stmp = A.take(scan_temp_bytes(nq));
  if (!dq || !qmbr || !qvalid || !qcnt || !qoff || !d_total || !d_cnt || !stmp) return ST_OUT_OF_MEMORY;
  const int64_t t_stage1 = now_ns();
  cudaEventRecord(ev[0], s);
  cudaMemsetAsync(d_err, 0, sizeof(int), s);
  cudaMemsetAsync(d_cnt, 0, 8 * sizeof(unsigned long long), s);
  cudaMemcpyAsync(dq, hin.p, bxy + bvn + bvp, cudaMemcpyHostToDevice, s);
  cudaEventRecord(ev[1], s);
  LayerDev Lq{reinterpret_cast<double*>(dq), reinterpret_cast<int32_t*>(dq + bxy),
              reinterpret_cast<int64_t*>(dq + bxy + bvn), nq};
  { serve_mbr_kernel<<<blocks_for_warps(nq), kThreads, 0, s>>>(Lq, qmbr, qvalid); note_launch(); }
  // ---- MBR candidates
  const int obits = key_bits_for(r_n), qbits = key_bits_for(nq);
  if (obits + qbits > 64) return ST_INVALID_ARGUMENT;
  { candidate_kernel<0><<<blocks_for_warps(nq), kThreads, 0, s>>>(qmbr, qvalid, nq, r_mbr, grid, qcnt, nullptr,
                                                                   nullptr, obits); note_launch(); }
  exclusive_scan_i32(qcnt, qoff, nq, d_total, stmp, d_err, s);
  cudaMemcpyAsync(h_scratch, d_total, sizeof(int64_t), cudaMemcpyDeviceToHost, s);
  if (cudaStreamSynchronize(s) != cudaSuccess) return ST_CUDA_ERROR;
  const int64_t K = h_scratch[0];
  std::vector<int32_t> candPerQuery(nq);
  JoinDev J;
  J.mbr_b = qmbr;
  J.mbr_o = r_mbr;
  ClipDev CD;
  int st = ST_OK;
  if (K > 0) {
    uint64_t* keys = A.take_n<uint64_t>(K);
    uint32_t* vals = A.take_n<uint32_t>(K);
    uint64_t* kAlt = A.take_n<uint64_t>(K);
    uint32_t* vAlt = A.take_n<uint32_t>(K);
    void* rtmp = A.take(radix_temp_bytes(K));
    if (!keys || !vals || !kAlt || !vAlt || !rtmp) return ST_OUT_OF_MEMORY;
    { candidate_kernel<1><<<blocks_for_warps(nq), kThreads, 0, s>>>(qmbr, qvalid, nq, r_mbr, grid, nullptr, qoff,
                                                                     keys, obits); note_launch(); }
    radix_sort_pairs(keys, vals, kAlt, vAlt, K, ((obits + qbits + 7) / 8) * 8, rtmp, d_err, s);
    cudaEventRecord(ev[2], s);
    // The common-MBR filter counts, then writes (two passes): a batch's edge lists vary too
    // much in size (queries of up to tens of thousands of vertices) for a one-pass capacity
    // taken from the last batch, and every overflow would repeat the pass.
    st = join_from_keys(Lq, resident(), keys, K, obits, A, J, d_total, d_cnt, d_err, h_scratch, s, nullptr, aux,
                        0, 0, true);
    if (st != ST_OK) return st;
    cudaEventRecord(ev[3], s);
    if (J.n_clip > 0) {
      ClipParams prm;
      prm.eps = opt.eps;
      prm.eps_clean = opt.eps_clean;
      prm.union_mode = opt.union_mode ? 1 : 0;
      prm.exact = opt.exact ? 1 : 0;
      // the clip's edge filter takes the join's common-MBR edge lists of the clip set
      const JoinEdges je{J.clip_cand, J.join_flag, J.bE, J.oE, J.bOff, J.oOff, J.bList, J.oList};
      st = run_clip(Lq, resident(), J.clip_b, J.clip_o, J.n_clip, prm, C, CD, d_err, h_scratch, s, nullptr, aux,
                    nullptr, nullptr, nullptr, nullptr, &je);
      if (st != ST_OK) return st;
    }
  } else {
    cudaEventRecord(ev[2], s);
    cudaEventRecord(ev[3], s);
  }
  cudaEventRecord(ev[4], s);
  // ---- results to the host
  const int64_t np = J.n_clip, nc = CD.n_components, nvo = CD.n_vertices;
  const size_t o_cnt = 0, o_b = align16(sizeof(int32_t) * nq), o_o = o_b + align16(sizeof(int32_t) * np),
               o_st = o_o + align16(sizeof(int32_t) * np), o_nc = o_st + align16(sizeof(int32_t) * np),
               o_cs = o_nc + align16(sizeof(int32_t) * np), o_xy = o_cs + align16(sizeof(int32_t) * nc),
               o_err = o_xy + align16(sizeof(double) * 2 * nvo), total = o_err + 16;
  auto out = std::make_shared<BatchOut>();
  out->blk = out_pool.get(total);
  if (!out->blk.p) return ST_OUT_OF_MEMORY;
  out->pool = &out_pool;
  char* H = out->blk.p;
  cudaMemcpyAsync(H + o_cnt, qcnt, sizeof(int32_t) * nq, cudaMemcpyDeviceToHost, s);
  if (np > 0) {
    cudaMemcpyAsync(H + o_b, J.clip_b, sizeof(int32_t) * np, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(H + o_o, J.clip_o, sizeof(int32_t) * np, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(H + o_st, CD.status, sizeof(int32_t) * np, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(H + o_nc, CD.ncomp, sizeof(int32_t) * np, cudaMemcpyDeviceToHost, s);
  }
  if (nc > 0) cudaMemcpyAsync(H + o_cs, CD.comp_size, sizeof(int32_t) * nc, cudaMemcpyDeviceToHost, s);
  if (nvo > 0) cudaMemcpyAsync(H + o_xy, CD.xy, sizeof(double) * 2 * nvo, cudaMemcpyDeviceToHost, s);
  cudaMemcpyAsync(H + o_err, d_err, sizeof(int), cudaMemcpyDeviceToHost, s);
  cudaEventRecord(ev[5], s);
  if (cudaStreamSynchronize(s) != cudaSuccess) return ST_CUDA_ERROR;
  if (*reinterpret_cast<int*>(H + o_err) != 0) return ST_DEVICE_ERROR;
  const int64_t t_done = now_ns();
  float gpu_ms[5] = {0, 0, 0, 0, 0};
  for (int i = 0; i < 5; ++i) cudaEventElapsedTime(&gpu_ms[i], ev[i], ev[i + 1]);
  // the batch's results stay in the block, shared by its requests (each takes its ranges)
  out->o_b = o_b; out->o_o = o_o; out->o_st = o_st; out->o_nc = o_nc; out->o_cs = o_cs; out->o_xy = o_xy;
  const int32_t* hcnt = reinterpret_cast<const int32_t*>(H + o_cnt);
  const int32_t* hb = out->i32(o_b);
  const int32_t* hnc = out->i32(o_nc);
  const int32_t* hcs = out->i32(o_cs);
  // pairs are sorted by (query, resident id); components and vertices follow pair order
  int64_t p = 0, c = 0, v = 0;
  for (int64_t i = 0; i < nq; ++i) {
    Request& r = *batch[i];
    r.n_candidates = hcnt[i];
    r.out = out;
    r.p0 = p; r.c0 = c; r.v0 = v;
    for (; p < np && hb[p] == i; ++p)
      for (int k = 0; k < hnc[p]; ++k) v += hcs[c++];
    r.p1 = p; r.c1 = c; r.v1 = v;
    r.done_ns = t_done;
    r.batch_id = batch_id;
    r.batch_queries = nq;
    r.status = GCMFGH_OK;
  }
  {
    std::lock_guard<std::mutex> lk(stats_mu);
    phase_ms[0] += (t_stage1 - t_stage0) * 1e-6;
    for (int i = 0; i < 5; ++i) phase_ms[1 + i] += gpu_ms[i];
    phase_ms[6] += (now_ns() - t_done) * 1e-6;
    work[0] += nv;
    work[1] += np;
    work[2] += CD.n_ring_vertices;
    work[3] += nvo;
  }
  return ST_OK;
}

void gcmfgh_server::worker_main(int wid) {
  (void)wid;
  cudaSetDevice(device);
  cudaStream_t s = nullptr;
  cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
  cudaStream_t aux = create_priority_stream();
  Arena A, C;
  int* d_err = nullptr;
  int64_t* h_scratch = nullptr;
  cudaMalloc(&d_err, sizeof(int));
  cudaMallocHost(&h_scratch, 64 * sizeof(int64_t));
  Pinned<char> hin;
  cudaEvent_t ev[6];
  for (auto& e : ev) cudaEventCreate(&e);
  for (;;) {
    std::vector<std::shared_ptr<Request>> batch;
    int64_t bid;
    {
      std::unique_lock<std::mutex> lk(mu);
      cv_work.wait(lk, [&] { return stopping || !queue.empty(); });
      if (queue.empty() && stopping) break;
      // admission: FIFO up to the query and vertex budgets; the vertex budget shrinks
      // with the device memory that is free beyond the reserve
      size_t freeB = 0, totalB = 0;
      cudaMemGetInfo(&freeB, &totalB);
      int64_t vbudget = opt.max_batch_vertices;
      const int64_t spare = (int64_t)freeB - opt.reserve_bytes;
      const int64_t memBudget = spare > 0 ? spare / std::max<int64_t>(1, opt.bytes_per_vertex) : 0;
      vbudget = std::min(vbudget, memBudget);
      int64_t vsum = 0;
      const int64_t now = now_ns();
      while (!queue.empty() && (int64_t)batch.size() < opt.max_batch_queries) {
        auto it = reqs.find(queue.front());
        if (it == reqs.end()) { queue.pop_front(); continue; }
        const int64_t add = it->second->n + 1;
        if (!batch.empty() && vsum + add > vbudget) break;
        vsum += add;
        it->second->admitted_ns = now;
        batch.push_back(it->second);
        queue.pop_front();
      }
      bid = next_batch++;
      if (!queue.empty()) cv_work.notify_one();
    }
    if (batch.empty()) continue;
    int st = run_batch(batch, bid, s, aux, A, C, d_err, h_scratch, hin, ev);
    if (st == ST_OUT_OF_MEMORY && batch.size() > 1) {
      // split the batch until it fits; a single query that does not fit fails alone
      A.release(); C.release();
      std::vector<std::shared_ptr<Request>> half(batch.begin() + batch.size() / 2, batch.end());
      batch.resize(batch.size() / 2);
      st = run_batch(batch, bid, s, aux, A, C, d_err, h_scratch, hin, ev);
      int st2 = run_batch(half, bid, s, aux, A, C, d_err, h_scratch, hin, ev);
      if (st2 != ST_OK) for (auto& r : half) { r->status = st2; r->done_ns = now_ns(); }
      std::lock_guard<std::mutex> lk(mu);
      for (auto& r : half) r->done = true;
    }
    if (st != ST_OK) {
      cudaStreamSynchronize(s);
      cudaGetLastError();
      const int64_t t = now_ns();
      for (auto& r : batch) { r->status = st; r->done_ns = t; r->batch_id = bid; r->batch_queries = (int64_t)batch.size(); }
    }
    batches += 1;
    batched_queries += (int64_t)batch.size();
    int64_t pk = peak_batch.load();
    while ((int64_t)batch.size() > pk && !peak_batch.compare_exchange_weak(pk, (int64_t)batch.size())) {}
    {
      std::lock_guard<std::mutex> lk(mu);
      for (auto& r : batch) r->done = true;
    }
    cv_done.notify_all();
  }
  A.release();
  C.release();
  for (auto& e : ev) cudaEventDestroy(e);
  cudaFree(d_err);
  cudaFreeHost(h_scratch);
  cudaStreamDestroy(s);
  if (aux) cudaStreamDestroy(aux);
}

extern "C" {

gcmfgh_status gcmfgh_serve_default_options(gcmfgh_serve_options* o) {
  if (!o) return GCMFGH_INVALID_ARGUMENT;
  o->device = 0;
  o->workers = 2;
  o->max_batch_queries = 4096;
  o->max_batch_vertices = 1 << 22;
  o->reserve_bytes = 2ll << 30;
  o->bytes_per_vertex = 4096;
  o->eps = 1e-7;
  o->eps_clean = 1e-7;
  o->union_mode = 0;
  o->exact = 0;
  return GCMFGH_OK;
}

gcmfgh_status gcmfgh_serve_open(const gcmfgh_layer* L, const gcmfgh_serve_options* opt, gcmfgh_server** out) {
  if (!L || !out || L->n_polys < 1 || !L->coords || !L->vnum || !L->vps || L->n_polys >= (1ll << 31))
    return GCMFGH_INVALID_ARGUMENT;
  gcmfgh_serve_options o;
  gcmfgh_serve_default_options(&o);
  if (opt) o = *opt;
  if (o.workers < 1 || o.max_batch_queries < 1 || o.max_batch_vertices < 1 || o.bytes_per_vertex < 1)
    return GCMFGH_INVALID_ARGUMENT;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= o.device) { cudaGetLastError(); return GCMFGH_NO_DEVICE; }
  std::unique_ptr<gcmfgh_server> S(new (std::nothrow) gcmfgh_server());
  if (!S) return GCMFGH_OUT_OF_MEMORY;
  S->opt = o;
  S->device = o.device;
  cudaSetDevice(o.device);
  const int64_t n = L->n_polys;
  int64_t nv = L->n_vertices > 0 ? L->n_vertices : L->vps[n - 1];
  S->r_n = n;
  if (cudaMalloc(&S->r_xy, sizeof(double) * 2 * nv) != cudaSuccess ||
      cudaMalloc(&S->r_vnum, sizeof(int32_t) * n) != cudaSuccess ||
      cudaMalloc(&S->r_vps, sizeof(int64_t) * n) != cudaSuccess ||
      cudaMalloc(&S->r_mbr, sizeof(double) * 4 * n) != cudaSuccess ||
      cudaMalloc(&S->r_valid, n) != cudaSuccess) {
    cudaGetLastError();
    gcmfgh_serve_close(S.release());
    return GCMFGH_OUT_OF_MEMORY;
  }
  cudaMemcpy(S->r_xy, L->coords, sizeof(double) * 2 * nv, cudaMemcpyHostToDevice);
  cudaMemcpy(S->r_vnum, L->vnum, sizeof(int32_t) * n, cudaMemcpyHostToDevice);
  cudaMemcpy(S->r_vps, L->vps, sizeof(int64_t) * n, cudaMemcpyHostToDevice);
  { serve_mbr_kernel<<<blocks_for_warps(n), kThreads>>>(S->resident(), S->r_mbr, S->r_valid); note_launch(); }
  std::vector<double> hm(4 * n);
  std::vector<uint8_t> hv(n);
  cudaMemcpy(hm.data(), S->r_mbr, sizeof(double) * 4 * n, cudaMemcpyDeviceToHost);
  cudaMemcpy(hv.data(), S->r_valid, n, cudaMemcpyDeviceToHost);
  // grid over the valid MBRs: cells about the mean MBR size, at most 2048 per axis
  double x0 = INFINITY, y0 = INFINITY, x1 = -INFINITY, y1 = -INFINITY, sw = 0, sh = 0;
  int64_t nvalid = 0;
  for (int64_t i = 0; i < n; ++i) {
    if (!hv[i]) continue;
    x0 = std::min(x0, hm[4 * i]); y0 = std::min(y0, hm[4 * i + 1]);
    x1 = std::max(x1, hm[4 * i + 2]); y1 = std::max(y1, hm[4 * i + 3]);
    sw += hm[4 * i + 2] - hm[4 * i]; sh += hm[4 * i + 3] - hm[4 * i + 1];
    ++nvalid;
  }
  GridIndex G{0, 0, 1, 1, 1, 1, nullptr, nullptr};
  if (nvalid > 0) G = grid_over(x0, y0, x1, y1, sw / nvalid, sh / nvalid);
  const int64_t ncell = (int64_t)G.gx * G.gy;
  int32_t* cnt = nullptr;
  int64_t* total = nullptr;
  void* tmp = nullptr;
  bool ok = cudaMalloc(&cnt, sizeof(int32_t) * (ncell + 1)) == cudaSuccess &&
            cudaMalloc(&S->r_cellOff, sizeof(int64_t) * (ncell + 1)) == cudaSuccess &&
            cudaMalloc(&total, sizeof(int64_t)) == cudaSuccess &&
            cudaMalloc(&tmp, scan_temp_bytes(ncell + 1)) == cudaSuccess;
  int* d_err = nullptr;
  ok = ok && cudaMalloc(&d_err, sizeof(int)) == cudaSuccess;
  int64_t nent = 0;
  if (ok) {
    cudaMemset(cnt, 0, sizeof(int32_t) * (ncell + 1));
    cudaMemset(d_err, 0, sizeof(int));
    { index_kernel<0><<<blocks_for(n), kThreads>>>(S->r_mbr, S->r_valid, n, G, cnt, nullptr, nullptr); note_launch(); }
    exclusive_scan_i32(cnt, S->r_cellOff, ncell + 1, total, tmp, d_err, 0);
    cudaMemcpy(&nent, total, sizeof(int64_t), cudaMemcpyDeviceToHost);
    ok = cudaMalloc(&S->r_cellList, sizeof(int32_t) * std::max<int64_t>(nent, 1)) == cudaSuccess;
  }
  if (ok) {
    cudaMemset(cnt, 0, sizeof(int32_t) * (ncell + 1));
    G.cellOff = S->r_cellOff;
    { index_kernel<1><<<blocks_for(n), kThreads>>>(S->r_mbr, S->r_valid, n, G, cnt, S->r_cellOff, S->r_cellList); note_launch(); }
    G.cellList = S->r_cellList;
    ok = cudaDeviceSynchronize() == cudaSuccess;
  }
  cudaFree(cnt); cudaFree(total); cudaFree(tmp); cudaFree(d_err);
  if (!ok) {
    cudaGetLastError();
    gcmfgh_serve_close(S.release());
    return GCMFGH_OUT_OF_MEMORY;
  }
  S->grid = G;
  gcmfgh_server* raw = S.release();
  for (int w = 0; w < o.workers; ++w) raw->workers.emplace_back(&gcmfgh_server::worker_main, raw, w);
  *out = raw;
  return GCMFGH_OK;
}

gcmfgh_status gcmfgh_serve_submit(gcmfgh_server* S, const double* xy, int32_t n, int64_t arrival_ns,
                                  uint64_t* ticket) {
  if (!S || !xy || n < 1 || !ticket) return GCMFGH_INVALID_ARGUMENT;
  auto r = std::make_shared<Request>();
  r->ring.assign(xy, xy + 2 * (size_t)n);
  r->n = n;
  r->arrival_ns = arrival_ns > 0 ? arrival_ns : now_ns();
  {
    std::lock_guard<std::mutex> lk(S->mu);
    if (S->stopping) return GCMFGH_INVALID_ARGUMENT;
    uint64_t t = S->next_ticket++;
    S->reqs.emplace(t, r);
    S->queue.push_back(t);
    *ticket = t;
  }
  S->cv_work.notify_one();
  return GCMFGH_OK;
}

static void fill_info(const Request& r, gcmfgh_serve_result* info) {
  if (!info) return;
  info->status = r.status;
  info->n_hits = r.p1 - r.p0;
  info->n_components = r.c1 - r.c0;
  info->n_vertices = r.v1 - r.v0;
  info->n_candidates = r.n_candidates;
  info->arrival_ns = r.arrival_ns;
  info->admitted_ns = r.admitted_ns;
  info->done_ns = r.done_ns;
  info->batch_id = r.batch_id;
  info->batch_queries = r.batch_queries;
}

gcmfgh_status gcmfgh_serve_poll(gcmfgh_server* S, uint64_t ticket, gcmfgh_serve_result* info) {
  if (!S) return GCMFGH_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(S->mu);
  auto it = S->reqs.find(ticket);
  if (it == S->reqs.end()) return GCMFGH_INVALID_ARGUMENT;
  if (!it->second->done) return GCMFGH_NOT_READY;
  fill_info(*it->second, info);
  return GCMFGH_OK;
}

gcmfgh_status gcmfgh_serve_wait(gcmfgh_server* S, uint64_t ticket, int64_t timeout_ms, gcmfgh_serve_result* info) {
  if (!S) return GCMFGH_INVALID_ARGUMENT;
  std::unique_lock<std::mutex> lk(S->mu);
  auto it = S->reqs.find(ticket);
  if (it == S->reqs.end()) return GCMFGH_INVALID_ARGUMENT;
  std::shared_ptr<Request> r = it->second;
  auto ready = [&] { return r->done; };
  if (timeout_ms < 0) S->cv_done.wait(lk, ready);
  else if (!S->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready)) return GCMFGH_NOT_READY;
  fill_info(*r, info);
  return GCMFGH_OK;
}

gcmfgh_status gcmfgh_serve_take(gcmfgh_server* S, uint64_t ticket, int32_t* hit_ids, int32_t* hit_status,
                                int32_t* hit_ncomp, int32_t* comp_size, double* xy) {
  if (!S) return GCMFGH_INVALID_ARGUMENT;
  std::shared_ptr<Request> r;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    auto it = S->reqs.find(ticket);
    if (it == S->reqs.end()) return GCMFGH_INVALID_ARGUMENT;
    if (!it->second->done) return GCMFGH_NOT_READY;
    r = it->second;
    S->reqs.erase(it);
  }
  const BatchOut* o = r->out.get();
  if (!o) return GCMFGH_OK;                       // a failed batch has no results
  const int64_t np = r->p1 - r->p0, nc = r->c1 - r->c0, nv = r->v1 - r->v0;
  if (hit_ids) std::memcpy(hit_ids, o->i32(o->o_o) + r->p0, sizeof(int32_t) * np);
  if (hit_status) std::memcpy(hit_status, o->i32(o->o_st) + r->p0, sizeof(int32_t) * np);
  if (hit_ncomp) std::memcpy(hit_ncomp, o->i32(o->o_nc) + r->p0, sizeof(int32_t) * np);
  if (comp_size) std::memcpy(comp_size, o->i32(o->o_cs) + r->c0, sizeof(int32_t) * nc);
  if (xy) std::memcpy(xy, o->xy() + 2 * r->v0, sizeof(double) * 2 * nv);
  return GCMFGH_OK;
}

gcmfgh_status gcmfgh_serve_stats(gcmfgh_server* S, int64_t* batches, int64_t* queries, int64_t* peak_batch) {
  if (!S) return GCMFGH_INVALID_ARGUMENT;
  if (batches) *batches = S->batches.load();
  if (queries) *queries = S->batched_queries.load();
  if (peak_batch) *peak_batch = S->peak_batch.load();
  return GCMFGH_OK;
}

gcmfgh_status gcmfgh_serve_phases(gcmfgh_server* S, double* ms, int64_t* work) {
  if (!S) return GCMFGH_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(S->stats_mu);
  if (ms) for (int i = 0; i < 7; ++i) ms[i] = S->phase_ms[i];
  if (work) for (int i = 0; i < 4; ++i) work[i] = S->work[i];
  return GCMFGH_OK;
}

gcmfgh_status gcmfgh_serve_close(gcmfgh_server* S) {
  if (!S) return GCMFGH_INVALID_ARGUMENT;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->stopping = true;
  }
  S->cv_work.notify_all();
  for (auto& t : S->workers) t.join();
  cudaSetDevice(S->device);
  cudaFree(S->r_xy); cudaFree(S->r_vnum); cudaFree(S->r_vps); cudaFree(S->r_mbr); cudaFree(S->r_valid);
  cudaFree(S->r_cellOff); cudaFree(S->r_cellList);
  delete S;
  return GCMFGH_OK;
}

}  // extern "C"
