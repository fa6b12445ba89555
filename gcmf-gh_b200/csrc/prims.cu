// prims.cu -- single-pass decoupled look-back scan and stable LSD radix sort.
#include "common.cuh"
#include "prims.cuh"

namespace gcmfgh {

namespace {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;   // 2048 elements per tile
// look-back status word: bits 62-63 flag (0 pending, 1 tile aggregate, 2 inclusive
// prefix), bits 0-61 the value in two's complement (|sums| stay below 2^61, so the
// reader sign-extends bit 61).
constexpr uint64_t kFlagAgg = 1ull << 62;
constexpr uint64_t kFlagPrefix = 2ull << 62;
constexpr uint64_t kValueMask = (1ull << 62) - 1;
constexpr long long kSpinLimit = 1ll << 26;

struct ScanState {
  unsigned long long ticket;
  unsigned long long pad[15];
  // followed by one status word per tile
};

template <class T>
__global__ void __launch_bounds__(kScanThreads)
scan_kernel(const T* __restrict__ in, int64_t* __restrict__ out, int64_t n, int64_t* total,
            ScanState* st, int* err) {
  __shared__ int64_t warp_tot[kScanThreads / 32];
  __shared__ int64_t tile_excl;
  __shared__ unsigned long long tile_id_s;
  unsigned long long* status = reinterpret_cast<unsigned long long*>(st + 1);
  if (threadIdx.x == 0) tile_id_s = atomicAdd(&st->ticket, 1ull);
  __syncthreads();
  const int64_t tile = (int64_t)tile_id_s;
  const int64_t base = tile * kScanTile;
  // blocked load: thread t owns elements [base + t*8, base + t*8 + 8)
  int64_t v[kScanItems];
  int64_t acc = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    int64_t i = base + (int64_t)threadIdx.x * kScanItems + k;
    v[k] = (i < n) ? (int64_t)in[i] : 0;
    acc += v[k];
  }
  // block exclusive scan of per-thread sums
  int64_t incl = warp_incl_scan(acc);
  const int w = threadIdx.x >> 5;
  if (lane_id() == 31) warp_tot[w] = incl;
  __syncthreads();
  if (w == 0) {
    int64_t t = (lane_id() < kScanThreads / 32) ? warp_tot[lane_id()] : 0;
    int64_t ti = warp_incl_scan(t);
    if (lane_id() < kScanThreads / 32) warp_tot[lane_id()] = ti - t;   // exclusive
    int64_t agg = __shfl_sync(0xffffffffu, ti, kScanThreads / 32 - 1);
    // publish and look back
    if (lane_id() == 0) {
      unsigned long long word = (tile == 0 ? kFlagPrefix : kFlagAgg) | ((unsigned long long)agg & kValueMask);
      atomicExch(&status[tile], word);
    }
    int64_t excl = 0;
    if (tile > 0) {
      int64_t look = tile - 1;
      bool done = false;
      long long spins = 0;
      while (!done) {
        int64_t idx = look - (int64_t)lane_id();
        unsigned long long word = kFlagPrefix;   // out-of-range lanes act as zero prefixes
        if (idx >= 0) word = *((volatile unsigned long long*)&status[idx]);
        if (idx < 0) word = kFlagPrefix;
        unsigned pending = __ballot_sync(0xffffffffu, (word >> 62) == 0);
        if (pending) {
          if (++spins > kSpinLimit) { if (lane_id() == 0) raise_error(err, DEV_TIMEOUT); break; }
          continue;
        }
        unsigned prefix = __ballot_sync(0xffffffffu, (word >> 62) == 2);
        // lanes up to and including the first (lowest lane) inclusive prefix contribute
        int stop = prefix ? __ffs(prefix) - 1 : 31;
        // the value field holds the low 62 bits of a signed sum: sign-extend it
        int64_t val = ((int)lane_id() <= stop && idx >= 0) ? ((int64_t)(word << 2) >> 2) : 0;
        excl += warp_sum(val);
        if (prefix) done = true;
        else look -= 32;
      }
      if (lane_id() == 0) atomicExch(&status[tile], kFlagPrefix | ((unsigned long long)(excl + agg) & kValueMask));
    }
    if (lane_id() == 0) {
      tile_excl = excl;
      if (total && (base + kScanTile >= n)) *total = excl + agg;
    }
  }
  __syncthreads();
  int64_t run = tile_excl + warp_tot[w] + (incl - acc);
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    int64_t i = base + (int64_t)threadIdx.x * kScanItems + k;
    if (i < n) out[i] = run;
    run += v[k];
  }
}

template <class T>
void scan_impl(const T* in, int64_t* out, int64_t n, int64_t* total, void* tmp, int* err,
               cudaStream_t s) {
  if (n <= 0) {
    if (total) cudaMemsetAsync(total, 0, sizeof(int64_t), s);
    return;
  }
  int64_t tiles = (n + kScanTile - 1) / kScanTile;
  ScanState* st = reinterpret_cast<ScanState*>(tmp);
  cudaMemsetAsync(st, 0, sizeof(ScanState) + tiles * sizeof(unsigned long long), s);
  { scan_kernel<T><<<(unsigned)tiles, kScanThreads, 0, s>>>(in, out, n, total, st, err); note_launch(); }
}

// ------------------------------------------------------------------ radix sort
constexpr int kRadixThreads = 256;
constexpr int kRadixWarps = kRadixThreads / 32;
constexpr int kRadixRounds = 8;                       // items per lane
constexpr int kRadixTile = kRadixThreads * kRadixRounds;   // 2048 keys per block

__global__ void __launch_bounds__(kRadixThreads)
radix_hist_kernel(const uint64_t* __restrict__ keys, int64_t n, int shift, int64_t nblocks,
                  int64_t* __restrict__ hist) {
  __shared__ int cnt[256];
  cnt[threadIdx.x] = 0;
  __syncthreads();
  int64_t base = (int64_t)blockIdx.x * kRadixTile;
  for (int k = threadIdx.x; k < kRadixTile; k += kRadixThreads) {
    int64_t i = base + k;
    if (i < n) atomicAdd(&cnt[(keys[i] >> shift) & 0xff], 1);
  }
  __syncthreads();
  hist[(int64_t)threadIdx.x * nblocks + blockIdx.x] = cnt[threadIdx.x];
}

__global__ void __launch_bounds__(kRadixThreads)
radix_scatter_kernel(const uint64_t* __restrict__ keys, const uint32_t* __restrict__ vals,
                     uint64_t* __restrict__ okeys, uint32_t* __restrict__ ovals, int64_t n,
                     int shift, int64_t nblocks, const int64_t* __restrict__ offs) {
  __shared__ int wcnt[kRadixWarps][256];
  for (int k = threadIdx.x; k < kRadixWarps * 256; k += kRadixThreads) (&wcnt[0][0])[k] = 0;
  __syncthreads();
  const int w = threadIdx.x >> 5;
  const unsigned lane = lane_id();
  const int64_t wbase = (int64_t)blockIdx.x * kRadixTile + (int64_t)w * 32 * kRadixRounds;
  uint64_t key[kRadixRounds];
  uint32_t val[kRadixRounds];
  int rank[kRadixRounds];
  int dig[kRadixRounds];
#pragma unroll
  for (int r = 0; r < kRadixRounds; ++r) {
    int64_t i = wbase + r * 32 + lane;
    bool ok = i < n;
    key[r] = ok ? keys[i] : 0;
    val[r] = ok ? vals[i] : 0;
    int d = ok ? (int)((key[r] >> shift) & 0xff) : 256 + (int)lane;   // invalid lanes: unique
    dig[r] = d;
    unsigned peers = __match_any_sync(0xffffffffu, d);
    int before = __popc(peers & lanemask_lt());
    int b = (ok) ? wcnt[w][d] : 0;
    __syncwarp();
    if (ok && before == 0) wcnt[w][d] = b + __popc(peers);
    __syncwarp();
    rank[r] = b + before;
  }
  __syncthreads();
  // per digit: exclusive prefix over warps
  {
    int d = threadIdx.x;
    int run = 0;
    for (int ww = 0; ww < kRadixWarps; ++ww) { int t = wcnt[ww][d]; wcnt[ww][d] = run; run += t; }
  }
  __syncthreads();
#pragma unroll
  for (int r = 0; r < kRadixRounds; ++r) {
    int64_t i = wbase + r * 32 + lane;
    if (i < n) {
      int d = dig[r];
      int64_t pos = offs[(int64_t)d * nblocks + blockIdx.x] + wcnt[w][d] + rank[r];
      okeys[pos] = key[r];
      ovals[pos] = val[r];
    }
  }
}

}  // namespace

size_t scan_temp_bytes(int64_t n) {
  int64_t tiles = (n + kScanTile - 1) / kScanTile;
  return sizeof(ScanState) + (size_t)(tiles + 1) * sizeof(unsigned long long);
}

void exclusive_scan_i32(const int32_t* in, int64_t* out, int64_t n, int64_t* total, void* tmp,
                        int* err, cudaStream_t s) {
  scan_impl<int32_t>(in, out, n, total, tmp, err, s);
}
void exclusive_scan_i64(const int64_t* in, int64_t* out, int64_t n, int64_t* total, void* tmp,
                        int* err, cudaStream_t s) {
  scan_impl<int64_t>(in, out, n, total, tmp, err, s);
}
void exclusive_scan_u8(const uint8_t* in, int64_t* out, int64_t n, int64_t* total, void* tmp,
                       int* err, cudaStream_t s) {
  scan_impl<uint8_t>(in, out, n, total, tmp, err, s);
}

size_t radix_temp_bytes(int64_t n) {
  int64_t nb = (n + kRadixTile - 1) / kRadixTile;
  int64_t h = 256 * nb;
  return 2 * (size_t)h * sizeof(int64_t) + scan_temp_bytes(h) + 256;
}

void radix_sort_pairs(uint64_t* keys, uint32_t* vals, uint64_t* keys_alt, uint32_t* vals_alt,
                      int64_t n, int key_bits, void* tmp, int* err, cudaStream_t s) {
  if (n <= 1) return;
  int64_t nb = (n + kRadixTile - 1) / kRadixTile;
  int64_t h = 256 * nb;
  int64_t* hist = reinterpret_cast<int64_t*>(tmp);
  int64_t* offs = hist + h;
  void* stmp = reinterpret_cast<char*>(offs + h);
  uint64_t* ka = keys;
  uint32_t* va = vals;
  uint64_t* kb = keys_alt;
  uint32_t* vb = vals_alt;
  int passes = (key_bits + 7) / 8;
  for (int p = 0; p < passes; ++p) {
    int shift = 8 * p;
    { radix_hist_kernel<<<(unsigned)nb, kRadixThreads, 0, s>>>(ka, n, shift, nb, hist); note_launch(); }
    exclusive_scan_i64(hist, offs, h, nullptr, stmp, err, s);
    { radix_scatter_kernel<<<(unsigned)nb, kRadixThreads, 0, s>>>(ka, va, kb, vb, n, shift, nb, offs); note_launch(); }
    uint64_t* tk = ka; ka = kb; kb = tk;
    uint32_t* tv = va; va = vb; vb = tv;
  }
  if (ka != keys) {
    cudaMemcpyAsync(keys, ka, n * sizeof(uint64_t), cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(vals, va, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s);
  }
}

}  // namespace gcmfgh

// ============================================================================
// Allocation-free scan.  Some callers cannot let a library call cudaMalloc: a host
// engine that accounts for every byte of device memory through its own pool, or a
// latency-sensitive loop that must not hit cudaMalloc's implicit device-wide
// synchronisation.  This variant runs the same look-back scan kernel as
// exclusive_scan_i32, but its look-back scratch (the tile ticket, one status word per
// 2,048-element tile and the error word) lives in the file-scope device array below,
// which every GPU that loads the library holds until the process exits (about 66 KB).
#include <cstdio>
#include <mutex>
#include "../../include/gcmfgh.h"

namespace {

constexpr int64_t kNoAllocMaxTiles = GCMFGH_NOALLOC_SCAN_MAX_ELEMENTS / gcmfgh::kScanTile;
constexpr int64_t kNoAllocHeaderWords = sizeof(gcmfgh::ScanState) / sizeof(unsigned long long);
static_assert(GCMFGH_NOALLOC_SCAN_MAX_ELEMENTS % gcmfgh::kScanTile == 0, "whole tiles");

// [header (ticket) | one status word per tile | error word]
static __device__ __align__(256) unsigned long long
    g_noalloc_scan_scratch[kNoAllocHeaderWords + kNoAllocMaxTiles + 8];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
unsigned long long* g_noalloc_ptr[kMaxDevices] = {};

// The device address of the scratch array on the current device.  Host code may not use
// the array's name as an address (it is a host-side stand-in), so the address is looked
// up once per device with that device current and cached.
unsigned long long* noalloc_scratch(int dev) {
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scan_scratch) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    g_noalloc_ptr[dev] = static_cast<unsigned long long*>(p);
  }
  return g_noalloc_ptr[dev];
}

}  // namespace

extern "C" gcmfgh_status gcmfgh_exclusive_scan_i32_noalloc(const int32_t* d_in, int64_t* d_out, int64_t n,
                                                           int64_t* d_total, void* stream) {
  if (n < 0 || (n > 0 && (!d_in || !d_out))) return GCMFGH_INVALID_ARGUMENT;
  if (n > GCMFGH_NOALLOC_SCAN_MAX_ELEMENTS) {
    fprintf(stderr, "gcmfgh_exclusive_scan_i32_noalloc: n = %lld exceeds the maximum of %lld elements\n",
            (long long)n, (long long)GCMFGH_NOALLOC_SCAN_MAX_ELEMENTS);
    return GCMFGH_INVALID_ARGUMENT;
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return GCMFGH_CUDA_ERROR;
  unsigned long long* scratch = noalloc_scratch(dev);
  if (!scratch) return GCMFGH_CUDA_ERROR;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int* err = reinterpret_cast<int*>(scratch + kNoAllocHeaderWords + kNoAllocMaxTiles);
  const int64_t tiles = (n + gcmfgh::kScanTile - 1) / gcmfgh::kScanTile;
  // the array keeps the previous call's contents: zero the ticket, the status words this
  // call uses and the error word
  if (cudaMemsetAsync(scratch, 0, (kNoAllocHeaderWords + tiles) * sizeof(unsigned long long), s) != cudaSuccess ||
      cudaMemsetAsync(err, 0, sizeof(int), s) != cudaSuccess)
    return GCMFGH_CUDA_ERROR;
  if (n == 0) {
    if (d_total && cudaMemsetAsync(d_total, 0, sizeof(int64_t), s) != cudaSuccess) return GCMFGH_CUDA_ERROR;
  } else {
    gcmfgh::scan_kernel<int32_t><<<(unsigned)tiles, gcmfgh::kScanThreads, 0, s>>>(
        d_in, d_out, n, d_total, reinterpret_cast<gcmfgh::ScanState*>(scratch), err);
    gcmfgh::note_launch();
    // the launch's own status, taken right after it
    if (cudaGetLastError() != cudaSuccess) return GCMFGH_CUDA_ERROR;
  }
  int h_err = 0;
  if (cudaMemcpyAsync(&h_err, err, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess) return GCMFGH_CUDA_ERROR;
  if (cudaStreamSynchronize(s) != cudaSuccess) return GCMFGH_CUDA_ERROR;
  return h_err ? GCMFGH_DEVICE_ERROR : GCMFGH_OK;
}
