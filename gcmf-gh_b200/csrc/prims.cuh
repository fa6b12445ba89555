// prims.cuh -- device-wide primitives: single-pass exclusive scan with decoupled
// look-back, and a stable LSD radix sort of (u64 key, u32 value) pairs.
//
// These replace the reference's hierarchical multi-pass Hillis-Steele scan
// (GPU_PrefixSum.h:139-706, GPU_Utility.h:62-238) and its decimal LSD radix sort of
// MBR endpoint keys (GPU_RadixSort.h:4-148, GPU_Utility.h:242-290).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace gcmfgh {

struct Arena;   // device workspace (api.cu)

// out[i] = sum(in[0..i-1]) as int64; *total (device pointer, may be null) = sum(in).
// tmp must hold scan_temp_bytes(n) bytes.  err: device error word.
size_t scan_temp_bytes(int64_t n);
void exclusive_scan_i32(const int32_t* in, int64_t* out, int64_t n, int64_t* total,
                        void* tmp, int* err, cudaStream_t s);
void exclusive_scan_i64(const int64_t* in, int64_t* out, int64_t n, int64_t* total,
                        void* tmp, int* err, cudaStream_t s);
void exclusive_scan_u8(const uint8_t* in, int64_t* out, int64_t n, int64_t* total,
                       void* tmp, int* err, cudaStream_t s);

// Stable sort of n (key, value) pairs by the low `key_bits` bits of key (multiple of 8).
// keys/vals are sorted in place; keys_alt/vals_alt are scratch of the same size.
size_t radix_temp_bytes(int64_t n);
void radix_sort_pairs(uint64_t* keys, uint32_t* vals, uint64_t* keys_alt, uint32_t* vals_alt,
                      int64_t n, int key_bits, void* tmp, int* err, cudaStream_t s);

}  // namespace gcmfgh
