// Device-wide sort / scan / run-length primitives (sbp_sort.cu).
#pragma once
#include <cuda_runtime.h>

#include <algorithm>

namespace sbpb {

// Exclusive scan of n unsigned ints into int64 out; `partial` needs scan_partial_capacity(sms).
void exclusive_scan_u32(const unsigned* in, long long* out, long long n, unsigned long long* partial, int sms,
                        cudaStream_t s);
long long scan_partial_capacity(int sms);

// Stable LSD radix sort of the low `bits` bits of n 64-bit keys; `tmp` has n entries, `hist`
// radix_hist_capacity(n, sms) entries.  *result points at keys or tmp (the sorted copy).
void radix_sort_u64(unsigned long long* keys, unsigned long long* tmp, long long n, int bits, unsigned* hist,
                    unsigned long long* partial, int sms, cudaStream_t s, unsigned long long** result);
long long radix_hist_capacity(long long n, int sms);

// Run-length encoding of sorted keys: flags[n] and pos[n] scratch; ukeys/heads receive the
// unique keys and the index of each run's first element; the run count is pos[n-1]+flags[n-1].
void rle(const unsigned long long* keys, long long n, unsigned* flags, long long* pos, unsigned long long* ukeys,
         long long* heads, unsigned long long* partial, int sms, cudaStream_t s);

}  // namespace sbpb
