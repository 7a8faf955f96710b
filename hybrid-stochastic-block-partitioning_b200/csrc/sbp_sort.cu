// Device-wide primitives for the sparse block matrix: a stable LSD radix sort of 64-bit keys,
// a multi-CTA exclusive scan of ints and run-length encoding of sorted keys.  Written for this
// engine (no library sort); used to rebuild the block matrix from the edge list when B is large.
#include "sbp_sort.cuh"

namespace sbpb {

constexpr int kSortThreads = 256;
constexpr int kRadixBits = 8;
constexpr int kRadix = 1 << kRadixBits;

// Per-CTA digit histogram of a contiguous tile; hist is digit-major: hist[d * G + cta].
__global__ void k_radix_hist(const unsigned long long* __restrict__ keys, long long n, long long tile, int shift,
                             unsigned* hist) {
  __shared__ unsigned h[kRadix];
  for (int i = threadIdx.x; i < kRadix; i += blockDim.x) h[i] = 0;
  __syncthreads();
  const long long b0 = (long long)blockIdx.x * tile, b1 = min(n, b0 + tile);
  for (long long i = b0 + threadIdx.x; i < b1; i += blockDim.x) atomicAdd(&h[(keys[i] >> shift) & (kRadix - 1)], 1u);
  __syncthreads();
  for (int i = threadIdx.x; i < kRadix; i += blockDim.x) hist[(size_t)i * gridDim.x + blockIdx.x] = h[i];
}

// Stable scatter: elements of a tile keep their order inside each digit.  Each chunk of
// blockDim elements ranks its elements per warp (match_any) and across warps (per-digit
// exclusive prefix over warps in warp order).
__global__ void k_radix_scatter(const unsigned long long* __restrict__ in, unsigned long long* __restrict__ out,
                                long long n, long long tile, int shift, const unsigned* __restrict__ offsets) {
  __shared__ unsigned base[kRadix];
  __shared__ unsigned tot[kRadix];
  __shared__ unsigned wcount[kSortThreads / 32][kRadix];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int nw = blockDim.x >> 5;
  for (int i = threadIdx.x; i < kRadix; i += blockDim.x) base[i] = offsets[(size_t)i * gridDim.x + blockIdx.x];
  const long long b0 = (long long)blockIdx.x * tile, b1 = min(n, b0 + tile);
  for (long long c0 = b0; c0 < b1; c0 += blockDim.x) {
    for (int i = threadIdx.x; i < nw * kRadix; i += blockDim.x) (&wcount[0][0])[i] = 0;
    __syncthreads();
    const long long i = c0 + threadIdx.x;
    const bool valid = i < b1;
    const unsigned long long k = valid ? in[i] : 0ull;
    const int d = valid ? (int)((k >> shift) & (kRadix - 1)) : -1;
    const unsigned peers = __match_any_sync(0xffffffffu, d);
    const unsigned rank_in_warp = __popc(peers & ((1u << lane) - 1));
    if (valid && (__ffs(peers) - 1) == lane) wcount[w][d] = __popc(peers);
    __syncthreads();
    for (int dd = threadIdx.x; dd < kRadix; dd += blockDim.x) {
      unsigned run = 0;
      for (int ww = 0; ww < nw; ++ww) {
        const unsigned c = wcount[ww][dd];
        wcount[ww][dd] = run;
        run += c;
      }
      tot[dd] = run;
    }
    __syncthreads();
    if (valid) out[base[d] + wcount[w][d] + rank_in_warp] = k;
    __syncthreads();
    for (int dd = threadIdx.x; dd < kRadix; dd += blockDim.x) base[dd] += tot[dd];
    __syncthreads();
  }
}

// Exclusive scan of digit-major histograms (and of any unsigned array) in three phases.
__global__ void k_scan_partials(const unsigned* __restrict__ in, long long n, long long tile,
                                unsigned long long* partial) {
  __shared__ unsigned long long red[32];
  const long long b0 = (long long)blockIdx.x * tile, b1 = min(n, b0 + tile);
  unsigned long long acc = 0;
  for (long long i = b0 + threadIdx.x; i < b1; i += blockDim.x) acc += in[i];
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long t = 0;
    for (int j = 0; j < (int)(blockDim.x >> 5); ++j) t += red[j];
    partial[blockIdx.x] = t;
  }
}

__global__ void k_scan_top(unsigned long long* partial, int g) {   // single thread: g is small
  if (threadIdx.x || blockIdx.x) return;
  unsigned long long run = 0;
  for (int i = 0; i < g; ++i) {
    const unsigned long long c = partial[i];
    partial[i] = run;
    run += c;
  }
  partial[g] = run;
}

// out[i] = partial[cta] + exclusive prefix inside the tile (tile-serial chunks of blockDim).
// in and out may be the same array (the radix sort scans its histogram in place): every
// element is read by the thread that later writes it, so neither pointer is __restrict__.
template <class OutT>
__global__ void k_scan_down(const unsigned* in, OutT* out, long long n, long long tile,
                            const unsigned long long* __restrict__ partial) {
  __shared__ unsigned long long wsum[32];
  __shared__ unsigned long long carry;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (threadIdx.x == 0) carry = partial[blockIdx.x];
  __syncthreads();
  const long long b0 = (long long)blockIdx.x * tile, b1 = min(n, b0 + tile);
  for (long long c0 = b0; c0 < b1; c0 += blockDim.x) {
    const long long i = c0 + threadIdx.x;
    const unsigned long long v = i < b1 ? in[i] : 0;
    unsigned long long incl = v;
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned long long y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    if (lane == 31) wsum[w] = incl;
    __syncthreads();
    if (w == 0) {
      unsigned long long t = lane < (int)(blockDim.x >> 5) ? wsum[lane] : 0;
      for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long y = __shfl_up_sync(0xffffffffu, t, o);
        if (lane >= o) t += y;
      }
      wsum[lane] = t;
    }
    __syncthreads();
    const unsigned long long before = carry + (w > 0 ? wsum[w - 1] : 0);
    if (i < b1) out[i] = (OutT)(before + incl - v);
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) carry = before + incl;
    __syncthreads();
  }
}

// Run-length encoding of sorted keys: head flags.
__global__ void k_rle_flags(const unsigned long long* __restrict__ keys, long long n, unsigned* flags) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    flags[i] = (i == 0 || keys[i] != keys[i - 1]) ? 1u : 0u;
}

// Unique keys and their counts: run j spans [head_j, head_{j+1}).
__global__ void k_rle_emit(const unsigned long long* __restrict__ keys, long long n, const unsigned* __restrict__ flags,
                           const long long* __restrict__ pos, unsigned long long* ukeys, long long* heads) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    if (flags[i]) {
      ukeys[pos[i]] = keys[i];
      heads[pos[i]] = i;
    }
}

static int scan_grid(long long n, int sms) {
  long long g = (n + 4095) / 4096;
  if (g < 1) g = 1;
  if (g > 4LL * sms) g = 4LL * sms;
  return (int)g;
}

void exclusive_scan_u32(const unsigned* in, long long* out, long long n, unsigned long long* partial, int sms,
                        cudaStream_t s) {
  const int g = scan_grid(n, sms);
  const long long tile = (n + g - 1) / g;
  k_scan_partials<<<g, 256, 0, s>>>(in, n, tile, partial);
  k_scan_top<<<1, 32, 0, s>>>(partial, g);
  k_scan_down<long long><<<g, 256, 0, s>>>(in, out, n, tile, partial);
}

long long scan_partial_capacity(int sms) { return 4LL * sms + 1; }

void radix_sort_u64(unsigned long long* keys, unsigned long long* tmp, long long n, int bits, unsigned* hist,
                    unsigned long long* partial, int sms, cudaStream_t s, unsigned long long** result) {
  unsigned long long* a = keys;
  unsigned long long* b = tmp;
  const int g = (int)std::min<long long>(std::max<long long>((n + 8191) / 8192, 1), 2LL * sms);
  const long long tile = (n + g - 1) / g;
  for (int shift = 0; shift < bits; shift += kRadixBits) {
    k_radix_hist<<<g, kSortThreads, 0, s>>>(a, n, tile, shift, hist);
    const long long hn = (long long)kRadix * g;
    const int sg = scan_grid(hn, sms);
    const long long stile = (hn + sg - 1) / sg;
    k_scan_partials<<<sg, 256, 0, s>>>(hist, hn, stile, partial);
    k_scan_top<<<1, 32, 0, s>>>(partial, sg);
    k_scan_down<unsigned><<<sg, 256, 0, s>>>(hist, hist, hn, stile, partial);
    k_radix_scatter<<<g, kSortThreads, 0, s>>>(a, b, n, tile, shift, hist);
    std::swap(a, b);
  }
  *result = a;
}

long long radix_hist_capacity(long long n, int sms) {
  const long long g = std::min<long long>(std::max<long long>((n + 8191) / 8192, 1), 2LL * sms);
  return (long long)kRadix * g;
}

void rle(const unsigned long long* keys, long long n, unsigned* flags, long long* pos, unsigned long long* ukeys,
         long long* heads, unsigned long long* partial, int sms, cudaStream_t s) {
  const int g = (int)std::min<long long>(std::max<long long>((n + 255) / 256, 1), 8LL * sms);
  k_rle_flags<<<g, 256, 0, s>>>(keys, n, flags);
  exclusive_scan_u32(flags, pos, n, partial, sms, s);
  k_rle_emit<<<g, 256, 0, s>>>(keys, n, flags, pos, ukeys, heads);
}

}  // namespace sbpb
