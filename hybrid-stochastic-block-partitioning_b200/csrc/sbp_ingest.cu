// Graph ingest on the device: the Graph constructor of the reference (src/graph.cpp:123-213,
// duplicate edges dropped as utils::insert_nodup does, src/utils.cpp:52-60) from an edge list
// already in device memory.
//  1. k_ingest_first: a hash table over the (src, dst) pairs keeps the smallest edge index of
//     each pair, so edge i survives exactly when it is the pair's first occurrence;
//  2. k_ingest_keep: every surviving edge writes the key (src << ib | i) for the out-lists and,
//     unless it is a self loop, (dst << ib | i) for the in-lists, and counts the degrees;
//  3. the engine's radix sort orders the keys by vertex, then by edge index (input order), which
//     is the order of the reference's adjacency lists;
//  4. k_ingest_fill writes the neighbour (and the source, for out_src) of every sorted key.
#include "sbp_kernels.cuh"

namespace sbpb {

__device__ __forceinline__ unsigned long long pair_slot(unsigned long long key, int tbits) {
  return (key * 0x9E3779B97F4A7C15ull) >> (64 - tbits);
}

// Insert every edge's pair; first[slot] = smallest edge index of the pair.  The table has at
// least twice as many slots as edges, so a probe always ends; the bound is a guard.  An endpoint
// out of range sets *bad and the edge is skipped.
__global__ void k_ingest_first(const int* __restrict__ src, const int* __restrict__ dst, long long n, int V,
                               unsigned long long* keys, int* first, int tbits, int* bad) {
  const unsigned long long mask = (1ull << tbits) - 1;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const int s = src[i], d = dst[i];
    if (s < 0 || s >= V || d < 0 || d >= V) {
      atomicOr(bad, 1);
      continue;
    }
    const unsigned long long key = (unsigned long long)s * (unsigned long long)V + (unsigned long long)d;
    unsigned long long h = pair_slot(key, tbits);
    for (unsigned long long probe = 0; probe <= mask; ++probe) {
      unsigned long long k = *(volatile unsigned long long*)(keys + h);
      if (k == ~0ull) {
        const unsigned long long prev = atomicCAS(keys + h, ~0ull, key);
        k = prev == ~0ull ? key : prev;
      }
      if (k == key) {
        atomicMin(first + h, (int)i);
        break;
      }
      h = (h + 1) & mask;
    }
  }
}

// Surviving edges: keys for the two sorts, degree counts and self-loop flags.  ctr[0] / ctr[1]
// count the out / in keys.
__global__ void k_ingest_keep(const int* __restrict__ src, const int* __restrict__ dst, long long n, int V,
                              const unsigned long long* __restrict__ keys, const int* __restrict__ first, int tbits,
                              int ib, unsigned long long* out_keys, unsigned long long* in_keys,
                              unsigned long long* ctr, unsigned* out_cnt, unsigned* in_cnt, unsigned char* self) {
  const unsigned long long mask = (1ull << tbits) - 1;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const int s = src[i], d = dst[i];
    if (s < 0 || s >= V || d < 0 || d >= V) continue;
    const unsigned long long key = (unsigned long long)s * (unsigned long long)V + (unsigned long long)d;
    unsigned long long h = pair_slot(key, tbits);
    bool keep = false;
    for (unsigned long long probe = 0; probe <= mask; ++probe) {
      if (keys[h] == key) {
        keep = first[h] == (int)i;
        break;
      }
      h = (h + 1) & mask;
    }
    if (!keep) continue;
    out_keys[atomicAdd(ctr, 1ull)] = ((unsigned long long)s << ib) | (unsigned long long)i;
    atomicAdd(out_cnt + s, 1u);
    if (s == d) {
      self[s] = 1;
    } else {
      in_keys[atomicAdd(ctr + 1, 1ull)] = ((unsigned long long)d << ib) | (unsigned long long)i;
      atomicAdd(in_cnt + d, 1u);
    }
  }
}

// Adjacency entries from the sorted keys: idx[p] = other[edge of key p] (dst for the out-lists,
// src for the in-lists) and, when given, srcs[p] = the key's vertex.
__global__ void k_ingest_fill(const unsigned long long* __restrict__ sorted, long long m, int ib,
                              const int* __restrict__ other, int* idx, int* srcs) {
  const unsigned long long imask = (1ull << ib) - 1;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < m; p += stride) {
    const unsigned long long k = sorted[p];
    idx[p] = other[k & imask];
    if (srcs) srcs[p] = (int)(k >> ib);
  }
}

// Exclusive-scan output (int64) to the int offsets of a CSR.
__global__ void k_ingest_ptr(const long long* __restrict__ in, int* out, long long n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    out[i] = (int)in[i];
}

__global__ void k_iota(int* out, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out[i] = i;
}

}  // namespace sbpb
