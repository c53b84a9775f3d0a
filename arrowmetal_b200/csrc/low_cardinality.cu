// Low-cardinality integer keys: a key column with at most LOWCARD_MAX distinct value keys is sorted
// by its dense rank instead of its values.
//
// Ranks are taken over the encoded keys (the key map, the direction included), so ascending order of
// the ranks is the key's own order and equal values share a rank; null rows keep their validity, so
// the null placement is unchanged. A rank fits one 8-bit digit: one digit pass instead of up to four
// (32-bit keys) or eight (64-bit). The rank column replaces the key only where the key's values are
// not needed back (argsort and lexsort, not a sorted copy of the key itself).
//
// Three steps on the device and one small readback: a probe counts the distinct value keys (each
// block keeps the keys it has seen in a shared-memory table and adds only new ones to a global table;
// it gives up as soon as more than LOWCARD_MAX are found); one block ranks the distinct keys; one
// pass writes every row's rank. A column found to hold more keys is marked on its values buffer, so
// its later sorts (a served table's requests, slices of it) skip the probe and its readback.
#include <algorithm>

#include "am_internal.h"
#include "key_encode.cuh"

namespace am {
namespace rs {
namespace {

constexpr uint32_t LOWCARD_MAX = 256;
constexpr uint32_t SLOTS = 1024;                 // global table: open addressing, at most 1/4 full
constexpr uint32_t BLOCK_SLOTS = 512;            // each block's table of the keys it has seen
constexpr unsigned long long EMPTY = ~0ull;
constexpr int PROBE_THREADS = 256, PROBE_ITEMS = 8;
constexpr int64_t LOWCARD_MIN_ROWS = int64_t(1) << 22;

struct Table {
  unsigned long long keys[SLOTS];
  uint32_t rank[SLOTS];
  uint32_t count;                                // distinct value keys inserted
  uint32_t overflow;                             // more than LOWCARD_MAX
  uint32_t has_max;                              // the all-ones key, which the table cannot hold (EMPTY)
  uint32_t max_rank;                             // its rank: above every key in the table
};

__device__ __forceinline__ uint32_t hash_key(unsigned long long k, uint32_t mask) {
  k ^= k >> 33;
  k *= 0xff51afd7ed558ccdull;
  k ^= k >> 33;
  return uint32_t(k) & mask;
}

// Inserts `k` into the global table unless present; true when it was new. Once more than LOWCARD_MAX
// keys are in, nothing more is inserted (the table never fills).
__device__ bool global_insert(Table* t, unsigned long long k) {
  if (*reinterpret_cast<volatile uint32_t*>(&t->count) >= LOWCARD_MAX) {
    atomicExch(&t->overflow, 1u);
    return false;
  }
  uint32_t h = hash_key(k, SLOTS - 1);
  for (uint32_t probe = 0; probe < SLOTS; probe++, h = (h + 1) & (SLOTS - 1)) {
    const unsigned long long old = atomicCAS(&t->keys[h], EMPTY, k);
    if (old == EMPTY) {
      if (atomicAdd(&t->count, 1u) >= LOWCARD_MAX) atomicExch(&t->overflow, 1u);
      return true;
    }
    if (old == k) return false;
  }
  atomicExch(&t->overflow, 1u);                  // unreachable while the table is at most 1/4 full
  return false;
}

template <typename KeyT>
__global__ void __launch_bounds__(PROBE_THREADS) distinct_probe_kernel(const __grid_constant__ ColView col, uint64_t n,
                                                                       Table* __restrict__ t) {
  __shared__ unsigned long long seen[BLOCK_SLOTS];
  __shared__ uint32_t s_count, s_stop;
  for (uint32_t i = threadIdx.x; i < BLOCK_SLOTS; i += PROBE_THREADS) seen[i] = EMPTY;
  if (threadIdx.x == 0) s_count = 0;
  __syncthreads();
  constexpr uint64_t CHUNK = uint64_t(PROBE_THREADS) * PROBE_ITEMS;
  for (uint64_t base = uint64_t(blockIdx.x) * CHUNK; base < n; base += uint64_t(gridDim.x) * CHUNK) {
    // Every block stops once any block has seen too many keys (the decision is the block's, taken by
    // one thread, so every thread leaves the loop at the same round).
    if (threadIdx.x == 0)
      s_stop = (*reinterpret_cast<volatile uint32_t*>(&t->overflow) || s_count > LOWCARD_MAX) ? 1u : 0u;
    __syncthreads();
    if (s_stop) break;
    uint32_t row[PROBE_ITEMS];
    uint32_t ok = 0;
#pragma unroll
    for (int i = 0; i < PROBE_ITEMS; i++) {
      const uint64_t g = base + uint64_t(i) * PROBE_THREADS + threadIdx.x;
      row[i] = uint32_t(g);
      if (g < n) ok |= 1u << i;
    }
    KeyT key[PROBE_ITEMS];
    int cat[PROBE_ITEMS];
    encode_rows<KeyT, PROBE_ITEMS>(col, row, ok, key, cat);
#pragma unroll
    for (int i = 0; i < PROBE_ITEMS; i++) {
      // Past LOWCARD_MAX keys of its own a block inserts nothing more (its table stays under half full).
      if (!((ok >> i) & 1u) || cat[i] != 0 || *reinterpret_cast<volatile uint32_t*>(&s_count) > LOWCARD_MAX) continue;
      const unsigned long long k = (unsigned long long)key[i];
      if (k == EMPTY) {
        if (atomicCAS(&t->has_max, 0u, 1u) == 0u && atomicAdd(&t->count, 1u) >= LOWCARD_MAX)
          atomicExch(&t->overflow, 1u);
        continue;
      }
      uint32_t h = hash_key(k, BLOCK_SLOTS - 1);
      for (uint32_t probe = 0; probe < BLOCK_SLOTS; probe++, h = (h + 1) & (BLOCK_SLOTS - 1)) {
        const unsigned long long cur = seen[h];
        if (cur == k) break;
        if (cur == EMPTY) {
          const unsigned long long old = atomicCAS(&seen[h], EMPTY, k);
          if (old == EMPTY) {
            atomicAdd(&s_count, 1u);
            global_insert(t, k);
            break;
          }
          if (old == k) break;
        }
      }
    }
    __syncthreads();
  }
  // A block that has seen more than LOWCARD_MAX keys of its own says so.
  if (threadIdx.x == 0 && s_count > LOWCARD_MAX) atomicExch(&t->overflow, 1u);
}

// One block: each distinct key's rank is the number of distinct keys below it.
__global__ void __launch_bounds__(256) rank_distinct_kernel(Table* __restrict__ t) {
  __shared__ unsigned long long keys[LOWCARD_MAX];
  __shared__ uint32_t slot_of[LOWCARD_MAX];
  __shared__ uint32_t k;
  if (threadIdx.x == 0) k = 0;
  __syncthreads();
  for (uint32_t s = threadIdx.x; s < SLOTS; s += blockDim.x) {
    const unsigned long long v = t->keys[s];
    if (v == EMPTY) continue;
    const uint32_t at = atomicAdd(&k, 1u);
    if (at < LOWCARD_MAX) {
      keys[at] = v;
      slot_of[at] = s;
    }
  }
  __syncthreads();
  const uint32_t m = min(k, LOWCARD_MAX);
  if (threadIdx.x == 0) t->max_rank = m;
  for (uint32_t i = threadIdx.x; i < m; i += blockDim.x) {
    uint32_t r = 0;
    for (uint32_t j = 0; j < m; j++) r += keys[j] < keys[i] ? 1u : 0u;
    t->rank[slot_of[i]] = r;
  }
}

template <typename KeyT>
__global__ void __launch_bounds__(256) rank_column_kernel(const __grid_constant__ ColView col, uint64_t n,
                                                          const Table* __restrict__ t, uint8_t* __restrict__ out,
                                                          uint32_t* __restrict__ err) {
  constexpr int ITEMS = 8;
  for (uint64_t base = uint64_t(blockIdx.x) * 256 * ITEMS; base < n; base += uint64_t(gridDim.x) * 256 * ITEMS) {
    uint32_t row[ITEMS];
    uint32_t ok = 0;
#pragma unroll
    for (int i = 0; i < ITEMS; i++) {
      const uint64_t g = base + uint64_t(i) * 256 + threadIdx.x;
      row[i] = uint32_t(g);
      if (g < n) ok |= 1u << i;
    }
    KeyT key[ITEMS];
    int cat[ITEMS];
    encode_rows<KeyT, ITEMS>(col, row, ok, key, cat);
#pragma unroll
    for (int i = 0; i < ITEMS; i++) {
      if (!((ok >> i) & 1u)) continue;
      uint8_t r = 0;
      if (cat[i] == 0 && (unsigned long long)key[i] == EMPTY) {
        r = uint8_t(t->max_rank);
      } else if (cat[i] == 0) {
        const unsigned long long k = (unsigned long long)key[i];
        uint32_t h = hash_key(k, SLOTS - 1);
        uint32_t probe = 0;
        for (; probe < SLOTS; probe++, h = (h + 1) & (SLOTS - 1))
          if (t->keys[h] == k) break;
        if (probe == SLOTS) atomicOr(err, ERR_BOUNDS);   // every value key was inserted by the probe
        else r = uint8_t(t->rank[h]);
      }
      out[row[i]] = r;
    }
  }
}

bool integer_key(int pt) {
  return pt == PT_I32 || pt == PT_U32 || pt == PT_I64 || pt == PT_U64;
}

}  // namespace
}  // namespace rs

am_array* low_cardinality_ranks(const SortKey& k, cudaStream_t s) {
  using namespace rs;
  const am_array* a = k.col;
  const int64_t n = a->length;
  if (n < LOWCARD_MIN_ROWS || a->dictionary || !integer_key(a->pt) || n >= (int64_t(1) << 32) || !a->values) return nullptr;
  if (a->values->many_values.load(std::memory_order_relaxed)) return nullptr;
  const ColView cv = make_view(k);
  Table* t = static_cast<Table*>(dmalloc(sizeof(Table), s));
  AM_CUDA(cudaMemsetAsync(t, 0xFF, sizeof(t->keys), s));
  AM_CUDA(cudaMemsetAsync(reinterpret_cast<char*>(t) + offsetof(Table, rank), 0, sizeof(Table) - offsetof(Table, rank), s));
  const int grid = device().sm_count * 8;
  {
    KernelTimer kt("low_cardinality_probe", s);
    if (pt_key_bytes(a->pt) == 8) distinct_probe_kernel<uint64_t><<<grid, PROBE_THREADS, 0, s>>>(cv, uint64_t(n), t);
    else distinct_probe_kernel<uint32_t><<<grid, PROBE_THREADS, 0, s>>>(cv, uint64_t(n), t);
    AM_CUDA(cudaGetLastError());
  }
  uint32_t host[2] = {0, 0};
  AM_CUDA(cudaMemcpyAsync(host, &t->count, sizeof(host), cudaMemcpyDeviceToHost, s));
  AM_CUDA(cudaStreamSynchronize(s));
  if (host[1] != 0 || host[0] == 0 || host[0] > LOWCARD_MAX) {
    if (host[1] != 0 || host[0] > LOWCARD_MAX) a->values->many_values.store(true, std::memory_order_relaxed);
    dfree(t, s);
    return nullptr;
  }
  am_array* r = new_array(PT_U8, "C", n);
  try {
    r->values = DevBuffer::alloc(size_t(n) + 16, s);
    r->validity = a->null_count != 0 ? a->validity : nullptr;
    r->validity_offset = a->validity_offset;
    r->null_count = a->null_count;
    r->last_stream = s;
    KernelTimer kt("low_cardinality_rank", s);
    rank_distinct_kernel<<<1, 256, 0, s>>>(t);
    AM_CUDA(cudaGetLastError());
    const int cgrid = int(std::min<int64_t>((n + 2047) / 2048, int64_t(device().sm_count) * 8));
    if (pt_key_bytes(a->pt) == 8)
      rank_column_kernel<uint64_t><<<cgrid, 256, 0, s>>>(cv, uint64_t(n), t, static_cast<uint8_t*>(r->values->ptr), stream_scratch(s, 0).err);
    else
      rank_column_kernel<uint32_t><<<cgrid, 256, 0, s>>>(cv, uint64_t(n), t, static_cast<uint8_t*>(r->values->ptr), stream_scratch(s, 0).err);
    AM_CUDA(cudaGetLastError());
  } catch (...) {
    dfree(t, s);
    am::release(r);
    throw;
  }
  dfree(t, s);
  return r;
}

}  // namespace am
