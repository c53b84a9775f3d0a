/* CPU oracle for the full-sort path: TEST INFRASTRUCTURE ONLY.
 *
 * This file is the checker, never the product: only the tests, the smoke check and the benchmark's
 * CPU-baseline leg load it. It restates, in plain C, the reference algorithm of ArrowMetal 0.6.1's
 * sort path as its Metal code runs it:
 *
 *   key maps          Sources/ArrowMetal/Kernels/SortSource.swift:131-190 (key_from_{i32,u32,f32,
 *                     i64,u64,f64}, _total, _nanlargest); narrow ints widen to int32 (Sort.swift:220-221)
 *   NaN / zero keys   Sources/ArrowMetal/Kernels/Sort.swift:32-43 (nanKey: after +inf ascending,
 *                     all-ones descending, the plain complement for nan_largest)
 *   partition         SortSource.swift:226-330 and Sort.swift:224-231,317-341: a stable split into
 *                     values / NaN / nulls, the NaN block only for the ieee order at the start;
 *                     arrangement [values][NaN][nulls] at the end, [nulls][NaN][values] at the start
 *                     (Sort.swift:11-28)
 *   radix passes      SortSource.swift:31-91,334-386 and Sort.swift:404-494: 8-bit LSD digits, a pass
 *                     dropped when its digit is the same in every row (OR ^ AND over the keys)
 *   lexsort           Sources/ArrowMetal/Kernels/MultiSort.swift:28-65: per key from the last to the
 *                     first, keys = column.take(perm); idx = argsort(keys); perm = perm.take(idx)
 *   take              Sources/ArrowMetal/Kernels/Take.swift:41-79, KernelSource.swift:209-228: a null
 *                     index gives a null row, an index out of range is an error
 *
 * The passes run on `threads` host threads (per-thread digit counts, then a stable scatter of each
 * thread's chunk), which is how the CPU baseline uses the box's cores. Physical type codes match the
 * library's: 0 bool, 1 i8, 2 u8, 3 i16, 4 u16, 5 i32, 6 u32, 7 i64, 8 u64, 9 f16, 10 f32, 11 f64. */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

enum { PT_BOOL, PT_I8, PT_U8, PT_I16, PT_U16, PT_I32, PT_U32, PT_I64, PT_U64, PT_F16, PT_F32, PT_F64 };
enum { FO_IEEE = 0, FO_TOTAL = 1, FO_NANLARGEST = 2 };

static int bit_at(const uint8_t* p, int64_t i) { return (p[i >> 3] >> (i & 7)) & 1; }

static int key_bytes(int pt) { return (pt == PT_I64 || pt == PT_U64 || pt == PT_F64) ? 8 : 4; }

/* IEEE half to single, exactly (every half is a float). */
static uint32_t half_to_float_bits(uint16_t h) {
  uint32_t sign = (uint32_t)(h & 0x8000u) << 16, exp = (h >> 10) & 0x1Fu, man = h & 0x3FFu;
  if (exp == 0x1F) return sign | 0x7F800000u | (man << 13);           /* inf / NaN */
  if (exp == 0) {
    if (man == 0) return sign;                                          /* zero */
    int e = -1;
    do { man <<= 1; e++; } while (!(man & 0x400u));                     /* subnormal: normalise */
    return sign | ((uint32_t)(127 - 15 - e) << 23) | ((man & 0x3FFu) << 13);
  }
  return sign | ((exp + 112u) << 23) | (man << 13);
}

/* Key of one value. cat: 0 value, 1 NaN (its own block: ieee), 2 null. */
static uint64_t encode(const void* vals, int pt, int64_t row, int64_t bool_off, int desc, int fo, int* cat) {
  *cat = 0;
  if (pt == PT_I64 || pt == PT_U64 || pt == PT_F64) {
    uint64_t b = ((const uint64_t*)vals)[row], k;
    if (pt == PT_I64) k = b ^ 0x8000000000000000ull;
    else if (pt == PT_U64) k = b;
    else {
      const uint64_t S = 0x8000000000000000ull;
      if (fo == FO_TOTAL) {
        k = (b & S) ? ~b : (b | S);
      } else {
        int nan = (b & ~S) > 0x7FF0000000000000ull;
        if (nan && fo == FO_IEEE) { *cat = 1; return 0; }
        if ((b & ~S) == 0) b = 0;
        if (nan) b = 0x7FF0000000000001ull;
        k = (b & S) ? ~b : (b | S);
      }
    }
    return desc ? ~k : k;
  }
  int32_t v;
  uint32_t k;
  switch (pt) {
    case PT_BOOL: v = bit_at((const uint8_t*)vals, bool_off + row); break;
    case PT_I8: v = ((const int8_t*)vals)[row]; break;
    case PT_U8: v = ((const uint8_t*)vals)[row]; break;
    case PT_I16: v = ((const int16_t*)vals)[row]; break;
    case PT_U16: v = ((const uint16_t*)vals)[row]; break;
    case PT_I32: v = ((const int32_t*)vals)[row]; break;
    case PT_U32: k = ((const uint32_t*)vals)[row]; return desc ? (uint32_t)~k : k;
    default: {
      uint32_t b = pt == PT_F16 ? half_to_float_bits(((const uint16_t*)vals)[row]) : ((const uint32_t*)vals)[row];
      const uint32_t S = 0x80000000u;
      if (fo == FO_TOTAL) {
        k = (b & S) ? ~b : (b | S);
      } else {
        int nan = (b & ~S) > 0x7F800000u;
        if (nan && fo == FO_IEEE) { *cat = 1; return 0; }
        if ((b & ~S) == 0) b = 0;
        if (nan) b = 0x7F800001u;
        k = (b & S) ? ~b : (b | S);
      }
      return desc ? (uint32_t)~k : k;
    }
  }
  k = (uint32_t)v ^ 0x80000000u;
  return desc ? (uint32_t)~k : k;
}

/* ---- parallel LSD radix sort of (key, id) pairs -------------------------------------------- */

typedef struct {
  int t, T;
  int64_t m;
  const uint64_t* kin;
  const uint32_t* iin;
  uint64_t* kout;
  uint32_t* iout;
  int shift;
  int64_t* counts;   /* [T][256] */
} PassJob;

static void* pass_count(void* p) {
  PassJob* j = (PassJob*)p;
  int64_t lo = j->m * j->t / j->T, hi = j->m * (j->t + 1) / j->T;
  int64_t* c = j->counts + (int64_t)j->t * 256;
  memset(c, 0, 256 * sizeof(int64_t));
  for (int64_t i = lo; i < hi; i++) c[(j->kin[i] >> j->shift) & 255]++;
  return NULL;
}
static void* pass_scatter(void* p) {
  PassJob* j = (PassJob*)p;
  int64_t lo = j->m * j->t / j->T, hi = j->m * (j->t + 1) / j->T;
  int64_t* c = j->counts + (int64_t)j->t * 256;   /* now: this thread's start per digit */
  for (int64_t i = lo; i < hi; i++) {
    int d = (int)((j->kin[i] >> j->shift) & 255);
    int64_t at = c[d]++;
    j->kout[at] = j->kin[i];
    j->iout[at] = j->iin[i];
  }
  return NULL;
}

static void run_threads(void* (*fn)(void*), PassJob* jobs, int T) {
  pthread_t th[256];
  for (int t = 1; t < T; t++) pthread_create(&th[t], NULL, fn, &jobs[t]);
  fn(&jobs[0]);
  for (int t = 1; t < T; t++) pthread_join(th[t], NULL);
}

/* Stable LSD sort of m (key, id) pairs; passes whose digit is constant are dropped
 * (Sort.swift:404-417). The result ends in (k, ids). Returns the passes run. */
static int lsd_sort(uint64_t* k, uint32_t* ids, int64_t m, int kb, int threads) {
  if (m <= 1) return 0;
  uint64_t or_ = 0, and_ = ~0ull;
  for (int64_t i = 0; i < m; i++) { or_ |= k[i]; and_ &= k[i]; }
  uint64_t differing = or_ ^ and_;
  uint64_t* k2 = (uint64_t*)malloc((size_t)m * 8);
  uint32_t* i2 = (uint32_t*)malloc((size_t)m * 4);
  int T = threads < 1 ? 1 : (threads > 256 ? 256 : threads);
  if (m < 65536) T = 1;
  int64_t* counts = (int64_t*)malloc((size_t)T * 256 * sizeof(int64_t));
  PassJob jobs[256];
  uint64_t *ka = k, *kb2 = k2;
  uint32_t *ia = ids, *ib = i2;
  int passes = 0;
  for (int p = 0; p < kb; p++) {
    int shift = 8 * p;
    if (((differing >> shift) & 255) == 0) continue;
    for (int t = 0; t < T; t++) {
      jobs[t] = (PassJob){t, T, m, ka, ia, kb2, ib, shift, counts};
    }
    run_threads(pass_count, jobs, T);
    int64_t run = 0;
    for (int d = 0; d < 256; d++)
      for (int t = 0; t < T; t++) {
        int64_t c = counts[(int64_t)t * 256 + d];
        counts[(int64_t)t * 256 + d] = run;
        run += c;
      }
    run_threads(pass_scatter, jobs, T);
    uint64_t* tk = ka; ka = kb2; kb2 = tk;
    uint32_t* ti = ia; ia = ib; ib = ti;
    passes++;
  }
  if (ka != k) {
    memcpy(k, ka, (size_t)m * 8);
    memcpy(ids, ia, (size_t)m * 4);
  }
  free(k2);
  free(i2);
  free(counts);
  return passes;
}

/* Arrow array_sort_indices of one column (MetalArray.argsort, Sort.swift:56-65): out[n] uint32. */
int oracle_argsort(const void* vals, const uint8_t* valid, int64_t valid_off, int64_t bool_off, int64_t n, int pt,
                   int desc, int nulls_first, int fo, uint32_t* out, int threads) {
  if (n <= 0) return 0;
  if (pt != PT_F16 && pt != PT_F32 && pt != PT_F64) fo = FO_IEEE;
  const int kb = key_bytes(pt);
  uint64_t* keys = (uint64_t*)malloc((size_t)n * 8);
  uint32_t* ids = (uint32_t*)malloc((size_t)n * 4);
  uint32_t* nan_ids = (uint32_t*)malloc((size_t)n * 4);
  uint32_t* null_ids = (uint32_t*)malloc((size_t)n * 4);
  int64_t m = 0, nn = 0, nnan = 0;
  /* Stable three-way partition (SortSource.swift:226-330). */
  for (int64_t i = 0; i < n; i++) {
    if (valid && !bit_at(valid, valid_off + i)) { null_ids[nn++] = (uint32_t)i; continue; }
    int cat;
    uint64_t k = encode(vals, pt, i, bool_off, desc, fo, &cat);
    if (cat == 1) { nan_ids[nnan++] = (uint32_t)i; continue; }
    keys[m] = k;
    ids[m++] = (uint32_t)i;
  }
  lsd_sort(keys, ids, m, kb, threads);
  int64_t at = 0;
  if (nulls_first) {
    memcpy(out, null_ids, (size_t)nn * 4); at += nn;
    memcpy(out + at, nan_ids, (size_t)nnan * 4); at += nnan;
    memcpy(out + at, ids, (size_t)m * 4);
  } else {
    memcpy(out, ids, (size_t)m * 4); at += m;
    memcpy(out + at, nan_ids, (size_t)nnan * 4); at += nnan;
    memcpy(out + at, null_ids, (size_t)nn * 4);
  }
  free(keys); free(ids); free(nan_ids); free(null_ids);
  return 0;
}

/* Arrow take (Take.swift:41-79). idx_kind: 0 u32, 1 i32, 2 i64. width: bytes, 0 = boolean bits.
 * out_valid (may be NULL) receives one byte per row. Returns 1 for an index out of range. */
int oracle_take(const void* src, const uint8_t* src_valid, int64_t src_voff, int64_t src_bool_off, int64_t src_len,
                int width, const void* idx, int idx_kind, const uint8_t* idx_valid, int64_t idx_voff, int64_t n,
                void* out, uint8_t* out_valid) {
  int bad = 0;
  for (int64_t i = 0; i < n; i++) {
    int ok = !(idx_valid && !bit_at(idx_valid, idx_voff + i));
    int64_t r = 0;
    if (ok) {
      r = idx_kind == 0 ? (int64_t)((const uint32_t*)idx)[i]
                        : idx_kind == 1 ? (int64_t)((const int32_t*)idx)[i] : ((const int64_t*)idx)[i];
      if (r < 0 || r >= src_len) { bad = 1; ok = 0; }
    }
    int v = ok && !(src_valid && !bit_at(src_valid, src_voff + r));
    if (out_valid) out_valid[i] = (uint8_t)v;
    switch (width) {
      case 8: ((uint64_t*)out)[i] = ok ? ((const uint64_t*)src)[r] : 0; break;
      case 4: ((uint32_t*)out)[i] = ok ? ((const uint32_t*)src)[r] : 0; break;
      case 2: ((uint16_t*)out)[i] = ok ? ((const uint16_t*)src)[r] : 0; break;
      case 1: ((uint8_t*)out)[i] = ok ? ((const uint8_t*)src)[r] : 0; break;
      default: {
        uint8_t* o = (uint8_t*)out;
        int b = ok && bit_at((const uint8_t*)src, src_bool_off + r);
        if (b) o[i >> 3] |= (uint8_t)(1u << (i & 7));
        else o[i >> 3] &= (uint8_t)~(1u << (i & 7));
      }
    }
  }
  return bad;
}

/* Multi-key sort the reference's way (MultiSort.swift:56-64): least significant key first, each
 * key's column gathered through the permutation so far, argsorted, and the permutation composed. */
int oracle_lexsort(int K, const void* const* vals, const uint8_t* const* valid, const int64_t* valid_off,
                   const int64_t* bool_off, const int* pts, const int* desc, const int* nulls_first, const int* fo,
                   int64_t n, uint32_t* out, int threads) {
  if (n <= 0) return 0;
  uint32_t* perm = NULL;
  uint32_t* idx = (uint32_t*)malloc((size_t)n * 4);
  for (int k = K - 1; k >= 0; k--) {
    const int pt = pts[k];
    const int w = pt == PT_BOOL ? 0 : (pt == PT_I8 || pt == PT_U8) ? 1
                : (pt == PT_I16 || pt == PT_U16 || pt == PT_F16) ? 2 : (pt == PT_I64 || pt == PT_U64 || pt == PT_F64) ? 8 : 4;
    const void* kv = vals[k];
    const uint8_t* kvalid = valid[k];
    int64_t kvoff = valid_off[k], kboff = bool_off[k];
    void* gathered = NULL;
    uint8_t* gvalid_bits = NULL;
    if (perm) {
      size_t bytes = w ? (size_t)n * (size_t)w : (size_t)(n + 7) / 8;
      gathered = calloc(bytes + 8, 1);
      uint8_t* gbytes = (uint8_t*)malloc((size_t)n);
      oracle_take(kv, kvalid, kvoff, kboff, n, w, perm, 0, NULL, 0, n, gathered, gbytes);
      if (kvalid) {
        gvalid_bits = (uint8_t*)calloc((size_t)(n + 7) / 8 + 8, 1);
        for (int64_t i = 0; i < n; i++) if (gbytes[i]) gvalid_bits[i >> 3] |= (uint8_t)(1u << (i & 7));
      }
      free(gbytes);
      kv = gathered; kvalid = gvalid_bits; kvoff = 0; kboff = 0;
    }
    oracle_argsort(kv, kvalid, kvoff, kboff, n, pt, desc[k], nulls_first[k], fo[k], idx, threads);
    if (perm) {
      uint32_t* composed = (uint32_t*)malloc((size_t)n * 4);
      for (int64_t i = 0; i < n; i++) composed[i] = perm[idx[i]];
      free(perm);
      perm = composed;
    } else {
      perm = (uint32_t*)malloc((size_t)n * 4);
      memcpy(perm, idx, (size_t)n * 4);
    }
    free(gathered);
    free(gvalid_bits);
  }
  memcpy(out, perm, (size_t)n * 4);
  free(perm);
  free(idx);
  return 0;
}
