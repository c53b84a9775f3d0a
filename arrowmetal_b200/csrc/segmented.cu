// Segmented (batched) argsort: many independent arrays sorted in one call.
#include "am_internal.h"
#include "radix_sort.cuh"

using namespace am;

// am_argsort_batch: every array's argsort, identical to am_argsort_ex2 on that array alone, with the
// arrays of each key width sorted together: one histogram launch, one plan launch and one launch per
// digit pass for all of them (radix_argsort_batch), instead of a sort's ~11 launches per array.
extern "C" int am_argsort_batch(am_array** arrays, const int* descending, const int* null_placement,
                                const int* float_order, int64_t count, am_array** outs) {
  if (!arrays || !outs || count < 0) return 2;
  for (int64_t i = 0; i < count; i++) if (!arrays[i]) return 2;
  try {
    cudaStream_t s = stream();
    std::vector<am_array*> res;
    std::vector<SortKey> keys;
    std::vector<void*> ptrs;
    try {
      for (int64_t i = 0; i < count; i++) {
        SortKey k{arrays[i], descending ? descending[i] != 0 : false, null_placement ? null_placement[i] == 1 : false,
                  float_order ? float_order[i] : 0};
        if (k.float_order < 0 || k.float_order > 2) throw invalid("unknown float_order " + std::to_string(k.float_order));
        const int64_t n = arrays[i]->length;
        check_index_rows(n, "argsort");
        use_on(arrays[i], s);
        am_array* o = new_array(PT_U32, "I", n);
        res.push_back(o);
        o->values = DevBuffer::alloc(size_t(std::max<int64_t>(n, 1)) * 4 + 16, s);
        o->null_count = 0;
        o->perm_of = n;
        o->last_stream = s;
        keys.push_back(k);
        ptrs.push_back(o->values->ptr);
      }
      radix_argsort_batch(keys, ptrs, s);
    } catch (...) {
      for (am_array* r : res) am::release(r);
      throw;
    }
    for (int64_t i = 0; i < count; i++) outs[i] = res[size_t(i)];
    return 0;
  } catch (const Error& e) {
    set_last_error(e.what());
    return e.code;
  } catch (const std::exception& e) {
    set_last_error(e.what());
    return 1;
  }
}
