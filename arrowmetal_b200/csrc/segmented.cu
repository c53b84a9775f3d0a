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
      // Every output index array is a view into one block (each array's rows rounded up to 16 bytes):
      // one stream-ordered allocation for the batch, not one per array. The block is freed when the
      // last view is released.
      std::vector<size_t> offs(size_t(count) + 1, 0);
      for (int64_t i = 0; i < count; i++)
        offs[size_t(i) + 1] = offs[size_t(i)] + ((size_t(std::max<int64_t>(arrays[i]->length, 1)) * 4 + 15) & ~size_t(15));
      BufPtr block = count > 0 ? DevBuffer::alloc(offs[size_t(count)] + 16, s) : nullptr;
      for (int64_t i = 0; i < count; i++) {
        SortKey k{arrays[i], descending ? descending[i] != 0 : false, null_placement ? null_placement[i] == 1 : false,
                  float_order ? float_order[i] : 0};
        if (k.float_order < 0 || k.float_order > 2) throw invalid("unknown float_order " + std::to_string(k.float_order));
        const int64_t n = arrays[i]->length;
        check_index_rows(n, "argsort");
        use_on(arrays[i], s);
        am_array* o = new_array(PT_U32, "I", n);
        res.push_back(o);
        auto view = std::make_shared<DevBuffer>();
        view->ptr = static_cast<char*>(block->ptr) + offs[size_t(i)];
        view->bytes = offs[size_t(i) + 1] - offs[size_t(i)];
        view->stream = s;
        view->owned = false;
        // The block is freed on its own stream once every view is gone: each view's release first
        // orders that stream after the view's last stream.
        DevBuffer* vp = view.get();
        view->on_release = [block, vp] {
          if (vp->stream && vp->stream != block->stream) {
            cudaEvent_t e;
            if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) == cudaSuccess) {
              (void)cudaEventRecord(e, vp->stream);
              (void)cudaStreamWaitEvent(block->stream, e, 0);
              (void)cudaEventDestroy(e);
            }
          }
        };
        o->values = view;
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
