/* Apache Arrow C Data Interface, C Stream Interface and C Device Data Interface.
 *
 * The struct layouts are fixed by the Arrow specification
 * (https://arrow.apache.org/docs/format/CDataInterface.html, CStreamInterface.html and
 *  https://arrow.apache.org/docs/format/CDeviceDataInterface.html); every producer and consumer of
 * the interface, pyarrow and arrow-rs included, must agree on them byte for byte. The guard macros
 * are the specification's own, so this header coexists with any other copy of the definitions. */
#ifndef AM_ARROW_ABI_H
#define AM_ARROW_ABI_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#ifndef ARROW_C_DATA_INTERFACE
#define ARROW_C_DATA_INTERFACE

#define ARROW_FLAG_DICTIONARY_ORDERED 1
#define ARROW_FLAG_NULLABLE 2
#define ARROW_FLAG_MAP_KEYS_SORTED 4

struct ArrowSchema {
  const char* format;
  const char* name;
  const char* metadata;
  int64_t flags;
  int64_t n_children;
  struct ArrowSchema** children;
  struct ArrowSchema* dictionary;
  void (*release)(struct ArrowSchema*);
  void* private_data;
};

struct ArrowArray {
  int64_t length;
  int64_t null_count;
  int64_t offset;
  int64_t n_buffers;
  int64_t n_children;
  const void** buffers;
  struct ArrowArray** children;
  struct ArrowArray* dictionary;
  void (*release)(struct ArrowArray*);
  void* private_data;
};

#endif /* ARROW_C_DATA_INTERFACE */

#ifndef ARROW_C_STREAM_INTERFACE
#define ARROW_C_STREAM_INTERFACE

/* The Arrow C Stream Interface (https://arrow.apache.org/docs/format/CStreamInterface.html): a
 * producer of record batches, each a struct array whose children are the columns. */
struct ArrowArrayStream {
  int (*get_schema)(struct ArrowArrayStream*, struct ArrowSchema* out);
  int (*get_next)(struct ArrowArrayStream*, struct ArrowArray* out);
  const char* (*get_last_error)(struct ArrowArrayStream*);
  void (*release)(struct ArrowArrayStream*);
  void* private_data;
};

#endif /* ARROW_C_STREAM_INTERFACE */

#ifndef ARROW_C_DEVICE_DATA_INTERFACE
#define ARROW_C_DEVICE_DATA_INTERFACE

#define ARROW_DEVICE_CPU 1
#define ARROW_DEVICE_CUDA 2
#define ARROW_DEVICE_CUDA_HOST 3
#define ARROW_DEVICE_CUDA_MANAGED 13

typedef int32_t ArrowDeviceType;

struct ArrowDeviceArray {
  struct ArrowArray array;
  int64_t device_id;
  ArrowDeviceType device_type;
  void* sync_event;      /* for ARROW_DEVICE_CUDA: a cudaEvent_t* the consumer waits on, or NULL */
  int64_t reserved[3];
};

#endif /* ARROW_C_DEVICE_DATA_INTERFACE */

#ifdef __cplusplus
}
#endif

#endif /* AM_ARROW_ABI_H */
