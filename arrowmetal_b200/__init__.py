"""ArrowMetal's sort path on NVIDIA B200: Apache Arrow arrays in HBM, sorted by sm_100a kernels.

A ctypes binding over ``libArrowMetalC.so`` with the names, arguments and errors of ArrowMetal's own
Python binding for the sort path (python/arrowmetal/__init__.py: ``MetalArray.from_arrow`` / ``to_arrow``
:265-300, ``take`` :444-450, ``argsort`` / ``sort`` / ``top_k`` :460-480 and the option form :3940-3970,
``lexsort_indices`` :1325-1359, ``ArrowMetalError`` :210-211). Results come back as pyarrow
arrays, so they drop straight into pyarrow, Polars or pandas::

    import pyarrow as pa, arrowmetal_b200 as am
    col = am.MetalArray.from_arrow(pa.array([3, None, 1]))
    col.argsort().to_arrow()                 # -> [2, 0, 1] (uint32)

There is no CPU fallback: a missing library or a missing GPU raises.
"""
import contextlib
import ctypes
import json
import os

import pyarrow as pa

__version__ = "0.6.1"

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libArrowMetalC.so")

NULL_PLACEMENT = ("at_end", "at_start")
FLOAT_ORDERS = ("ieee", "total", "nan_largest")
TIEBREAKERS = ("min", "max", "first", "dense")       # Arrow's rank tiebreakers, in the C ABI's numbering
VALUE_ORDERS = ("first_appearance", "sorted")        # unique / value_counts
WINDOW_OPS = ("row_number", "rank", "dense_rank", "percent_rank", "cume_dist")   # am_window ops 0-4


def _find_library():
    """`$ARROWMETAL_LIB` (a full path, which must exist), else the in-tree build."""
    env = os.environ.get("ARROWMETAL_LIB")
    if env:
        if not os.path.exists(env):
            raise OSError("arrowmetal_b200: $ARROWMETAL_LIB is set to " + env + ", which does not exist")
        return env
    if not os.path.exists(LIB_PATH):
        raise OSError("arrowmetal_b200: " + LIB_PATH + " is missing; build it with "
                      "`make -C arrowmetal_b200/csrc` (or __graft_entry__.build())")
    return LIB_PATH


_lib = ctypes.CDLL(_find_library())
_P = ctypes.c_void_p
_PP = ctypes.POINTER(_P)
_I = ctypes.c_int
_I64 = ctypes.c_int64
_IP = ctypes.POINTER(ctypes.c_int)


class _ArrowSchema(ctypes.Structure):
    _fields_ = [("format", ctypes.c_char_p), ("name", ctypes.c_char_p), ("metadata", ctypes.c_char_p),
                ("flags", _I64), ("n_children", _I64), ("children", _P), ("dictionary", _P),
                ("release", _P), ("private_data", _P)]


class _ArrowArray(ctypes.Structure):
    _fields_ = [("length", _I64), ("null_count", _I64), ("offset", _I64), ("n_buffers", _I64),
                ("n_children", _I64), ("buffers", _P), ("children", _P), ("dictionary", _P),
                ("release", _P), ("private_data", _P)]


class _ArrowDeviceArray(ctypes.Structure):
    _fields_ = [("array", _ArrowArray), ("device_id", _I64), ("device_type", ctypes.c_int32),
                ("sync_event", _P), ("reserved", _I64 * 3)]


class ServerStats(ctypes.Structure):
    _fields_ = [(n, _I64) for n in ("requests", "solo_requests", "batches", "batched_requests", "rows",
                                    "peak_in_flight_bytes", "in_flight_bytes", "queued", "shared_sorts",
                                    "shared_requests")]


class BatchShape(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int32) for n in ("key_bytes", "size_class", "max_rows", "method", "threads", "items",
                                              "digit_bits")]


class SortStats(ctypes.Structure):
    _fields_ = [("rows", _I64), ("value_rows", _I64), ("passes_run", ctypes.c_int32),
                ("passes_skipped", ctypes.c_int32), ("kernel_us", ctypes.c_double),
                ("payload_in_records", ctypes.c_int32), ("reserved", ctypes.c_int32)]


def _sig(name, res, args):
    f = getattr(_lib, name)
    f.restype = res
    f.argtypes = args


for _name, _res, _args in [
    ("am_version", ctypes.c_char_p, []), ("am_device_name", ctypes.c_char_p, []),
    ("am_last_error", ctypes.c_char_p, []),
    ("am_import", _I, [_P, _P, _PP]), ("am_import_device", _I, [_P, _P, _PP]),
    ("am_import_chunks", _I, [_P, _P, _I64, _PP]), ("am_import_chunks_supported", _I, [_P]),
    ("am_set_import_threads", _I, [_I]), ("am_get_import_threads", _I, []),
    ("am_export", _I, [_P, _P, _P]), ("am_export_device", _I, [_P, _P, _P]),
    ("am_release", None, [_P]), ("am_length", _I64, [_P]), ("am_null_count", _I64, [_P]),
    ("am_format", ctypes.c_char_p, [_P]), ("am_compute_format", ctypes.c_char_p, [_P]),
    ("am_take", _I, [_P, _P, _PP]), ("am_slice", _I, [_P, _I64, _I64, _PP]),
    ("am_take_columns", _I, [_PP, _I64, _P, _PP]),
    ("am_argsort", _I, [_P, _I, _PP]), ("am_sort", _I, [_P, _I, _PP]), ("am_top_k", _I, [_P, _I64, _I, _PP]),
    ("am_argsort_ex", _I, [_P, _I, _I, _PP]), ("am_sort_ex", _I, [_P, _I, _I, _PP]),
    ("am_argsort_ex2", _I, [_P, _I, _I, _I, _PP]), ("am_sort_ex2", _I, [_P, _I, _I, _I, _PP]),
    ("am_argsort_ex3", _I, [_P, _I, _I, _I, _I, _PP]),
    ("am_top_k_ex", _I, [_P, _I64, _I, _I, _I, _PP]),
    ("am_lexsort", _I, [_PP, _IP, _I64, _PP]), ("am_lexsort_ex", _I, [_PP, _IP, _I64, _I, _PP]),
    ("am_lexsort_ex2", _I, [_PP, _IP, _IP, _IP, _I64, _PP]),
    ("am_argsort_batch", _I, [_PP, _IP, _IP, _IP, _I64, _PP]),
    ("am_batch_begin", _I, []), ("am_batch_end", _I, []),
    ("am_plan_source_create", _I, [ctypes.c_char_p, _PP, ctypes.POINTER(ctypes.c_char_p), _I64, _PP]),
    ("am_plan_source_release", None, [_P]),
    ("am_plan_run", _I, [ctypes.c_char_p, _PP, _I64, _I, _PP]),
    ("am_plan_explain", ctypes.c_char_p, [ctypes.c_char_p, _PP, _I64, _I]),
    ("am_plan_column_count", _I64, [_P]), ("am_plan_row_count", _I64, [_P]),
    ("am_plan_column_name", ctypes.c_char_p, [_P, _I64]), ("am_plan_column", _I, [_P, _I64, _PP]),
    ("am_plan_result_release", None, [_P]),
    ("am_router_set_mode", _I, [_I]), ("am_router_get_mode", _I, []),
    ("am_cuda_set_stream", _I, [_P]), ("am_cuda_get_stream", _P, []), ("am_cuda_synchronize", _I, []),
    ("am_cuda_device", _I, []), ("am_last_sort_stats", _I, [ctypes.POINTER(SortStats)]),
    ("am_cuda_batch_tuning", _I, [ctypes.POINTER(BatchShape), _I64, ctypes.POINTER(_I64)]),
    ("am_cuda_profile", _I, [_I]), ("am_cuda_profile_count", _I64, []),
    ("am_cuda_profile_entry", _I, [_I64, ctypes.POINTER(ctypes.c_char_p), ctypes.POINTER(_I64),
                                   ctypes.POINTER(ctypes.c_double)]),
    ("am_cuda_profile_reset", _I, []),
    ("am_debug_set_max_row_index", _I, [_I64]), ("am_debug_fail_alloc_after", _I, [_I64]),
    ("am_debug_skip_first_tile", _I, [_I]), ("am_debug_force_batch_shape", _I, [_I]),
    ("am_server_create", _I, [_I, _I64, _I64, _PP]),
    ("am_server_submit", _I, [_P, _P, _I64, _I64, ctypes.POINTER(ctypes.c_char_p), _IP, _IP, _IP, _I64,
                              ctypes.POINTER(ctypes.c_char_p), _I64, ctypes.POINTER(_I64)]),
    ("am_server_wait", _I, [_P, _I64, _PP, ctypes.POINTER(ctypes.c_double)]),
    ("am_server_get_stats", _I, [_P, ctypes.POINTER(ServerStats)]),
    ("am_server_release", _I, [_P]),
    ("am_partition_nth_indices", _I, [_P, _I64, _PP]), ("am_partition_nth_ex", _I, [_P, _I64, _I, _PP]),
    ("am_rank_ex", _I, [_P, _I, _I, _I, _PP]), ("am_rank_quantile_ex", _I, [_P, _I, _I, _I, _PP]),
    ("am_rank", _I, [_P, _I, _PP]), ("am_window", _I, [_P, _I, _I64, _I64, _P, _PP]),
    ("am_stream_last_error", ctypes.c_char_p, []), ("am_stream_from_c_stream", _P, [_P, _I]),
    ("am_stream_open_ipc", _P, [ctypes.c_char_p, _I, _I]), ("am_stream_release", None, [_P]),
    ("am_stream_select", _I, [_P, ctypes.POINTER(ctypes.c_char_p), _I64]), ("am_stream_export_c", _I, [_P, _P]),
    ("am_stream_sort_ex", _I, [_P, ctypes.POINTER(ctypes.c_char_p), _IP, _IP, _IP, _I64, _I64, ctypes.c_char_p,
                               ctypes.c_char_p, _PP]),
    ("am_stream_sort", _I, [_P, ctypes.POINTER(ctypes.c_char_p), _IP, _I64, _I64, ctypes.c_char_p, ctypes.c_char_p,
                            _PP]),
    ("am_stream_result_column_count", _I64, [_P]), ("am_stream_result_column_name", ctypes.c_char_p, [_P, _I64]),
    ("am_stream_result_column", _I, [_P, _I64, _PP]), ("am_stream_result_rows_out", _I64, [_P]),
    ("am_stream_result_stats", _I, [_P] + [ctypes.POINTER(_I64)] * 3 + [ctypes.POINTER(ctypes.c_double)] * 5),
    ("am_stream_result_stalls", _I, [_P, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]),
    ("am_stream_result_release", None, [_P]),
    ("am_unique", _I, [_P, _PP]), ("am_unique_ex", _I, [_P, _I, _PP]),
    ("am_value_counts", _I, [_P, _PP]), ("am_value_counts_ex", _I, [_P, _I, _PP]),
]:
    _sig(_name, _res, _args)


def version():
    return _lib.am_version().decode()


def device_name():
    return _lib.am_device_name().decode()


class ArrowMetalError(RuntimeError):
    """A library call returned a non-zero status. `status` keeps the C ABI's code: 1 operation error,
    2 invalid argument, 3 a type the chunked import does not take."""

    def __init__(self, message, status=1):
        super().__init__(message)
        self.status = status


def _failure(status, entry=None):
    text = _lib.am_last_error()
    if text:
        return ArrowMetalError(text.decode(), status)
    return ArrowMetalError(f"{getattr(entry, '__name__', 'call')} returned status {status}", status)


def _ok(status):
    """Raises for the status of an entry point that has no output handle."""
    if status:
        raise _failure(status)


def _produce(entry, *args):
    """Calls an entry point whose last parameter receives a new array handle, and wraps that handle."""
    slot = _P()
    status = entry(*args, ctypes.byref(slot))
    if status:
        raise _failure(status, entry)
    return MetalArray(slot)


def _index_of(names, value, what):
    try:
        return names.index(value)
    except ValueError:
        raise ArrowMetalError(f"unknown {what} {value!r}; expected one of {', '.join(names)}", 2) from None


# Index types the gather reads as they are (None), and the type narrower ones widen to; any other type
# (uint64, floats, a plain Python sequence) becomes int64.
_GATHER_INDEX = {pa.int32(): None, pa.int64(): None, pa.uint32(): None, pa.int8(): pa.int32(),
                 pa.int16(): pa.int32(), pa.uint8(): pa.uint32(), pa.uint16(): pa.uint32()}


def _gather_indices(indices):
    """A MetalArray of `take` indices from a MetalArray, a pyarrow (chunked) array, a numpy array or a
    sequence of row numbers."""
    if isinstance(indices, MetalArray):
        return indices
    if isinstance(indices, pa.ChunkedArray):
        indices = indices.combine_chunks()
    elif not isinstance(indices, pa.Array):
        indices = pa.array(indices) if hasattr(indices, "dtype") else pa.array(list(indices), pa.int64())
    target = _GATHER_INDEX.get(indices.type, pa.int64())
    return MetalArray.from_arrow(indices if target is None else indices.cast(target))


def _sort_options(count, descending, null_placement, float_order):
    """The three per-key option vectors of the C ABI (direction, null placement, float order) as
    c_int arrays. `descending` is None (all ascending), one bool, or one flag per key; the other two are
    one name for every key or one name per key."""
    def per_key(value, what):
        if isinstance(value, (str, bool)) or value is None:
            return [value] * count
        items = list(value)
        if len(items) != count:
            raise ArrowMetalError(f"{what} has {len(items)} entries for {count} columns", 2)
        return items

    vec = ctypes.c_int * count
    flags = per_key(False if descending is None else descending, "descending")
    places = per_key(null_placement, "null_placement")
    orders = per_key(float_order, "float_order")
    return (vec(*[1 if d else 0 for d in flags]),
            vec(*[_index_of(NULL_PLACEMENT, p, "null_placement") for p in places]),
            vec(*[_index_of(FLOAT_ORDERS, f, "float_order") for f in orders]))


class MetalArray:
    """One Arrow array in this GPU's memory, owned through a library handle. Calls never modify it:
    each returns a new MetalArray (or a pyarrow result)."""

    def __init__(self, handle):
        self._h = handle

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and _lib is not None:          # module globals are cleared at interpreter exit
            _lib.am_release(h)
            self._h = None

    # ---- interop
    @classmethod
    def from_arrow(cls, obj):
        """Import anything pyarrow can turn into an array (a ChunkedArray of several chunks goes
        through the chunked import). The buffers are copied into HBM."""
        if isinstance(obj, pa.ChunkedArray):
            if obj.num_chunks > 1:
                return _import_chunks(obj)
            obj = obj.chunk(0) if obj.num_chunks == 1 else pa.array([], type=obj.type)
        if not isinstance(obj, pa.Array):
            obj = pa.array(obj)
        schema, array = _ArrowSchema(), _ArrowArray()
        obj._export_to_c(ctypes.addressof(array), ctypes.addressof(schema))
        try:
            return _produce(_lib.am_import, ctypes.addressof(schema), ctypes.addressof(array))
        finally:
            if array.release:
                ctypes.CFUNCTYPE(None, _P)(array.release)(ctypes.addressof(array))
            if schema.release:
                ctypes.CFUNCTYPE(None, _P)(schema.release)(ctypes.addressof(schema))

    @classmethod
    def from_device(cls, data_ptr, length, fmt, validity_ptr=0, null_count=0, offset=0, keep=None):
        """Wrap arrays already in this GPU's memory (ARROW_DEVICE_CUDA) without a copy. `keep` is held
        until the array is released."""
        arr = _ArrowDeviceArray()
        bufs = (_P * 2)(validity_ptr or None, data_ptr)
        holder = _DeviceHolder(bufs, keep, fmt)
        arr.array.length = length
        arr.array.null_count = null_count
        arr.array.offset = offset
        arr.array.n_buffers = 2
        arr.array.buffers = ctypes.cast(bufs, _P)
        arr.array.release = ctypes.cast(holder.release_cb, _P)
        arr.device_type = 2
        arr.device_id = _lib.am_cuda_device()
        schema = _ArrowSchema()
        schema.format = fmt.encode()
        out = _produce(_lib.am_import_device, ctypes.addressof(schema), ctypes.addressof(arr))
        out._device_holder = holder
        return out

    def to_arrow(self):
        """Export as a pyarrow.Array (copied into pinned host memory owned by the array)."""
        schema, array = _ArrowSchema(), _ArrowArray()
        _ok(_lib.am_export(self._h, ctypes.addressof(schema), ctypes.addressof(array)))
        return pa.Array._import_from_c(ctypes.addressof(array), ctypes.addressof(schema))

    def __len__(self):
        return int(_lib.am_length(self._h))

    @property
    def null_count(self):
        return int(_lib.am_null_count(self._h))

    @property
    def format(self):
        return _lib.am_format(self._h).decode()

    # ---- selection
    def take(self, indices):
        """Arrow `take`: int32, int64 and uint32 indices; a null index gives a null row."""
        indices = _gather_indices(indices)       # held until the call returns
        return _produce(_lib.am_take, self._h, indices._h)

    def slice(self, offset, length):
        return _produce(_lib.am_slice, self._h, offset, length)

    # ---- sorting (stable radix sort on the GPU)
    def argsort(self, descending=False, null_placement="at_end", float_order="ieee"):
        """UInt32 indices that sort the array (Arrow `array_sort_indices`; pyarrow returns uint64 with
        the same values). `null_placement` is independent of the direction, as in Arrow.
        `float_order`: "ieee" (pyarrow's order: -0.0 ties +0.0, NaN next to the nulls), "total"
        (IEEE 754 totalOrder, arrow-rs), "nan_largest" (Polars)."""
        return _produce(_lib.am_argsort_ex2, self._h, 1 if descending else 0,
                        _index_of(NULL_PLACEMENT, null_placement, "null_placement"),
                        _index_of(FLOAT_ORDERS, float_order, "float_order"))

    def argsort64(self, descending=False, null_placement="at_end", float_order="ieee"):
        """`argsort` with uint64 indices, the type pyarrow's sort_indices returns."""
        return _produce(_lib.am_argsort_ex3, self._h, 1 if descending else 0,
                        _index_of(NULL_PLACEMENT, null_placement, "null_placement"),
                        _index_of(FLOAT_ORDERS, float_order, "float_order"), 8)

    def sort(self, descending=False, null_placement="at_end", float_order="ieee"):
        """Sorted copy of the array, with the ordering rules of `argsort`."""
        return _produce(_lib.am_sort_ex2, self._h, 1 if descending else 0,
                        _index_of(NULL_PLACEMENT, null_placement, "null_placement"),
                        _index_of(FLOAT_ORDERS, float_order, "float_order"))

    def top_k(self, k, largest=True, null_placement="at_end", float_order="ieee"):
        """UInt32 indices of the k largest (or smallest) values: the first k of `argsort`."""
        return _produce(_lib.am_top_k_ex, self._h, int(k), 1 if largest else 0,
                        _index_of(NULL_PLACEMENT, null_placement, "null_placement"),
                        _index_of(FLOAT_ORDERS, float_order, "float_order"))


    # ---- sort consumers (one argsort, then run marks, a scan and scatters)
    def partition_nth_indices(self, pivot, null_placement="at_end"):
        """Arrow `partition_nth_indices`: uint32 indices with, at position `pivot`, the row a stable
        ascending sort puts there; no row before it orders after it and none after it before it. Each
        of the three blocks (before, equal, after) keeps row order. A radix select, not a sort."""
        return _produce(_lib.am_partition_nth_ex, self._h, int(pivot),
                        _index_of(NULL_PLACEMENT, null_placement, "null_placement"))

    def rank(self, sort_keys="ascending", null_placement="at_end", tiebreaker="min"):
        """Arrow `rank` (uint32; pyarrow returns uint64 with the same values). Nulls and NaN rows are one
        tie group at the `null_placement` end, as in pyarrow."""
        return _produce(_lib.am_rank_ex, self._h, _index_of(TIEBREAKERS, tiebreaker, "tiebreaker"),
                        _direction(sort_keys), _index_of(NULL_PLACEMENT, null_placement, "null_placement"))

    def rank_quantile(self, sort_keys="ascending", null_placement="at_end"):
        """Arrow `rank_quantile`: (average 1-based rank of the row's tie group - 0.5) / n, float64."""
        return _produce(_lib.am_rank_quantile_ex, self._h, 0, _direction(sort_keys),
                        _index_of(NULL_PLACEMENT, null_placement, "null_placement"))

    def rank_normal(self, sort_keys="ascending", null_placement="at_end", float32=False):
        """Arrow `rank_normal`: the standard normal quantile of `rank_quantile()` (float64, or float32)."""
        return _produce(_lib.am_rank_quantile_ex, self._h, 2 if float32 else 1, _direction(sort_keys),
                        _index_of(NULL_PLACEMENT, null_placement, "null_placement"))

    def window(self, op):
        """One of the SQL ranking window functions by name (ascending, nulls last and tied)."""
        return _produce(_lib.am_window, self._h, _index_of(WINDOW_OPS, op, "op"), 0, 0, None)

    def row_number(self):
        return self.window("row_number")

    def dense_rank(self):
        return self.window("dense_rank")

    def percent_rank(self):
        return self.window("percent_rank")

    def cume_dist(self):
        return self.window("cume_dist")

    def unique(self, order="first_appearance"):
        """Arrow `unique`. "first_appearance" keeps Arrow's order and its one null entry (not for string
        columns); "sorted" is ascending with the nulls dropped. -0.0 matches 0.0 and every NaN is one
        value; the representative is the earliest row."""
        return _produce(_lib.am_unique_ex, self._h, _index_of(VALUE_ORDERS, order, "order"))

    def value_counts(self, order="first_appearance"):
        """Arrow `value_counts`: a struct array of `values` and their int64 `counts`, in `unique`'s order."""
        return _produce(_lib.am_value_counts_ex, self._h, _index_of(VALUE_ORDERS, order, "order"))


def _direction(sort_keys):
    if sort_keys not in ("ascending", "descending"):
        raise ArrowMetalError('sort_keys must be "ascending" or "descending"')
    return 1 if sort_keys == "descending" else 0


class _DeviceHolder:
    """Keeps a device import's Python owner alive until the library releases the array."""
    _live = set()

    def __init__(self, bufs, keep, fmt):
        self.bufs, self.keep, self.fmt = bufs, keep, fmt
        _DeviceHolder._live.add(self)

        def _release(p):
            ctypes.cast(p, ctypes.POINTER(_ArrowArray)).contents.release = None
            _DeviceHolder._live.discard(self)
        self.release_cb = ctypes.CFUNCTYPE(None, _P)(_release)


def _import_chunks(chunked):
    chunks = chunked.chunks
    n = len(chunks)
    arrays = (_ArrowArray * n)()
    schema = _ArrowSchema()
    chunks[0]._export_to_c(ctypes.addressof(arrays[0]), ctypes.addressof(schema))
    for i in range(1, n):
        chunks[i]._export_to_c(ctypes.addressof(arrays[i]))
    out = _P()
    try:
        rc = _lib.am_import_chunks(ctypes.addressof(schema), ctypes.addressof(arrays), n, ctypes.byref(out))
        if rc == 3:
            for a in arrays:
                if a.release:
                    ctypes.CFUNCTYPE(None, _P)(a.release)(ctypes.addressof(a))
            return MetalArray.from_arrow(chunked.combine_chunks())
        _ok(rc)
        return MetalArray(out)
    finally:
        for a in arrays:
            if a.release:
                ctypes.CFUNCTYPE(None, _P)(a.release)(ctypes.addressof(a))
        if schema.release:
            ctypes.CFUNCTYPE(None, _P)(schema.release)(ctypes.addressof(schema))


def lexsort_indices(columns, descending=None, null_placement="at_end", float_order="ieee"):
    """Multi-column sort: uint32 indices ordering the rows by each column in turn, the first column the
    most significant. `descending` is one flag per column (None: all ascending); `null_placement` and
    `float_order` are one value or one per key."""
    cols = [c if isinstance(c, MetalArray) else MetalArray.from_arrow(c) for c in columns]
    if not cols:
        raise ArrowMetalError("lexsort needs at least one column", 2)
    desc, places, orders = _sort_options(len(cols), descending, null_placement, float_order)
    handles = (_P * len(cols))(*[c._h for c in cols])
    return _produce(_lib.am_lexsort_ex2, handles, desc, places, orders, len(cols))


def take_columns(columns, indices):
    """`take` of several columns through one index array, with one index read on the GPU."""
    cols = [c if isinstance(c, MetalArray) else MetalArray.from_arrow(c) for c in columns]
    indices = _gather_indices(indices)
    n = len(cols)
    handles = (_P * n)(*[c._h for c in cols])
    outs = (_P * n)()
    _ok(_lib.am_take_columns(handles, n, indices._h, outs))
    return [MetalArray(outs[i]) for i in range(n)]


def argsort_batch(arrays, descending=None, null_placement=None, float_order=None):
    """Segmented sort: uint32 indices of each array, all sorted in one call."""
    cols = [c if isinstance(c, MetalArray) else MetalArray.from_arrow(c) for c in arrays]
    n = len(cols)
    handles = (_P * n)(*[c._h for c in cols])
    d, p, f = _sort_options(n, descending, null_placement or "at_end", float_order or "ieee")
    outs = (_P * max(n, 1))()
    _ok(_lib.am_argsort_batch(handles, d, p, f, n, outs))
    return [MetalArray(outs[i]) for i in range(n)]


# ---- batching, router, plan ----------------------------------------------------------------------

@contextlib.contextmanager
def batch():
    """Calls inside the block do not wait for the GPU; deferred errors raise at its end."""
    _ok(_lib.am_batch_begin())
    try:
        yield
    finally:
        _ok(_lib.am_batch_end())


_ROUTER = ("auto", "gpu", "cpu")


def set_router(mode):
    """Router mode ("auto", "gpu", "cpu"). The sort is never routed to the CPU."""
    _ok(_lib.am_router_set_mode(_index_of(_ROUTER, mode, "router mode")))


def get_router():
    return _ROUTER[_lib.am_router_get_mode()]


class PlanSource:
    """A named table the plan engine scans (am_plan_source_create)."""

    def __init__(self, name, columns):
        cols = {k: (v if isinstance(v, MetalArray) else MetalArray.from_arrow(v)) for k, v in columns.items()}
        n = len(cols)
        handles = (_P * n)(*[c._h for c in cols.values()])
        names = (ctypes.c_char_p * n)(*[k.encode() for k in cols])
        self._h = _P()
        _ok(_lib.am_plan_source_create(name.encode(), handles, names, n, ctypes.byref(self._h)))
        self.name = name
        self._cols = cols

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and _lib is not None:
            _lib.am_plan_source_release(h)
            self._h = None


def run_plan(plan, sources):
    """Runs a plan (a dict or its JSON) over PlanSource tables; returns {name: MetalArray}."""
    text = plan if isinstance(plan, str) else json.dumps(plan)
    n = len(sources)
    hs = (_P * max(n, 1))(*[s._h for s in sources])
    r = _P()
    _ok(_lib.am_plan_run(text.encode(), hs, n, 1, ctypes.byref(r)))
    return _plan_result_columns(r)


def _plan_result_columns(r):
    try:
        out = {}
        for i in range(_lib.am_plan_column_count(r)):
            h = _P()
            _ok(_lib.am_plan_column(r, i, ctypes.byref(h)))
            out[_lib.am_plan_column_name(r, i).decode()] = MetalArray(h)
        return out
    finally:
        _lib.am_plan_result_release(r)


class Server:
    """Sort server over tables resident in HBM (am_server_*): requests are admitted by their HBM
    footprint under `hbm_cap_bytes`, run by `workers` threads with a CUDA stream each, and single-key
    requests of at most `batch_rows` rows waiting together are sorted as one segmented batch.

    submit(source, offset, length, keys, payload) sorts rows [offset, offset + length) of a PlanSource
    by `keys` and takes `payload`; wait(ticket) returns ({name: MetalArray}, latency in ms)."""

    def __init__(self, workers=4, hbm_cap_bytes=120 * 10**9, batch_rows=1 << 20):
        self._h = _P()
        _ok(_lib.am_server_create(int(workers), int(hbm_cap_bytes), int(batch_rows), ctypes.byref(self._h)))
        self._sources = {}

    def submit(self, source, offset, length, keys, payload=(), descending=None, null_placement="at_end",
               float_order="ieee"):
        keys = [keys] if isinstance(keys, str) else list(keys)
        n = len(keys)
        kn = (ctypes.c_char_p * n)(*[k.encode() for k in keys])
        d, p, f = _sort_options(n, descending, null_placement, float_order)
        payload = list(payload)
        pn = (ctypes.c_char_p * max(len(payload), 1))(*[c.encode() for c in payload])
        t = _I64()
        self._sources[id(source)] = source          # the table outlives its requests
        _ok(_lib.am_server_submit(self._h, source._h, int(offset), int(length), kn, d, p, f, n, pn,
                                     len(payload), ctypes.byref(t)))
        return t.value

    def wait(self, ticket):
        r = _P()
        lat = ctypes.c_double()
        _ok(_lib.am_server_wait(self._h, int(ticket), ctypes.byref(r), ctypes.byref(lat)))
        return _plan_result_columns(r), lat.value

    def stats(self):
        s = ServerStats()
        _ok(_lib.am_server_get_stats(self._h, ctypes.byref(s)))
        return {name: getattr(s, name) for name, _ in ServerStats._fields_}

    def close(self):
        h = getattr(self, "_h", None)
        if h and _lib is not None:
            _lib.am_server_release(h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        self.close()


class _ArrowArrayStream(ctypes.Structure):
    _fields_ = [("get_schema", _P), ("get_next", _P), ("get_last_error", _P), ("release", _P), ("private_data", _P)]


def _stream_error(rc=None):
    raise ArrowMetalError((_lib.am_stream_last_error() or b"unknown error").decode())


def _as_reader(source):
    if isinstance(source, pa.RecordBatchReader):
        return source
    if isinstance(source, pa.Table):
        return source.to_reader()
    if isinstance(source, pa.RecordBatch):
        return pa.Table.from_batches([source]).to_reader()
    if hasattr(source, "to_reader"):
        return source.to_reader()
    if hasattr(source, "scanner"):                  # a pyarrow dataset
        return source.scanner().to_reader()
    if hasattr(source, "__arrow_c_stream__"):
        return pa.RecordBatchReader.from_stream(source)
    raise ArrowMetalError(f"cannot stream record batches from {type(source).__name__}")


def _sort_keys(by):
    """Column names and descending flags from a name, a (name, descending) pair or a list of either."""
    if isinstance(by, (str, tuple)):
        by = [by]
    names, desc = [], []
    for k in by:
        if isinstance(k, str):
            names.append(k)
            desc.append(False)
        else:
            name, d = k
            names.append(name)
            desc.append(d in (True, "descending") if not isinstance(d, bool) else d)
    return names, desc


class Stream:
    """A source of Arrow record batches larger than HBM, consumed by one terminal call (`sort`,
    `sort_to_ipc`). Anything that speaks the Arrow C Stream Interface: a pyarrow RecordBatchReader,
    Table, dataset or scanner. `prefetch` batches are read ahead on a library thread."""

    def __init__(self, source, prefetch=3, _handle=None):
        if _handle is None:
            reader = _as_reader(source)
            c = _ArrowArrayStream()
            reader._export_to_c(ctypes.addressof(c))
            _handle = _lib.am_stream_from_c_stream(ctypes.addressof(c), int(prefetch))
            if not _handle:
                if c.release:
                    ctypes.CFUNCTYPE(None, _P)(c.release)(ctypes.addressof(c))
                _stream_error()
        self._h = _handle
        self._consumed = False
        self.stats = None
        self.rows_out = None

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and _lib is not None:
            _lib.am_stream_release(h)
            self._h = None

    def select(self, names):
        """Keep these columns, in this order, in the output."""
        arr = (ctypes.c_char_p * len(names))(*[n.encode() for n in names])
        if _lib.am_stream_select(self._h, arr, len(names)) != 0:
            _stream_error()
        return self

    def _sort(self, by, limit, scratch, path, null_placement, float_order):
        if self._consumed:
            raise ArrowMetalError("this stream has already been consumed; open a new one")
        self._consumed = True
        names, desc = _sort_keys(by)
        k = len(names)
        cn = (ctypes.c_char_p * k)(*[n.encode() for n in names])
        cd, cp, cf = _sort_options(k, desc, null_placement, float_order)
        out = _P()
        rc = _lib.am_stream_sort_ex(self._h, cn, cd, cp, cf, k, int(limit),
                                    None if scratch is None else str(scratch).encode(),
                                    None if path is None else str(path).encode(), ctypes.byref(out))
        if rc != 0:
            _stream_error()
        try:
            I64, D = ctypes.c_int64, ctypes.c_double
            b, r, by_, wall, read, gpu, merge, overlap = I64(), I64(), I64(), D(), D(), D(), D(), D()
            _lib.am_stream_result_stats(out, *[ctypes.byref(x) for x in (b, r, by_, wall, read, gpu, merge, overlap)])
            rs, ms = D(), D()
            _lib.am_stream_result_stalls(out, ctypes.byref(rs), ctypes.byref(ms))
            self.rows_out = _lib.am_stream_result_rows_out(out)
            self.stats = {"batches": b.value, "rows": r.value, "bytes_read": by_.value, "wall_s": wall.value,
                          "read_s": read.value, "gpu_s": gpu.value, "merge_s": merge.value,
                          "overlap": overlap.value, "read_stall_s": rs.value, "merge_stall_s": ms.value,
                          "rows_out": self.rows_out}
            n = _lib.am_stream_result_column_count(out)
            cols, col_names = [], []
            for i in range(n):
                col_names.append(_lib.am_stream_result_column_name(out, i).decode())
                h = _P()
                _ok(_lib.am_stream_result_column(out, i, ctypes.byref(h)))
                cols.append(MetalArray(h).to_arrow())
            return pa.table(cols, names=col_names) if n > 0 else None
        finally:
            _lib.am_stream_result_release(out)

    def sort(self, by, limit=0, scratch=None, null_placement="at_end", float_order="ieee"):
        """External sort, collected into a pyarrow.Table: sorted runs in HBM (spilled under `scratch`
        when the stream does not fit one), merged on the GPU. `by` is a column name, a (name,
        descending) pair or a list of either; `limit` 0 keeps every row. Ties keep stream order."""
        return self._sort(by, limit, scratch, None, null_placement, float_order)

    def to_reader(self):
        """The stream's batches (the selected columns) as a pyarrow.RecordBatchReader; consumes the stream."""
        if self._consumed:
            raise ArrowMetalError("this stream has already been consumed; open a new one")
        self._consumed = True
        c = _ArrowArrayStream()
        if _lib.am_stream_export_c(self._h, ctypes.addressof(c)) != 0:
            _stream_error()
        return pa.RecordBatchReader._import_from_c(ctypes.addressof(c))

    def sort_to_ipc(self, by, path, scratch=None, null_placement="at_end", float_order="ieee"):
        """External sort written to `path` as an Arrow IPC stream; returns the run's statistics."""
        self._sort(by, 0, scratch, path, null_placement, float_order)
        return self.stats


def scan_arrow(source, prefetch=3):
    """A `Stream` over anything that speaks the Arrow C Stream Interface."""
    return Stream(source, prefetch)


def scan_ipc(path, prefetch=3, readers=1):
    """A `Stream` over an Arrow IPC file (file or stream format) or a directory of them, memory-mapped."""
    h = _lib.am_stream_open_ipc(str(path).encode(), int(prefetch), int(readers))
    if not h:
        _stream_error()
    return Stream(None, _handle=h)


def explain_plan(plan, sources):
    text = plan if isinstance(plan, str) else json.dumps(plan)
    n = len(sources)
    hs = (_P * max(n, 1))(*[s._h for s in sources])
    s = _lib.am_plan_explain(text.encode(), hs, n, 1)
    if s is None:
        _ok(1)
    return s.decode()


# ---- CUDA additions ------------------------------------------------------------------------------

def set_stream(stream_ptr):
    """Enqueue this thread's calls on an existing cudaStream_t (an int address; 0 = the library's)."""
    _ok(_lib.am_cuda_set_stream(stream_ptr or None))


def synchronize():
    _ok(_lib.am_cuda_synchronize())


def last_sort_stats():
    s = SortStats()
    _ok(_lib.am_last_sort_stats(ctypes.byref(s)))
    return {"rows": s.rows, "value_rows": s.value_rows, "passes_run": s.passes_run,
            "passes_skipped": s.passes_skipped, "payload_in_records": bool(s.payload_in_records)}


def batch_tuning():
    """The segmented sort's shapes as its autotuner chose them: one dict per key width and size class
    (method -1: not measured yet, 0: digit passes, 1: one CTA per array)."""
    count = _I64()
    _ok(_lib.am_cuda_batch_tuning(None, 0, ctypes.byref(count)))
    shapes = (BatchShape * max(count.value, 1))()
    _ok(_lib.am_cuda_batch_tuning(shapes, count.value, ctypes.byref(count)))
    return [{name: getattr(sh, name) for name, _ in BatchShape._fields_} for sh in shapes[:count.value]]


def profile(on=True):
    _ok(_lib.am_cuda_profile(1 if on else 0))


def profile_reset():
    _ok(_lib.am_cuda_profile_reset())


def profile_entries():
    """{kernel name: (launches, total ms)} of the launches timed since the last reset."""
    out = {}
    n = _lib.am_cuda_profile_count()
    if n < 0:
        _ok(1)
    for i in range(n):
        name, launches, ms = ctypes.c_char_p(), _I64(), ctypes.c_double()
        _ok(_lib.am_cuda_profile_entry(i, ctypes.byref(name), ctypes.byref(launches), ctypes.byref(ms)))
        out[name.value.decode()] = (launches.value, ms.value)
    return out
