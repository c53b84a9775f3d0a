"""Shared test set-up: the `gpu` marker, the golden fixtures, and array builders.

Tests marked `gpu` need a B200 and call the library through its C ABI (via the ctypes binding
`arrowmetal_b200`); everything else runs on a CPU-only machine.
"""
import json
import os
import sys

import numpy as np
import pyarrow as pa
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden", "sort_golden.npz")

TYPES = {str(t): t for t in (pa.bool_(), pa.int8(), pa.uint8(), pa.int16(), pa.uint16(), pa.int32(), pa.uint32(),
                             pa.int64(), pa.uint64(), pa.float16(), pa.float32(), pa.float64())}


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); calls the library through its C ABI")


def build_array(t, values, valid=None):
    """A pyarrow array over exactly these value bits (NaN payloads and -0.0 kept) and validity."""
    if isinstance(t, str):
        t = TYPES[t]
    n = len(values)
    vbuf = None
    if valid is not None:
        vbuf = pa.py_buffer(np.packbits(np.asarray(valid, dtype=np.uint8), bitorder="little").tobytes())
    return pa.Array.from_buffers(t, n, [vbuf, pa.py_buffer(np.ascontiguousarray(values).tobytes())],
                                 null_count=-1 if valid is not None else 0)


class Golden:
    def __init__(self):
        self.z = np.load(GOLDEN)
        self.cases = json.loads(bytes(self.z["cases_json"]).decode())

    def array(self, name, t):
        valid = self.z[name + "_valid"] if (name + "_valid") in self.z.files else None
        return build_array(t, self.z[name + "_values"], valid)

    def __getitem__(self, k):
        return self.z[k]


_golden = None


def golden():
    global _golden
    if _golden is None:
        _golden = Golden()
    return _golden


@pytest.fixture(scope="session")
def am():
    import arrowmetal_b200
    arrowmetal_b200.set_router("gpu")
    return arrowmetal_b200


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as o
    o.lib()
    return o
