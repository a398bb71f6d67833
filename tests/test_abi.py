"""The C ABI library loads, exports every declared entry point, and rejects
bad arguments with error codes (no device work: these run without a GPU)."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "b200sa.h")


def declared_functions():
    text = open(HEADER).read()
    return re.findall(r"B200SA_API\s+[\w\s\*]*?\b(b200sa_\w+)\s*\(", text)


def test_library_is_built_and_loads():
    from b200sa import _lib
    assert os.path.exists(_lib.LIB_PATH), "run python dwave-samplers_b200/build.py"
    L = _lib.load()
    assert L.b200sa_version().decode().startswith("b200sa")


def test_every_declared_symbol_is_exported():
    from b200sa import _lib
    names = declared_functions()
    assert set(names) >= {"b200sa_sample", "b200sa_sample_batch", "b200sa_plan_create",
                          "b200sa_plan_run", "b200sa_plan_destroy", "b200sa_plan_layout",
                          "b200sa_version"}
    lib = ctypes.CDLL(_lib.LIB_PATH)
    for name in names:
        assert hasattr(lib, name), f"{name} declared in include/b200sa.h but not exported"
    assert set(names) <= set(_lib.EXPORTS) | set(names)


def test_header_enums_match_reference_values():
    # cpu_sa.h:36-43 numbering
    text = open(HEADER).read()
    assert re.search(r"#define B200SA_GIBBS 0", text)
    assert re.search(r"#define B200SA_METROPOLIS 1", text)
    assert re.search(r"#define B200SA_SEQUENTIAL 0", text)
    assert re.search(r"#define B200SA_RANDOM 1", text)


def test_invalid_coupler_is_an_error_code_not_an_abort():
    # cpu_sa.cpp:302-304 throws (the process aborts); the C ABI returns EINVAL
    # before touching a device.
    from b200sa import simulated_annealing
    st = np.ones((2, 3), dtype=np.int8)
    with pytest.raises(ValueError, match="invalid variable"):
        simulated_annealing(2, [0.0, 0.0, 0.0], [0], [5], [1.0], 1, [1.0], 1, st)
    with pytest.raises(ValueError, match="invalid variable"):
        simulated_annealing(2, [0.0, 0.0, 0.0], [-1], [1], [1.0], 1, [1.0], 1, st)


def test_raw_abi_error_codes():
    from b200sa import _lib
    L = _lib.load()
    err = _lib.errbuf()
    h = np.zeros(3)
    u = np.array([0], np.int32)
    v = np.array([7], np.int32)
    J = np.ones(1)
    st = np.ones(3, np.int8)
    en = np.zeros(1)
    b = np.ones(1)
    seeds = np.ones(1, np.uint64)
    rc = L.b200sa_sample(3, h.ctypes.data, 1, u.ctypes.data, v.ctypes.data, J.ctypes.data, 1,
                         st.ctypes.data, en.ctypes.data, 1, 1, b.ctypes.data, seeds.ctypes.data,
                         1, 0, 1, _lib.INTERRUPT_FN(), None, 0, None, err, len(err))
    assert rc == _lib.EINVAL and b"invalid variable" in err.value
    # bad proposal enum
    v[0] = 1
    rc = L.b200sa_sample(3, h.ctypes.data, 1, u.ctypes.data, v.ctypes.data, J.ctypes.data, 1,
                         st.ctypes.data, en.ctypes.data, 1, 1, b.ctypes.data, seeds.ctypes.data,
                         1, 0, 7, _lib.INTERRUPT_FN(), None, 0, None, err, len(err))
    assert rc == _lib.EINVAL
    # num_seeds must be 1 or num_reads
    rc = L.b200sa_sample(3, h.ctypes.data, 1, u.ctypes.data, v.ctypes.data, J.ctypes.data, 1,
                         st.ctypes.data, en.ctypes.data, 1, 1, b.ctypes.data, seeds.ctypes.data,
                         3, 0, 1, _lib.INTERRUPT_FN(), None, 0, None, err, len(err))
    assert rc == _lib.EINVAL
    # zero reads completes trivially
    rc = L.b200sa_sample(3, h.ctypes.data, 1, u.ctypes.data, v.ctypes.data, J.ctypes.data, 0,
                         st.ctypes.data, en.ctypes.data, 1, 1, b.ctypes.data, seeds.ctypes.data,
                         1, 0, 1, _lib.INTERRUPT_FN(), None, 0, None, err, len(err))
    assert rc == 0


def test_no_device_reports_enodev(gpu_available):
    if gpu_available:
        pytest.skip("a GPU is present")
    from b200sa import simulated_annealing
    st = np.ones((1, 3), dtype=np.int8)
    with pytest.raises(RuntimeError, match="device"):
        simulated_annealing(1, [0.0, 0.1, 0.0], [0], [1], [1.0], 1, [1.0], 1, st)
