"""CPU-side checks of the C ABI library: it builds, loads without a GPU and
exports every function include/psm_b200.h declares; calls fail cleanly
(no crash) when no sm_100 device is present."""
import ctypes as C
import re
from pathlib import Path

import pytest

from psm_benchmark_b200 import native as N

ROOT = Path(__file__).resolve().parent.parent


def declared_functions(header: str):
    text = (ROOT / "include" / header).read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(psm_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = C.CDLL(str(N.LIB_PATH))
    names = declared_functions("psm_b200.h")
    assert len(names) >= 15
    for name in names:
        assert hasattr(lib, name), name
    assert set(names) == set(N.EXPORTS)


def test_generator_exports():
    from psm_benchmark_b200 import gen
    lib = gen._lib()
    for name in declared_functions("psm_gen.h"):
        assert hasattr(lib, name), name


def test_status_strings_and_version():
    L = N.lib()
    assert L.psm_status_string(0) == b"ok"
    assert L.psm_status_string(3) == b"time limit reached"
    assert b"sm_100a" in L.psm_version()


def test_method_parsing():
    assert N.parse_method("CFL_CFL_EXPLORE") == (2, 1, 2)
    assert N.parse_method("GQL_GQL_GQL") == (1, 0, 1)
    with pytest.raises(N.PsmError):
        N.parse_method("DPiso_DPiso_LFTJ")
    with pytest.raises(N.PsmError):
        N.parse_method("CFL_CFL")


def test_context_without_gpu_fails_cleanly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = C.c_void_p()
    rc = N.lib().psm_context_create(0, 1 << 20, C.byref(h))
    assert rc == N.PSM_ERR_CUDA
    assert N.lib().psm_last_error()


def header_defines(prefix: str):
    text = (ROOT / "include" / "psm_b200.h").read_text()
    return {m.group(1): int(m.group(2)) for m in re.finditer(rf"#define {prefix}([A-Z]+)\s+(\d+)", text)}


def test_binding_constants_match_the_header():
    """The Python names of the batch settings carry the header's values, and
    a psm_batch_tuning laid out by the binding has the C struct's size."""
    assert header_defines("PSM_ISECT_") == N.INTERSECTS
    assert header_defines("PSM_TEAM_") == N.TEAMS
    assert C.sizeof(N.BatchTuning) == 4 * 4 + 8
