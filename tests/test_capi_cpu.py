"""CPU-side checks of the C-ABI library: it loads, exports every declared entry point,
refuses to run without a device (no CPU fallback) and its host-side parts (the .ifs
bitstream) agree with the oracle."""
import os
import re

import numpy as np
import pytest

import mars_b200 as mb
from oracle import oracle as orc
from tests.conftest import cuda_available
from tests.golden_data import mars1_bytes, mars1_manifest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    src = open(os.path.join(ROOT, "include", "mars_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(mars_[a-z0-9_]+)\s*\(", src)))


def test_header_declarations_match_exports_list():
    assert declared_functions() == sorted(mb.EXPORTS)


def test_library_exports_every_declared_symbol():
    L = mb.lib()
    for name in declared_functions():
        assert hasattr(L, name), name


def test_version_string():
    assert b"sm_100a" in mb.lib().mars_version()


@pytest.mark.skipif(cuda_available(), reason="checks the no-device path")
def test_no_device_is_an_error_not_a_fallback():
    with pytest.raises(mb.MarsError) as e:
        mb.Context(0)
    assert e.value.code == -2


def test_ifs_roundtrip_matches_oracle_on_all_fixtures():
    for entry in mars1_manifest()["fixtures"]:
        data = mars1_bytes(entry)
        h, leaves = mb.ifs_parse(data)
        oh, ol = orc.ifs_parse(data)
        assert leaves.tobytes() == ol.tobytes()
        assert bytes(h) == bytes(oh)
        assert mb.ifs_write(h, leaves) == data


def test_ifs_rejects_truncated_and_padded_streams():
    data = mars1_bytes(mars1_manifest()["fixtures"][0])
    with pytest.raises(mb.MarsError) as e:
        mb.ifs_parse(data[: len(data) // 2])
    assert e.value.code == -7
    with pytest.raises(mb.MarsError):
        mb.ifs_parse(data + b"\x00")


def test_ifs_write_rejects_duplicate_leaves():
    data = mars1_bytes(mars1_manifest()["fixtures"][0])
    h, leaves = mb.ifs_parse(data)
    dup = np.concatenate([leaves, leaves[:1]])
    with pytest.raises(mb.MarsError):
        mb.ifs_write(h, dup)


def test_null_arguments_are_refused_without_a_device():
    # Entry points that take a plan or a context check their arguments before touching a
    # device: no CUDA call, no crash, MARS_EINVAL.
    import ctypes as C
    L = mb.lib()
    ms = C.c_float()
    assert L.mars_search_plan_kernel_ms(None, C.byref(ms)) == -1
    assert L.mars_ctx_set_search_path(None, 5) == -1
