"""C-ABI checks that need no GPU: the library loads, exports every symbol the
header declares, and reports the reference's errors for bad files."""
import os
import re
import struct

import numpy as np
import pytest

from conftest import ROOT

import hrnn_b200 as H


def declared_symbols():
    syms = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            src = open(os.path.join(ROOT, "include", fn)).read()
            syms |= set(re.findall(r"^\s*(?:[\w\s\*]+?)\b(hrnn_\w+)\s*\(", src, re.M))
    return syms


def test_exports_every_declared_symbol():
    syms = declared_symbols()
    assert len(syms) >= 20
    for s in syms:
        assert hasattr(H.lib(), s), s
    assert set(H.EXPORTS) == syms


def test_version_and_l2_order():
    assert H.lib().hrnn_version() == 10000
    lanes, fused = H.detect_l2_order()
    assert lanes in (4, 8, 16) and fused in (0, 2)


def test_load_missing_file():
    with pytest.raises(H.HrnnError) as e:
        H.HRNN.load("/nonexistent/x.idx", 32)
    assert e.value.code == H.ERR_IO and str(e.value) == "Cannot open file"


def test_load_bad_magic(tmp_path):
    p = tmp_path / "bad.idx"
    p.write_bytes(b"\x00" * 256)
    with pytest.raises(H.HrnnError) as e:
        H.HRNN.load(str(p), 32)
    assert e.value.code == H.ERR_FORMAT and "bad magic" in str(e.value)


def test_load_truncated(tmp_path, golden_idx):
    raw = open(golden_idx, "rb").read()
    p = tmp_path / "trunc.idx"
    p.write_bytes(raw[:60])
    with pytest.raises(H.HrnnError) as e:
        H.HRNN.load(str(p), 32)
    assert e.value.code == H.ERR_FORMAT


def test_load_dim_mismatch(golden_idx):
    with pytest.raises(H.HrnnError) as e:
        H.HRNN.load(golden_idx, 64)
    assert e.value.code == H.ERR_FORMAT
