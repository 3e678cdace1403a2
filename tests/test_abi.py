"""The C-ABI library loads on a machine without a GPU and exports every
entry point declared in include/louvain_b200.h."""
import ctypes
import os
import re
import subprocess

import pytest

from conftest import ROOT


def declared_symbols():
    with open(os.path.join(ROOT, "include", "louvain_b200.h")) as f:
        text = f.read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(lv_[a-z0-9_]+)\s*\(", text)))


def test_header_symbols_exported(lvb):
    L = ctypes.CDLL(lvb.LIB_PATH)
    syms = declared_symbols()
    assert len(syms) >= 25
    missing = [s for s in syms if not hasattr(L, s)]
    assert not missing, missing
    assert sorted(lvb.EXPORTED) == syms


def test_status_strings(lvb):
    assert lvb.status_string(0) == "ok"
    assert "device" in lvb.status_string(lvb.LV_ERR_NO_DEVICE)


def test_library_is_sm100a(lvb):
    out = subprocess.run(["cuobjdump", "--list-elf", lvb.LIB_PATH], capture_output=True, text=True)
    if out.returncode != 0:
        pytest.skip("cuobjdump unavailable")
    assert "sm_100a" in out.stdout


def test_create_without_device_fails_loudly(lvb, gnp):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    rp, cl, w = gnp.csr_from_edges(3, [(0, 1, 1.0), (1, 2, 1.0)])
    with pytest.raises(lvb.LouvainError) as e:
        lvb.Louvain(lvb.Graph(rp, cl, w))
    assert e.value.status == lvb.LV_ERR_NO_DEVICE
