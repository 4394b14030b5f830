"""The C-ABI library loads and exports every entry point include/pfvs_gpu.h
declares (no device needed)."""
import os
import re

from conftest import ROOT


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "pfvs_gpu.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(pfg_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_the_reference_interface():
    syms = declared_symbols()
    for s in ("pfg_max_h11", "pfg_backend", "pfg_device_count", "pfg_release",
              "pfg_coni_batch", "pfg_output_free"):
        assert s in syms


def test_library_exports_every_declared_symbol(lib):
    for s in declared_symbols():
        assert hasattr(lib, s), s


def test_library_constants(lib):
    assert lib.pfg_max_h11() == 64
    assert lib.pfg_backend() == b"cuda"


def test_struct_layouts_match_reference_ctypes():
    """pfg_input / pfg_output field order and types are the reference's
    (pfvs/gpu.py:37-50)."""
    from pfvs_b200 import gpu
    assert [f for f, _ in gpu._Input._fields_] == [
        "n_geo", "h", "Q", "qmax", "linmin", "kappa", "Mbasis", "n_p", "ps", "pgeo",
        "device", "batch", "verbose"]
    assert [f for f, _ in gpu._Output._fields_] == [
        "n", "M", "Kn", "q", "pidx", "pstat", "seconds_gpu", "err"]
