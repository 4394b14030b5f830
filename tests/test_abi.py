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


def test_input_packing_forms_agree_and_validate():
    """The p-vector forms the host accepts (a list of 1-d arrays, a narrow or
    full-width 2-d array) pack to the same (n_p, pfg_max_h11()) block; a
    full-width C-contiguous int64 array is used in place; entries beyond a
    geometry's h11 and a length mismatch with pgeo are rejected."""
    import numpy as np
    import pytest
    from pfvs_b200 import gpu, workloads
    from parity import layout
    geoms, ps, pgeo, _ = layout(workloads.build("mixed", n_p=64))
    MH = 64
    P_list = gpu._pack(geoms, ps, pgeo, MH)[6]
    W = max(len(p) for p in ps)
    narrow = np.zeros((len(ps), W), np.int64)
    for i, p in enumerate(ps):
        narrow[i, :len(p)] = p
    full = np.zeros((len(ps), MH), np.int64)
    full[:, :W] = narrow
    np.testing.assert_array_equal(gpu._pack(geoms, narrow, pgeo, MH)[6], P_list)
    P_full = gpu._pack(geoms, full, pgeo, MH)[6]
    assert P_full is full
    np.testing.assert_array_equal(P_full, P_list)
    h0 = np.asarray(geoms[int(pgeo[0])]["kappa"]).shape[0]
    for bad in (full.copy(), narrow.copy()):
        bad[0, h0] = 1
        with pytest.raises(ValueError):
            gpu._pack(geoms, bad, pgeo, MH)
    bad_list = [np.asarray(p) for p in ps]
    bad_list[0] = np.concatenate([bad_list[0], [0] * (h0 - len(bad_list[0])), [1]])
    with pytest.raises(ValueError):
        gpu._pack(geoms, bad_list, pgeo, MH)
    with pytest.raises(ValueError):
        gpu._pack(geoms, full[:-1], pgeo, MH)


def test_reference_loader_binds_this_library():
    """The reference's own loader (pfvs/gpu.py, loaded by file path; it needs
    only ctypes and numpy) binds this library through PFVS_GPU_LIB: its
    struct layouts and the six entry points resolve, the constants come
    through, and without a device its pipeline call ends in the library's
    error (RuntimeError with the err string), not in a crash.  (On a GPU
    machine the reference tree is absent; there the tests call the same
    exported pfg_coni_batch through pfvs_b200.gpu.)"""
    import ctypes
    import importlib.util
    import pytest
    from conftest import REFERENCE
    from pfvs_b200 import build, gpu
    path = os.path.join(REFERENCE, "pfvs", "gpu.py")
    if not os.path.exists(path):
        pytest.skip("the reference tree is not present")
    so = build.build()
    old = os.environ.get("PFVS_GPU_LIB")
    os.environ["PFVS_GPU_LIB"] = so
    try:
        spec = importlib.util.spec_from_file_location("reference_pfvs_gpu", path)
        refmod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(refmod)
        assert refmod._load() is not None, refmod._lib_error
        assert refmod.max_h11() == 64 and refmod.backend() == "cuda"
        assert ctypes.sizeof(refmod._Input) == ctypes.sizeof(gpu._Input)
        assert ctypes.sizeof(refmod._Output) == ctypes.sizeof(gpu._Output)
        if not refmod.available():
            import numpy as np
            from pfvs_b200 import workloads
            w = workloads.build("small", n_p=4)
            g = w.geoms[0]
            geoms = [dict(kappa=g.kappa, Mbasis=g.Mbasis, Q=g.Q, dilation=1.0, M0min=13)]
            with pytest.raises(RuntimeError, match="GPU pipeline failed"):
                refmod.coni_batch_multi(geoms, w.ps, np.zeros(len(w.ps), np.int32))
    finally:
        if old is None:
            os.environ.pop("PFVS_GPU_LIB", None)
        else:
            os.environ["PFVS_GPU_LIB"] = old
