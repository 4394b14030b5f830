"""
pfg_coni_direction_static -- the entry point for callers that cannot
allocate device memory while they run (code inside a framework that owns
all device memory through its own pool, work issued during stream capture):
given device buffers for the inputs and outputs, it runs the whole pipeline
for one p-vector with its scratch in a static device array.  Its rows must
equal pfg_coni_batch's rows for the same p-vector, element for element
(the same bit-exact bar as the other parity tests), on two calls in a row
(the second call finds the scratch the first one left behind).

The test allocates the device buffers itself (the caller's side) with torch.
"""
import ctypes

import numpy as np
import pytest

from pfvs_b200 import gpu, workloads
from parity import layout

pytestmark = pytest.mark.gpu

MH = 64


def _entry(lib):
    f = lib.pfg_coni_direction_static
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_int, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64,
                  ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64,
                  ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                  ctypes.c_void_p, ctypes.c_void_p]
    return f


def _cases():
    """(geometry spec, p-vectors) with a spread of point counts."""
    out = []
    for name, n, dils in [("mixed", 96, None), ("plain", 48, (150.0,)), ("small", 32, (800.0,))]:
        w = workloads.build(name, n_p=n, dilations=dils)
        out.append(layout(w))
    return out


def test_static_entry_matches_batch_entry():
    torch = pytest.importorskip("torch")
    if not gpu.available():
        pytest.fail("no CUDA device: " + gpu.unavailable_reason())
    lib = gpu._require()
    f = _entry(lib)
    cap = 2048
    dev = torch.device("cuda", 0)
    dM = torch.zeros((cap, MH), dtype=torch.int64, device=dev)
    dK = torch.zeros((cap, MH), dtype=torch.int64, device=dev)
    dq = torch.zeros(cap, dtype=torch.int64, device=dev)
    dn = torch.zeros(1, dtype=torch.int64, device=dev)
    dst = torch.zeros(1, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    checked = with_points = 0
    for geoms, ps, pgeo, hs in _cases():
        M, Kn, q, pidx, pstat, _ = gpu.coni_batch_multi(geoms, ps, pgeo)     # the existing entry point
        counts = np.bincount(pidx, minlength=len(ps)) if len(pidx) else np.zeros(len(ps), int)
        for i in range(len(ps)):
            if counts[i] > cap:
                continue
            g = geoms[pgeo[i]]
            h = np.asarray(g["kappa"]).shape[0]
            kap = torch.tensor(np.ascontiguousarray(g["kappa"], dtype=np.int64).ravel(), device=dev)
            mb = torch.tensor(np.ascontiguousarray(g["Mbasis"], dtype=np.int64).ravel(), device=dev)
            p = torch.tensor(np.asarray(ps[i], dtype=np.int64), device=dev)
            sel = pidx == i
            for call in range(2):                     # two calls in a row
                rc = f(h, int(g["Q"]), gpu._qmax(int(g["Q"]), g["dilation"]),
                       int(np.ceil(g["M0min"] - 1e-9)), kap.data_ptr(), mb.data_ptr(), p.data_ptr(),
                       cap, dM.data_ptr(), dK.data_ptr(), dq.data_ptr(), dn.data_ptr(), dst.data_ptr(),
                       stream)
                assert rc == 0
                torch.cuda.synchronize(dev)
                n = int(dn.item())
                assert int(dst.item()) == int(pstat[i])
                assert n == int(counts[i])
                np.testing.assert_array_equal(dM[:n].cpu().numpy(), M[sel])
                np.testing.assert_array_equal(dK[:n].cpu().numpy(), Kn[sel])
                np.testing.assert_array_equal(dq[:n].cpu().numpy(), q[sel])
            checked += 1
            with_points += counts[i] > 0
    assert checked > 100 and with_points > 5


def test_static_entry_rejects_oversized_requests():
    lib = gpu._require()
    f = _entry(lib)
    assert f(65, 1, 1, 13, 1, 1, 1, 0, 1, 1, 1, 1, 1, None) == 1          # h11 beyond 64
    assert f(5, 1, 1, 13, 1, 1, 1, 4096, 1, 1, 1, 1, 1, None) == 1        # cap beyond the static scratch
