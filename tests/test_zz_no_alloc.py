"""
pfg_coni_direction_static -- the entry point for callers that cannot
allocate device memory while they run (code inside a framework that owns
all device memory through its own pool or arena, where an allocation of the
library's own would go around that pool or fail): given device buffers for
the inputs and outputs, it runs the whole pipeline for one p-vector with its
scratch in a static device array.  Its rows must equal pfg_coni_batch's rows
for the same p-vector, element for element (the same bit-exact bar as the
other parity tests), on two calls in a row (the second call finds the
scratch the first one left behind), for every h11 class the library
handles (h11 <= 32 and the two-slot search of h11 = 40 and 60).

The test allocates the device buffers itself (the caller's side) with torch.
This file sorts last so that a run stopping at its first failure has run
every other test before it.
"""
import ctypes

import numpy as np
import pytest

from pfvs_b200 import gpu, workloads
from parity import layout

pytestmark = pytest.mark.gpu

MH = 64
CAP = 2048          # PFG_STATIC_MAX_POINTS


def _entry(lib):
    f = lib.pfg_coni_direction_static
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_int, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64,
                  ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64,
                  ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                  ctypes.c_void_p, ctypes.c_void_p]
    return f


def _cases():
    """(geometries, p-vectors, pgeo, h11s) with a spread of point counts and
    every h11 class: 8..32 (one search level per lane), 40 and 60 (two)."""
    out = []
    for name, n, dils in [("mixed", 96, None), ("plain", 48, (150.0,)), ("small", 32, (800.0,)),
                          ("precision", 16, None), ("large", 12, (10.0,))]:
        w = workloads.build(name, n_p=n, dilations=dils)
        out.append(layout(w))
    return out


class _Caller:
    """The caller's side: device buffers (torch) and the call."""

    def __init__(self, torch, cap=CAP):
        self.torch = torch
        self.f = _entry(gpu._require())
        self.dev = torch.device("cuda", 0)
        z = lambda *s, dt=torch.int64: torch.zeros(s, dtype=dt, device=self.dev)
        self.M, self.K, self.q = z(cap, MH), z(cap, MH), z(cap)
        self.n, self.st = z(1), z(1, dt=torch.int32)
        self.stream = torch.cuda.current_stream(self.dev).cuda_stream

    def inputs(self, g, p):
        t = self.torch
        kap = t.tensor(np.ascontiguousarray(g["kappa"], dtype=np.int64).ravel(), device=self.dev)
        mb = t.tensor(np.ascontiguousarray(g["Mbasis"], dtype=np.int64).ravel(), device=self.dev)
        return kap, mb, t.tensor(np.asarray(p, dtype=np.int64), device=self.dev)

    def call(self, g, inputs, cap):
        kap, mb, p = inputs
        h = np.asarray(g["kappa"]).shape[0]
        return self.f(h, int(g["Q"]), gpu._qmax(int(g["Q"]), g["dilation"]),
                      int(np.ceil(g["M0min"] - 1e-9)), kap.data_ptr(), mb.data_ptr(), p.data_ptr(),
                      cap, self.M.data_ptr(), self.K.data_ptr(), self.q.data_ptr(), self.n.data_ptr(),
                      self.st.data_ptr(), self.stream)


@pytest.fixture(scope="module")
def caller():
    torch = pytest.importorskip("torch")
    if not gpu.available():
        pytest.fail("no CUDA device: " + gpu.unavailable_reason())
    return _Caller(torch)


def test_static_entry_matches_batch_entry(caller):
    torch = caller.torch
    checked, with_points, wide = 0, 0, 0
    for geoms, ps, pgeo, hs in _cases():
        M, Kn, q, pidx, pstat, _ = gpu.coni_batch_multi(geoms, ps, pgeo)     # the existing entry point
        counts = np.bincount(pidx, minlength=len(ps)) if len(pidx) else np.zeros(len(ps), int)
        for i in range(len(ps)):
            if counts[i] > CAP:
                continue
            g = geoms[pgeo[i]]
            inputs = caller.inputs(g, ps[i])
            sel = pidx == i
            for call in range(2):                     # two calls in a row
                assert caller.call(g, inputs, CAP) == 0
                torch.cuda.synchronize(caller.dev)
                n = int(caller.n.item())
                assert int(caller.st.item()) == int(pstat[i])
                assert n == int(counts[i])
                np.testing.assert_array_equal(caller.M[:n].cpu().numpy(), M[sel])
                np.testing.assert_array_equal(caller.K[:n].cpu().numpy(), Kn[sel])
                np.testing.assert_array_equal(caller.q[:n].cpu().numpy(), q[sel])
            checked += 1
            with_points += counts[i] > 0
            wide += hs[pgeo[i]] > 32
    assert checked > 150 and with_points > 5 and wide >= 20


def test_static_entry_reports_too_many_points(caller):
    """A direction with k points, called with room for k - 1: status -2 and no
    rows (the batch entry point's own count decides k)."""
    torch = caller.torch
    w = workloads.build("mixed", n_p=96)
    geoms, ps, pgeo, _ = layout(w)
    M, Kn, q, pidx, pstat, _ = gpu.coni_batch_multi(geoms, ps, pgeo)
    counts = np.bincount(pidx, minlength=len(ps))
    i = int(np.argmax(np.where(counts <= CAP, counts, 0)))
    k = int(counts[i])
    assert k >= 2
    g = geoms[pgeo[i]]
    inputs = caller.inputs(g, ps[i])
    assert caller.call(g, inputs, k - 1) == 0
    torch.cuda.synchronize(caller.dev)
    assert int(caller.st.item()) == -2 and int(caller.n.item()) == 0
    assert caller.call(g, inputs, k) == 0                  # and with room for exactly k
    torch.cuda.synchronize(caller.dev)
    assert int(caller.st.item()) == 0 and int(caller.n.item()) == k
    np.testing.assert_array_equal(caller.M[:k].cpu().numpy(), M[pidx == i])


def test_static_entry_allocates_nothing(caller):
    """After a first call (which loads the kernel and looks up the scratch's
    address), further calls leave the device's free memory unchanged: the
    library allocates nothing for them."""
    torch = caller.torch
    w = workloads.build("mixed", n_p=8)
    geoms, ps, pgeo, _ = layout(w)
    ins = [(geoms[pgeo[i]], caller.inputs(geoms[pgeo[i]], ps[i])) for i in range(len(ps))]
    assert caller.call(ins[0][0], ins[0][1], CAP) == 0
    torch.cuda.synchronize(caller.dev)
    free0, _ = torch.cuda.mem_get_info(caller.dev)
    for g, inputs in ins * 2:
        assert caller.call(g, inputs, CAP) == 0
    torch.cuda.synchronize(caller.dev)
    free1, _ = torch.cuda.mem_get_info(caller.dev)
    assert free1 == free0


def test_static_entry_rejects_oversized_requests():
    lib = gpu._require()
    f = _entry(lib)
    assert f(65, 1, 1, 13, 1, 1, 1, 0, 1, 1, 1, 1, 1, None) == 1          # h11 beyond 64
    assert f(5, 1, 1, 13, 1, 1, 1, CAP + 1, 1, 1, 1, 1, 1, None) == 1     # cap beyond the static scratch
