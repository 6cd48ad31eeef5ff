"""qv_velocity_direct_noalloc: the direct Biot-Savart sum without device allocation.

The entry point is for hosts that cannot call cudaMalloc/cudaFree on their hot
path: a driver that reserves its whole device memory budget up front and hands
out fixed buffers, a code whose device allocator belongs to another framework,
or a loop that cannot pay the device synchronisation those calls imply.  Its
temporaries live in one file-scope device array of fixed size.

The test calls it through the C ABI on device buffers, twice in a row, and
compares each result with the u_bs that the allocating entry point
qv_velocity returns for the same system, within the tolerances of the other
GPU tests: 1e-10 relative (FP64) and 1e-6 RMS relative (mixed precision), for
each boundary kind (the image sets and the ghost unwrapping differ).
This file is collected last so that a run stopping at its first failure has
already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _system():
    from qvort_b200 import workloads as W

    return W.random_rings(30, 0.006, 0.012, 5e-4, 0.1, seed=21)


@pytest.mark.parametrize("boundary", ["periodic", "open", "openx", "openxy"])
@pytest.mark.parametrize("prec,tol", [("fp64", 1e-10), ("mixed", 1e-6)])
def test_noalloc_matches_allocating_entry_point(prec, tol, boundary):
    import torch

    from qvort_b200 import lib as L

    w = _system()
    n = w.n
    assert 0 < n <= L.QV_NOALLOC_MAX_POINTS
    p = L.default_params(**dict(w.params, velocity="BS", tree_theta=0.0, precision=prec,
                                boundary=boundary))
    with L.Context(p) as c:
        c.set_points(w.x, w.infront, w.behind)
        _, _, ref, _ = c.velocity()

    dev = torch.device("cuda", 0)
    x = torch.tensor(w.x, dtype=torch.float64, device=dev)
    inf = torch.tensor(w.infront, dtype=torch.int32, device=dev)
    beh = torch.tensor(w.behind, dtype=torch.int32, device=dev)
    out = torch.empty((n, 3), dtype=torch.float64, device=dev)
    for _ in range(2):
        out.fill_(float("nan"))      # each call must write the whole result itself
        torch.cuda.synchronize()
        rc = L.lib().qv_velocity_direct_noalloc(C.byref(p), n, x.data_ptr(), inf.data_ptr(),
                                                beh.data_ptr(), out.data_ptr(), None)
        assert rc == 0, rc
        got = out.cpu().numpy()
        assert np.isfinite(got).all()
        if prec == "fp64":
            err = np.abs(got - ref).max() / np.abs(ref).max()
        else:
            err = np.sqrt(((got - ref) ** 2).sum() / (ref ** 2).sum())
        assert err < tol, err


def test_noalloc_rejects_more_points_than_its_array_holds():
    import torch

    from qvort_b200 import lib as L

    p = L.default_params(boundary="periodic", box_size=0.1)
    d = torch.zeros(8, dtype=torch.float64, device="cuda")
    i = torch.ones(8, dtype=torch.int32, device="cuda")
    rc = L.lib().qv_velocity_direct_noalloc(C.byref(p), L.QV_NOALLOC_MAX_POINTS + 1,
                                            d.data_ptr(), i.data_ptr(), i.data_ptr(),
                                            d.data_ptr(), None)
    assert rc == L.QV_ERR_NOALLOC_LIMIT
