"""Failure detection without a GPU fault.

Every failure here is made on the host or by a test hook, and none reaches a
kernel as an out-of-bounds index or an endless wait:

* corrupted links (an index outside 0..n, an active slot linked to an empty
  slot, a closest index outside 0..n) are refused by qv_set_points,
  qv_set_state and qv_step_exchange: the links are checked on a staging copy
  before the context takes anything -- the check is the only launch -- and the
  context stays usable;
* a NaN in the positions of an empty slot (which no kernel reads) is reported
  at the end of the step as QV_ERR_NAN, as the reference's NAN_finder
  (src/general.f90:253-280, src/run.f90:168) stops the run;
* the bounded wait of the direct sum's source-tile copies: with the test hook
  on, every acquire reports a wait that ran out while the copies still land;
  the call drains them and returns QV_ERR_CUDA, and the next call, hook off,
  gives the clean result again, bit for bit.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _mods():
    from qvort_b200 import lib as L
    from qvort_b200 import workloads as W

    return L, W


def _tangle(W):
    return W.random_rings(8, 0.006, 0.012, 5e-4, 0.1, seed=11, theta=0.4)


def _corruptions(w):
    n = w.n
    out = []
    inf = w.infront.copy(); inf[3] = n + 5
    out.append(("infront out of range", inf, w.behind.copy(), None))
    beh = w.behind.copy(); beh[7] = -2
    out.append(("negative behind", w.infront.copy(), beh, None))
    inf = w.infront.copy(); beh = w.behind.copy()
    k = 10                      # slot k emptied, its neighbours still point at it
    inf[k] = 0; beh[k] = 0
    out.append(("active slot linked to an empty slot", inf, beh, None))
    cl = np.zeros(n, np.int32); cl[5] = n + 1
    out.append(("closest out of range", w.infront.copy(), w.behind.copy(), cl))
    return out


def test_corrupted_links_are_refused_before_the_context_changes():
    L, W = _mods()
    w = _tangle(W)
    c = L.Context(L.default_params(**dict(w.params, line_ops=2)))
    n = w.n
    # a state of its own, which the refused calls must leave as it is
    x0 = w.x + 1e-4
    c.set_points(x0, w.infront, w.behind)
    for name, inf, beh, cl in _corruptions(w):
        before = c.counters()["launches"]
        refused = 2
        if cl is None:
            with pytest.raises(L.QvError) as e:
                c.set_points(w.x, inf, beh)
            assert e.value.code == L.QV_ERR_ARG, name
            refused += 1
        with pytest.raises(L.QvError) as e:
            c.set_state(n, x=w.x, infront=inf, behind=beh, closest=cl)
        assert e.value.code == L.QV_ERR_ARG, name
        hist = [np.zeros((n, 3)) for _ in range(3)]
        inp = dict(x=w.x.copy(), infront=inf, behind=beh, u1=hist[0], u2=hist[1], u3=hist[2],
                   closest=cl if cl is not None else np.zeros(n, np.int32))
        out = dict(x=np.empty((2 * n, 3)), infront=np.empty(2 * n, np.int32),
                   behind=np.empty(2 * n, np.int32))
        with pytest.raises(L.QvError) as e:
            c.step_exchange(1, n, 2 * n, inp, out)
        assert e.value.code == L.QV_ERR_ARG, name
        # one launch per refused call: the check itself
        assert c.counters()["launches"] == before + refused, name
    assert c.n == n
    x1, _ = c.get_points()
    assert np.array_equal(x1, x0)
    # the context is still usable
    c.set_points(w.x, w.infront, w.behind)
    c.step(1)
    assert c.n >= n
    c.close()


@pytest.mark.parametrize("boundary", ["periodic", "open"])
def test_nan_position_is_reported_after_the_step(boundary):
    L, W = _mods()
    w = _tangle(W)
    # one extra empty slot whose position is NaN: no kernel reads it, the
    # end-of-step test finds it
    x = np.concatenate([w.x, [[np.nan, 0.0, 0.0]]])
    inf = np.concatenate([w.infront, [0]]).astype(np.int32)
    beh = np.concatenate([w.behind, [0]]).astype(np.int32)
    prm = dict(w.params, boundary=boundary)
    c = L.Context(L.default_params(**prm))
    c.set_points(x, inf, beh)
    with pytest.raises(L.QvError) as e:
        c.step(1)
    assert e.value.code == L.QV_ERR_NAN
    # the same system without the NaN steps cleanly
    c.set_points(w.x, w.infront, w.behind)
    c.step(1)
    c.close()


def test_stage_wait_timeout_returns_an_error_and_recovers():
    L, W = _mods()
    w = _tangle(W)
    res = {}
    for prec in ("fp64", "mixed"):
        c = L.Context(L.default_params(**dict(w.params, velocity="BS", tree_theta=0.0,
                                              precision=prec)))
        c.set_points(w.x, w.infront, w.behind)
        clean = c.velocity(False)[0]
        try:
            L.test_stage_timeout(True)
            with pytest.raises(L.QvError) as e:
                c.velocity(False)
            assert e.value.code == L.QV_ERR_CUDA
            assert "source-tile" in str(e.value)
        finally:
            L.test_stage_timeout(False)
        again = c.velocity(False)[0]
        assert np.array_equal(again, clean), prec
        res[prec] = clean
        c.close()


def test_stage_wait_timeout_in_the_allocation_free_entry_point():
    import torch

    L, W = _mods()
    w = _tangle(W)
    p = L.default_params(**dict(w.params, velocity="BS", tree_theta=0.0, precision="fp64"))
    dev = torch.device("cuda")
    x = torch.tensor(w.x, dtype=torch.float64, device=dev)
    inf = torch.tensor(w.infront, dtype=torch.int32, device=dev)
    beh = torch.tensor(w.behind, dtype=torch.int32, device=dev)
    u = torch.empty_like(x)
    call = L.lib().qv_velocity_direct_noalloc
    args = (C.byref(p), w.n, x.data_ptr(), inf.data_ptr(), beh.data_ptr(), u.data_ptr(), None)
    assert call(*args) == L.QV_OK
    clean = u.cpu().numpy().copy()
    try:
        L.test_stage_timeout(True)
        assert call(*args) == L.QV_ERR_CUDA
    finally:
        L.test_stage_timeout(False)
    assert call(*args) == L.QV_OK
    assert np.array_equal(u.cpu().numpy(), clean)
