"""Restart dump and restore from the context's device buffers.

data_dump / data_restore (src/output.f90:272-285, src/initial.f90:501-538):
a run interrupted after step k, dumped with qv_dump and restored into a new
context with qv_restore, continues as the run that was never interrupted -- the
state after the remaining steps is the same bit for bit (positions, history,
links, candidate pairs).  The run is the default loop (line operations on) on
a tangle whose first steps reconnect and remove points, in both precisions.
The var%04d.log snapshot written from the device buffers reads back as the
context's positions and links.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _mods():
    from qvort_b200 import lib as L
    from qvort_b200 import workloads as W

    return L, W


def _state(c):
    x, u = c.get_points()
    inf, beh = c.get_links()
    cl, cd = c.get_closest()
    h = c.get_history()
    return dict(x=x, u1=h[0], u2=h[1], u3=h[2], infront=inf, behind=beh, closest=cl, closestd=cd)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_resumed_run_is_bitwise_the_uninterrupted_run(tmp_path, precision):
    L, W = _mods()
    w = W.random_rings(40, 0.004, 0.012, 5e-4, 0.1, seed=3, theta=0.4, centre_box=0.03)
    prm = L.default_params(**dict(w.params, precision=precision, line_ops=2, recon_shots=2))
    k, total = 3, 7
    a = L.Context(prm)
    a.set_points(w.x, w.infront, w.behind)
    for it in range(1, k + 1):
        a.step(it)
    path = tmp_path / "var.dat"
    a.dump(path, itime=k, t=k * prm.dt, recon_count=0)
    for it in range(k + 1, total + 1):
        a.step(it)
    ref = _state(a)
    a.close()
    b = L.Context(prm)
    itime, t, _ = b.restore(path)
    assert itime == k and t == k * prm.dt
    for it in range(itime + 1, total + 1):
        b.step(it)
    got = _state(b)
    b.close()
    assert got["x"].shape == ref["x"].shape
    for key in ref:
        assert np.array_equal(got[key], ref[key]), key


def test_snapshot_from_device_buffers(tmp_path):
    L, W = _mods()
    w = W.random_rings(6, 0.006, 0.01, 5e-4, 0.1, seed=2, theta=0.4)
    c = L.Context(L.default_params(**w.params))
    c.set_points(w.x, w.infront, w.behind)
    c.step(1)
    path = tmp_path / "var0001.log"
    c.write_snapshot(path, 1e-7)
    x, _ = c.get_points()
    inf, beh = c.get_links()
    c.close()
    t, xr, infr, behr = L.read_var_file(path)
    assert t == 1e-7
    assert np.array_equal(xr, x) and np.array_equal(infr, inf) and np.array_equal(behr, beh)
