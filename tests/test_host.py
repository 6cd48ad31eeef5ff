"""CPU tests of the host side (qv_read_run_file, var files, ring set-ups) and
the qvort_run driver executable (GPU)."""
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]


def _lib():
    from qvort_b200 import build

    build.build()
    from qvort_b200 import lib as L

    return L


def test_read_run_file_keys_and_defaults(tmp_path):
    L = _lib()
    f = tmp_path / "run.in"
    f.write_text(
        "--------------required parameters------------\n"
        "nsteps 1000\nshots 100\npcount 200\ndt 1E-7\ndelta 5.0d-4\nbox_size 0.1\n"
        "velocity Tree\ninitf single_loop\nboundary periodic\n"
        "tree_theta 0.4\ntree_extra_correction F\nruntime_label ignored\n"
        "deriv_order fourth\nquant_circ 9.97E-4\ncorea 1.3e-8\ngpu_precision fp64\n")
    r = L.read_run_file(f)
    assert (r.nsteps, r.shots, r.pcount) == (1000, 100, 200)
    assert r.p.dt == 1e-7 and r.p.delta == 5e-4 and r.p.box_size == 0.1
    assert r.p.velocity == L.VELOCITY["Tree"] and r.p.boundary == L.BC["periodic"]
    assert r.p.tree_theta == 0.4 and r.p.tree_extra_correction == 0
    assert r.p.deriv_order == 4 and r.p.corea == 1.3e-8 and r.p.precision == 0
    assert r.initf == b"single_loop"
    assert r.p.recon_shots == 1          # default (src/cdata.f90:198)


def test_read_run_file_stops_at_unreadable_value(tmp_path):
    """A value that fails its list-directed read sets iostat /= 0, which ends
    the reading loop (src/cdata.f90:434-437): later lines are not read."""
    L = _lib()
    f = tmp_path / "run.in"
    f.write_text("nsteps 10\ndt abc\nshots 7\n")
    with pytest.raises(L.QvError):
        L.read_run_file(f)


def test_var_file_round_trip_and_behind(tmp_path):
    L = _lib()
    from qvort_b200 import workloads as W

    w = W.random_rings(4, 0.005, 0.01, 5e-4, seed=3)
    inf = w.infront.copy()
    inf[5] = 0                      # an empty slot
    u = np.random.default_rng(0).normal(size=w.x.shape)
    p = tmp_path / "var0001.log"
    L.write_var_file(p, 1.5e-5, w.x, inf, u)
    t, x, inf2, beh = L.read_var_file(p)
    assert t == 1.5e-5
    np.testing.assert_array_equal(x, w.x)
    np.testing.assert_array_equal(inf2, inf)
    act = inf != 0
    expect = w.behind.copy()
    expect[inf == 0] = 0
    # slot 6's ring predecessor lost its infront link: no j points to it
    expect[w.infront[5] - 1] = 0 if inf[w.infront[5] - 1] != 0 else expect[w.infront[5] - 1]
    np.testing.assert_array_equal(beh[act], expect[act])
    # record layout: 8 + 4 + 3*8n + 4n + 3*8n + 8*8n bytes
    n = w.n
    assert p.stat().st_size == 12 + 24 * n + 4 * n + 24 * n + 64 * n


def test_setup_loops_match_reference_geometry():
    L = _lib()
    x, inf, beh = L.setup_loops("single_loop", 200, 5e-4)
    R = 0.75 * 200 * 5e-4 / (2 * np.pi)
    np.testing.assert_allclose(np.linalg.norm(x, axis=1), R, rtol=1e-15)
    assert inf[-1] == 1 and beh[0] == 200 and inf[0] == 2
    x2, inf2, beh2 = L.setup_loops("leap-frog", 100, 5e-4)
    assert np.all(x2[50:, 2] == 2 * 5e-4) and inf2[49] == 1 and inf2[99] == 51 and beh2[50] == 100
    with pytest.raises(L.QvError):
        L.setup_loops("random_loops", 100, 5e-4)


@pytest.mark.gpu
def test_qvort_run_driver_matches_oracle(tmp_path):
    """The C++ driver on a single_loop run.in, against the oracle's own steps."""
    from oracle import oracle as O

    L = _lib()
    nsteps = 50
    (tmp_path / "run.in").write_text(
        f"nsteps {nsteps}\nshots {nsteps}\npcount 200\ndt 1e-7\ndelta 5e-4\nbox_size 0.1\n"
        "velocity BS\ninitf single_loop\nboundary open\ncorea 1.3e-8\ngpu_precision fp64\n")
    exe = ROOT / "qvort_b200" / "qvort_run"
    r = subprocess.run([str(exe)], cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    t, x, inf, beh = L.read_var_file(tmp_path / "data" / "var0001.log")
    assert abs(t - nsteps * 1e-7) < 1e-20
    x0, inf0, beh0 = L.setup_loops("single_loop", 200, 5e-4)
    st = O.State(O.params(velocity="BS", boundary="open", box_size=0.1, dt=1e-7, delta=5e-4,
                          corea=1.3e-8), x0, inf0, beh0)
    for _ in range(nsteps):
        st.step()
    d = np.abs(x - st.x).max() / np.abs(st.x - x0).max()
    assert d < 1e-8, d


def _gfortran_records(path):
    """An independent reader of gfortran's sequential unformatted layout: the
    payloads of the records, each checked for equal leading and trailing
    4-byte length markers."""
    raw = Path(path).read_bytes()
    recs, k = [], 0
    while k < len(raw):
        m = int(np.frombuffer(raw[k:k + 4], np.int32)[0])
        recs.append(raw[k + 4:k + 4 + m])
        assert int(np.frombuffer(raw[k + 4 + m:k + 8 + m], np.int32)[0]) == m
        k += 8 + m
    return recs


def test_restart_file_layout_and_round_trip(tmp_path):
    """data_dump's var.dat (src/output.f90:272-285): seven records (pcount,
    recon_count, itime, t, f(:), quasi_pcount, part_count) with gfortran's
    4-byte markers, f(:) as pcount records of the 464-byte type qvort under
    -fdefault-real-8; the reader returns every field written, bit for bit."""
    from qvort_b200 import lib as L

    rng = np.random.default_rng(4)
    n = 37
    f = {k: rng.normal(size=(n, 3)) for k in L.RESTART_VEC}
    f["closestd"] = rng.uniform(size=n)
    f["infront"] = rng.integers(0, n + 1, n).astype(np.int32)
    f["behind"] = rng.integers(0, n + 1, n).astype(np.int32)
    f["closest"] = rng.integers(0, n + 1, n).astype(np.int32)
    path = tmp_path / "var.dat"
    L.write_restart_file(path, t=1.25e-4, itime=1250, recon_count=17, **f)
    recs = _gfortran_records(path)
    assert len(recs) == 7
    assert np.frombuffer(recs[0], np.int32)[0] == n
    assert np.frombuffer(recs[1], np.int32)[0] == 17
    assert np.frombuffer(recs[2], np.int32)[0] == 1250
    assert np.frombuffer(recs[3], np.float64)[0] == 1.25e-4
    assert len(recs[4]) == n * 464
    assert np.frombuffer(recs[5], np.int32)[0] == 0 and np.frombuffer(recs[6], np.int32)[0] == 0
    # the record type by offset: x at 0, u at 48, ghosti at 264, infront at
    # 400, behind at 404, closest at 408, closestd at 416, delta at 440
    e = np.frombuffer(recs[4], np.uint8).reshape(n, 464)
    np.testing.assert_array_equal(e[:, 0:24].copy().view(np.float64), f["x"])
    np.testing.assert_array_equal(e[:, 48:72].copy().view(np.float64), f["u"])
    np.testing.assert_array_equal(e[:, 264:288].copy().view(np.float64), f["gi"])
    np.testing.assert_array_equal(e[:, 400:404].copy().view(np.int32)[:, 0], f["infront"])
    np.testing.assert_array_equal(e[:, 404:408].copy().view(np.int32)[:, 0], f["behind"])
    np.testing.assert_array_equal(e[:, 408:412].copy().view(np.int32)[:, 0], f["closest"])
    np.testing.assert_array_equal(e[:, 416:424].copy().view(np.float64)[:, 0], f["closestd"])
    assert (e[:, 440:448].copy().view(np.float64) == 1.0).all()
    t, itime, rcn, g = L.read_restart_file(path)
    assert (t, itime, rcn) == (1.25e-4, 1250, 17)
    for k, v in f.items():
        np.testing.assert_array_equal(g[k], v, err_msg=k)


def test_restart_file_rejects_a_foreign_layout(tmp_path):
    """A var.dat whose f(:) record is not pcount * 464 bytes (another compiler
    layout or another type) is refused."""
    from qvort_b200 import lib as L

    path = tmp_path / "var.dat"
    with open(path, "wb") as fh:
        for payload in (np.int32(3).tobytes(), np.int32(0).tobytes(), np.int32(5).tobytes(),
                        np.float64(0.5).tobytes(), bytes(3 * 456), np.int32(0).tobytes(),
                        np.int32(0).tobytes()):
            m = np.int32(len(payload)).tobytes()
            fh.write(m + payload + m)
    with pytest.raises(L.QvError):
        L.read_restart_file(path)
