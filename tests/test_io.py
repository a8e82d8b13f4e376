"""State I/O (include/abyss_io.h).

* CPU: the reader of the reference's input format gives the same code-unit
  values, bit for bit, as the reference's own Particle::initialize and
  normalizeParticle (src_mpi/particle.h:139-147,204-214); short lines read as
  zeros; a wrong particle count is refused.
* GPU: an integration saved between blocks and restored continues exactly as
  the uninterrupted one; the snapshot writer follows the reference's layout;
  a truncated checkpoint is refused.
"""
import ctypes as C

import numpy as np
import pytest

import oracle
from abyss_b200 import _lib, ic

dp = C.POINTER(C.c_double)


def _write_ic(path, rows):
    with open(path, "w") as f:
        for r in rows:
            f.write("  ".join(repr(float(x)) for x in r) + "\n")


def test_reader_count_and_short_lines(tmp_path):
    p = tmp_path / "ic.txt"
    rows = [[0.001, -0.002, 0.0005, 3.0, -1.5, 0.25, 1e-6], [0.002, 0.001]]
    _write_ic(p, rows)
    c = ic.read_reference(p, k_nb=0)
    assert c.x.shape == (2, 3)
    assert c.m[1] == 0.0 and np.all(c.v[1] == 0.0) and c.x[1, 2] == 0.0
    L = _lib.lib()
    n = C.c_int(5)
    x, v, m = np.zeros((5, 3)), np.zeros((5, 3)), np.zeros(5)
    rc = L.abyss_read_reference_ic(str(p).encode(), C.byref(n), x.ctypes.data_as(dp), v.ctypes.data_as(dp),
                                   m.ctypes.data_as(dp))
    assert rc == _lib.ABYSS_ERR_ARG  # the file holds 2 particles, not 5


@pytest.mark.skipif(not oracle.ref_available(), reason="reference CPU library not built")
def test_reader_matches_reference_units(tmp_path):
    rng = np.random.default_rng(13)
    rows = np.column_stack([rng.normal(0, 0.003, (64, 3)), rng.normal(0, 5.0, (64, 3)),
                            rng.lognormal(-14, 1.0, 64)])
    p = tmp_path / "ic.txt"
    _write_ic(p, rows)
    c = ic.read_reference(p, k_nb=8)
    R = oracle.ref()
    for i, r in enumerate(rows):
        x, v, m = np.zeros(3), np.zeros(3), np.zeros(1)
        R.ref_particle_from_row(oracle._p(np.ascontiguousarray(r)), oracle._p(x), oracle._p(v), oracle._p(m))
        assert np.array_equal(c.x[i], x) and np.array_equal(c.v[i], v) and c.m[i] == m[0], i


@pytest.mark.gpu
def test_checkpoint_restart_is_exact(tmp_path):
    from abyss_b200.integrator import ACIntegrator
    from abyss_b200.regforce import RegularForce

    c = ic.plummer(512, 31, k_nb=24)
    rf = RegularForce(0)
    try:
        kw = dict(eps2=1e-8, fix_nb=24, nb_max=96, t_end=1.0, threads=4)
        a = ACIntegrator(rf, c.x, c.v, c.m, c.r2nb, **kw)
        for _ in range(30):
            a.advance_block()
        path = tmp_path / "run.ckpt"
        a.save(path)
        for _ in range(30):
            a.advance_block()
        want = a.state()
        want_t = a.time
        b = ACIntegrator.load(rf, path, threads=4)
        assert b.n == a.n and b.nb_max == a.nb_max
        for _ in range(30):
            b.advance_block()
        got = b.state()
        assert b.time == want_t
        for k in ("x", "v", "nnb", "r2nb"):
            assert np.array_equal(got[k], want[k]), k
        # a snapshot in the reference's layout
        snap = tmp_path / "snap.txt"
        b.write_snapshot(snap, 1.5, 0.25)
        lines = snap.read_text().splitlines()
        assert lines[0].endswith(" Myr, ")
        assert lines[1].startswith("1.5, 0.25, ")
        assert lines[2].split()[:3] == ["PID", "Mass", "(Msun)"]
        assert len(lines) == 3 + b.n
        cols = np.array([[float(x) for x in ln.split()] for ln in lines[3:]])
        assert np.array_equal(cols[:, 0], np.arange(b.n))
        assert np.allclose(cols[:, 1], c.m * 0.0001424198, rtol=1e-6, atol=1e-8)
        # a truncated file is not a checkpoint
        bad = tmp_path / "bad.ckpt"
        bad.write_bytes(path.read_bytes()[:-100])
        with pytest.raises(_lib.AbyssError):
            ACIntegrator.load(rf, bad)
        a.close()
        b.close()
    finally:
        rf.close()
