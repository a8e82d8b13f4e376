"""The host integrator's irregular steps and regular blocks, on the CPU, from a
checkpoint.

tests/golden/ac_plummer1024_b200.ckpt holds configuration 1 (Plummer N = 1024,
seed 1) after 200 regular blocks, written on a GPU by
tests/golden/make_ac_checkpoint.py.  Loaded without a GPU context
(ACIntegrator.load(None, ...); include/abyss_io.h), the integration runs the
irregular levels up to its next regular block (begin_block), and then whole
regular blocks whose forces come from the FP64 oracle (the split form:
block_state, end_block).  The resulting positions and velocities:
  * are the same, bit for bit, for 1 and 4 host threads (a level's particles
    are computed from the pre-level state and committed one by one);
  * match the digests recorded when the fixture was made, which pin the host's
    step (prediction, the vectorised neighbour terms, the correctors, neighbour
    changes, the time-step rules, radius updates, the level order) against any
    change of its results;
  * are the same again for four integrations advanced at once on four host
    threads, one thread each (how the serving loop runs them).
Calls that need the GPU raise instead of touching a device.
"""
import hashlib
import os

import numpy as np
import pytest

from abyss_b200 import _lib
from abyss_b200.integrator import ACIntegrator

HERE = os.path.dirname(os.path.abspath(__file__))
CKPT = os.path.join(HERE, "golden", "ac_plummer1024_b200.ckpt")
# sha256 of x then v (float64, [1024][3] each) after the first begin_block
STATE_DIGEST = "386e0cf5ccd5fe789ef67b0a5698b29b73fec2f20df81498168b89cb6dbaa162"
# the same after 30 regular blocks driven by the FP64 oracle's regular force
BLOCKS30_DIGEST = "de20b636a5ada0dc9cf4010882b1765f04feddbe321631f5507bbf20c8217a22"


def _digest(ac):
    st = ac.state()
    return hashlib.sha256(st["x"].tobytes() + st["v"].tobytes()).hexdigest()


def _load(threads):
    try:
        return ACIntegrator.load(None, CKPT, threads=threads)
    except (RuntimeError, OSError) as exc:
        pytest.skip(f"library not built: {exc}")


def run_blocks_with_oracle(ac, blocks):
    """Regular blocks of the split form, their forces from the FP64 oracle."""
    import oracle

    done_blocks = 0
    for _ in range(blocks):
        blk = ac.begin_block()
        if blk is None:
            break
        targets, new_time, scale = blk
        st = ac.block_state()
        px, pv = oracle.predict(st["x"], st["v"], st["a0"], st["a1"], st["t0"], new_time, scale)
        ref = oracle.reg_force(px, pv, st["mass"], st["r2nb"], ac.params.eps2, targets, ac.nb_max)
        out = ac.end_block(ref["acc_reg"], ref["jerk_reg"], ref["acc_irr"], ref["jerk_irr"], ref["nnb"],
                           ref["list"])
        assert out in ("ok", "done"), out
        done_blocks += 1
        if out == "done":
            break
    return done_blocks


def test_irregular_levels_from_checkpoint_on_cpu():
    digests = []
    for threads in (1, 4):
        ac = _load(threads)
        try:
            blk = ac.begin_block()
            assert blk is not None and len(blk[0]) > 0
            digests.append(_digest(ac))
            with pytest.raises(_lib.AbyssError):
                ac.energy()  # needs the GPU
        finally:
            ac.close()
    assert digests == [STATE_DIGEST, STATE_DIGEST]


def test_regular_blocks_with_the_oracle_force_on_cpu():
    digests = []
    for threads in (1, 4):
        ac = _load(threads)
        try:
            assert run_blocks_with_oracle(ac, 30) == 30
            digests.append(_digest(ac))
        finally:
            ac.close()
    assert digests == [BLOCKS30_DIGEST, BLOCKS30_DIGEST]


def test_concurrent_integrations_on_host_threads():
    """The serving pattern: several integrations, one host thread each (no
    thread team inside), advanced at the same time.  Each reaches the digest
    of the lone run."""
    import threading

    acs = [_load(1) for _ in range(4)]
    digests = [None] * len(acs)
    errors = []

    def work(k):
        try:
            assert run_blocks_with_oracle(acs[k], 30) == 30
            digests[k] = _digest(acs[k])
        except Exception as exc:  # reported below, on the main thread
            errors.append(exc)

    threads = [threading.Thread(target=work, args=(k,)) for k in range(len(acs))]
    try:
        for t in threads:
            t.start()
        for t in threads:
            t.join()
    finally:
        for ac in acs:
            ac.close()
    assert not errors, errors
    assert digests == [BLOCKS30_DIGEST] * len(acs)


def test_save_load_round_trip_on_cpu(tmp_path):
    """A checkpoint saved after host-only blocks loads back to the same state,
    continues to the same digest, and saves to the same bytes."""
    ac = _load(2)
    try:
        assert run_blocks_with_oracle(ac, 10) == 10
        path = tmp_path / "mid.ckpt"
        ac.save(str(path))
        assert run_blocks_with_oracle(ac, 20) == 20
        want = _digest(ac)
    finally:
        ac.close()
    b = ACIntegrator.load(None, str(path), threads=2)
    try:
        again = tmp_path / "again.ckpt"
        b.save(str(again))
        assert again.read_bytes() == path.read_bytes()
        assert run_blocks_with_oracle(b, 20) == 20
        assert _digest(b) == want == BLOCKS30_DIGEST
    finally:
        b.close()


def test_damaged_checkpoints_are_refused(tmp_path):
    """Truncated files, a wrong magic and damaged particle counts are refused
    with an error: never read past their end, never allocated for."""
    data = open(CKPT, "rb").read()
    cases = {f"cut{k}": data[:k] for k in (0, 7, 8, 64, len(data) // 2, len(data) - 8, len(data) - 1)}
    cases["magic"] = b"NOTABYSS" + data[8:]
    cases["tail"] = data[:-8] + b"NOTABYSS"
    # the particle count (after the magic, version and record size): a huge one
    # is refused before any allocation, one more than stored runs out of records
    n = int.from_bytes(data[16:20], "little")
    assert n == 1024
    for name, bad_n in (("n_huge", 2**31 - 1), ("n_plus", n + 1), ("n_one", 1)):
        cases[name] = data[:16] + bad_n.to_bytes(4, "little") + data[20:]
    # header and particle fields outside the range the integrator produces:
    # params at byte 20 (nb_max at 48), time_block at 76, particle 0's record
    # at 188 with its regular level at 188 + 432
    import struct

    assert struct.unpack_from("<i", data, 48)[0] == 320 and struct.unpack_from("<i", data, 76)[0] == -45
    assert struct.unpack_from("<ii", data, 620) == (-7, -9)

    def patch(off, fmt, val):
        b = bytearray(data)
        struct.pack_into(fmt, b, off, val)
        return bytes(b)

    cases["nb_max_zero"] = patch(48, "<i", 0)
    cases["nb_max_huge"] = patch(48, "<i", 2**30)
    cases["time_block_positive"] = patch(76, "<i", 5)
    cases["time_block_low"] = patch(76, "<i", -4000)
    cases["level_huge"] = patch(620, "<i", 10**6)
    cases["level_below_block"] = patch(624, "<i", -46)
    for name, blob in cases.items():
        p = tmp_path / (name + ".ckpt")
        p.write_bytes(blob)
        with pytest.raises(_lib.AbyssError):
            ACIntegrator.load(None, str(p))


def test_end_block_refuses_bad_results_and_stays_open():
    """A negative neighbour count or a neighbour index outside the cluster is
    refused (ABYSS_ERR_ARG) before anything is used; the block stays open, and
    the correct results then commit to the state of an undisturbed run."""
    import oracle

    want = None
    ac = _load(2)
    try:
        assert run_blocks_with_oracle(ac, 1) == 1
        want = _digest(ac)
    finally:
        ac.close()
    ac = _load(2)
    try:
        targets, new_time, scale = ac.begin_block()
        st = ac.block_state()
        px, pv = oracle.predict(st["x"], st["v"], st["a0"], st["a1"], st["t0"], new_time, scale)
        ref = oracle.reg_force(px, pv, st["mass"], st["r2nb"], ac.params.eps2, targets, ac.nb_max)
        args = [ref[k] for k in ("acc_reg", "jerk_reg", "acc_irr", "jerk_irr")]
        bad_nnb = ref["nnb"].copy()
        bad_nnb[len(bad_nnb) // 2] = -3
        with pytest.raises(_lib.AbyssError):
            ac.end_block(*args, bad_nnb, ref["list"])
        r = int(np.argmax(ref["nnb"]))
        for bad in (-1, ac.n, 2**31 - 1):
            lst = ref["list"].copy()
            lst[r, ref["nnb"][r] - 1] = bad
            with pytest.raises(_lib.AbyssError):
                ac.end_block(*args, ref["nnb"], lst)
        assert ac.end_block(*args, ref["nnb"], ref["list"]) in ("ok", "done")
        assert _digest(ac) == want
    finally:
        ac.close()


def test_device_modes_need_a_gpu_context():
    """An integration without a GPU context (a checkpoint loaded for host-side
    calls) refuses the device irregular levels and device blocks, and stays
    usable: switching them off is accepted and the state reads back."""
    from abyss_b200._lib import ABYSS_ERR_STATE, AbyssError

    ac = _load(1)
    try:
        before = _digest(ac)
        for switch in (ac.set_device_irregular, ac.set_device_resident):
            with pytest.raises(AbyssError) as err:
                switch(True)
            assert err.value.code == ABYSS_ERR_STATE
            switch(False)
        info = ac.device_resident_info()
        assert not info["on"] and info["borderline"] == 0
        assert _digest(ac) == before
    finally:
        ac.close()
