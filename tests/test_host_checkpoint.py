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
