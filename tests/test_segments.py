"""FP64 rows split into x-segments.

A 1256-wide FP64 row (the 1256 x 408 x 628 riblet channel) is 10 KB per
direction, 191 KB per stage of 19 directions: two whole-row stages do not fit
shared memory, so the bulk-copy kernel moves 16-byte-aligned x-segments of a
row, and the segment's edge cells move their e_x-shifted populations of an odd
step through global memory.  The populations must stay bit-identical to the
oracle (constant force) on long rows, on segments forced onto short rows
(including an odd row length, whose last segment ends in the row padding),
with smooth and textured walls, after either AA parity.
"""
import os

import numpy as np
import pytest

import dnslbm
import inputs

pytestmark = pytest.mark.gpu


def _run(nx, ny, nz, tex, steps, seg=None, const_g=True):
    old = os.environ.get("DNSLBM_SEGMENT")
    if seg is not None:
        os.environ["DNSLBM_SEGMENT"] = str(seg)
    try:
        fl = inputs.flags_longitudinal(nx, ny, nz, 3, 3) if tex == "ridges" else inputs.flags_smooth(nx, ny, nz)
        s0 = inputs.laminar_state(nx, ny, nz, 0.08, 0.1, 80 + nx)
        mode = dnslbm.CONST_G if const_g else dnslbm.CONST_Q
        with dnslbm.Channel(nx, ny, nz, 1.8, ubulk=0.06, gx=2e-5, force_mode=mode) as ch:
            ch.set_flags(fl)
            ch.load_state(s0)
            kernel = ch.kernel
            ch.step(steps)
            return kernel, s0, fl, ch.store_state(), ch.logs()
    finally:
        if old is None:
            os.environ.pop("DNSLBM_SEGMENT", None)
        else:
            os.environ["DNSLBM_SEGMENT"] = old


@pytest.mark.parametrize("steps", [7, 8])
@pytest.mark.parametrize("tex", ["smooth", "ridges"])
def test_long_fp64_rows_are_segmented_and_exact(oracle_mod, tex, steps):
    kernel, s0, fl, got, logs = _run(1256, 18, 14, tex, steps)
    assert "x-segments" in kernel, kernel
    ref_logs = oracle_mod.run(s0, fl, 1.8, gx=2e-5, const_g=True, nsteps=steps)
    np.testing.assert_array_equal(got, s0)
    np.testing.assert_allclose(logs[:, 1:], ref_logs[:, 1:], rtol=1e-10, atol=1e-15)


@pytest.mark.parametrize("nx,seg", [(100, 34), (101, 34), (64, 16)])
@pytest.mark.parametrize("tex", ["smooth", "ridges"])
def test_forced_segments_are_exact(oracle_mod, nx, seg, tex):
    kernel, s0, fl, got, logs = _run(nx, 12, 9, tex, 9, seg=seg)
    assert "x-segments" in kernel, kernel
    ref_logs = oracle_mod.run(s0, fl, 1.8, gx=2e-5, const_g=True, nsteps=9)
    np.testing.assert_array_equal(got, s0)
    np.testing.assert_allclose(logs[:, 1:], ref_logs[:, 1:], rtol=1e-10, atol=1e-15)


def test_segments_constant_q(oracle_mod):
    kernel, s0, fl, got, logs = _run(100, 12, 9, "ridges", 9, seg=34, const_g=False)
    assert "x-segments" in kernel
    ref_logs = oracle_mod.run(s0, fl, 1.8, ubulk=0.06, const_g=False, nsteps=9)
    np.testing.assert_allclose(got, s0, rtol=1e-11, atol=1e-15)
    np.testing.assert_allclose(logs[:, 1:], ref_logs[:, 1:], rtol=1e-10, atol=1e-15)
