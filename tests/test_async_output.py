"""Output without stopping the time loop (dnslbm_output_begin / _wait).

The outputs of an output step -- the lbf state, vel/den, the turb-fld rows --
are computed on the GPU and copied to page-locked host buffers while the next
steps run.  They must equal the synchronous calls' outputs bit for bit, and
an output step must cost the time loop less than one synchronous store of
the same outputs.  The host driver's two modes (ASYNC 1 / 0) must write the
same files byte for byte.
"""
import os
import subprocess
import time

import numpy as np
import pytest

import dnslbm
import inputs

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
RUN_DNS = os.path.join(ROOT, "dns-solvers_b200", "run-dns")


@pytest.mark.parametrize("prec", [64, 16])
def test_async_outputs_equal_the_synchronous_ones(prec):
    nx, ny, nz = 40, 24, 12
    fl = inputs.flags_longitudinal(nx, ny, nz, 3, 3)
    s0 = inputs.laminar_state(nx, ny, nz, 0.08, 0.1, 41)
    with dnslbm.Channel(nx, ny, nz, 1.8, ubulk=0.06, force_mode=dnslbm.CONST_Q, precision=prec) as ch:
        ch.set_flags(fl)
        ch.load_state(s0)
        for steps in (3, 4):  # either AA parity at the output step
            ch.step(steps)
            want = (ch.store_state(), *ch.moments(), ch.statistics())
            bufs = [dnslbm.PinnedArray(w.shape) for w in want]
            ch.output_begin(*(b.array for b in bufs))
            ch.step(5)  # runs while the copies drain; the snapshot is of the state before it
            ch.output_wait()
            for b, w, name in zip(bufs, want, ("state", "vel", "den", "stats")):
                np.testing.assert_array_equal(b.array, w, err_msg=name)
                b.free()


def test_output_step_costs_less_than_a_synchronous_store():
    """About 1.6 M cells at FP64: the steps after dnslbm_output_begin slow
    down by less than the synchronous store + moments + statistics take."""
    wl = inputs.workload("channel180_h20")
    nx, ny, nz = wl.nx * 2, wl.ny * 2, wl.nz
    s0 = inputs.laminar_state(nx, ny, nz, 0.05, 0.05, 3)
    with dnslbm.Channel(nx, ny, nz, wl.omega, gx=wl.gx, force_mode=dnslbm.CONST_G) as ch:
        ch.load_state(s0)
        out = [dnslbm.PinnedArray(sh) for sh in (ch.state_shape, ch.state_shape[:3] + (3,), ch.state_shape[:3],
                                                 (9, nz + 2))]
        ch.step(20)

        def sync_store():
            t0 = time.perf_counter()
            ch.store_state(out[0].array)
            ch.moments(out[1].array, out[2].array)
            out[3].array[...] = ch.statistics()
            return time.perf_counter() - t0

        def steps_with_output(n, output):
            ch.sync()
            t0 = time.perf_counter()
            if output:
                ch.output_begin(*(o.array for o in out))
            ch.step(n)
            if output:
                ch.output_wait()
            return time.perf_counter() - t0

        sync_store()
        t_sync = min(sync_store() for _ in range(3))
        n = 200
        steps_with_output(n, True)
        t_plain = min(steps_with_output(n, False) for _ in range(3))
        t_out = min(steps_with_output(n, True) for _ in range(3))
        for o in out:
            o.free()
    extra = t_out - t_plain
    assert extra < t_sync, (extra, t_sync, t_plain)


def _run_driver(d, async_mode):
    with open(os.path.join(d, "deck.txt"), "w") as f:
        f.write("xdv 16\nydv 8\nzdv 4\nRebs 100\nub 0.1\nCFL 0.1\nTSTR 0\nTEND 5\nITER 45\nTEXTURE riblets\n"
                f"RIBH 2\nRIBS 4\nASYNC {async_mode}\n")
    subprocess.run([RUN_DNS, "-s", "deck.txt"], cwd=d, check=True, timeout=120, capture_output=True)


def test_driver_async_and_synchronous_outputs_are_identical(tmp_path):
    a, s = tmp_path / "async", tmp_path / "sync"
    a.mkdir()
    s.mkdir()
    _run_driver(str(a), 1)
    _run_driver(str(s), 0)
    names = sorted(n for n in os.listdir(a) if n not in ("report.code", "deck.txt"))
    assert names == sorted(n for n in os.listdir(s) if n not in ("report.code", "deck.txt"))
    assert {"lbf.0000", "vel.0002", "den.0002", "turb-fld.000.002", "uavg-temp.dat"} <= set(names)
    for n in names:
        assert (a / n).read_bytes() == (s / n).read_bytes(), n
