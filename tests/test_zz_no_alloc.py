"""dnslbm_step_f64_noalloc: the FP64 step for callers that cannot allocate.

A host code that hands out all device memory from its own pool cannot let a
library call cudaMalloc; it keeps the populations in its own device buffer and
calls dnslbm_step_f64_noalloc, whose scratch is a static device array.  This
test drives that entry point through the C ABI on caller-owned buffers (made
here with torch) and checks it, over two calls in a row, against the context
entry point (dnslbm_create / dnslbm_load_state / dnslbm_step) on the same
input and against the CPU oracle: FP64 populations bit for bit, log records
within the 1e-11 relative tolerance used for FP64 logs elsewhere.  Odd call
lengths make the second call start from a state left by an odd number of
steps (parity 1).  Collected last so a failure here does not hide the other
tests.
"""
import ctypes
import os
import sys

import numpy as np
import pytest

import dnslbm
import inputs

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import oracle  # noqa: E402

pytestmark = pytest.mark.gpu

LINKS = ((0, 0), (1, 0), (-1, 0), (0, 1), (0, -1))


def wall_bits(flags):
    """Wall-link bits [2][ny][nx] from periodic-grid flags (the rule documented
    in include/dnslbm.h: a link bounces back iff both wall cells are -1)."""
    nx, ny, zd = flags.shape
    out = np.zeros((2, ny, nx), np.uint8)
    for w, k in enumerate((0, zd - 1)):
        s = flags[:, :, k].T  # [y][x]
        for b, (dx, dy) in enumerate(LINKS):
            t = np.roll(np.roll(s, -dx, axis=1), -dy, axis=0)
            out[w] |= (((t == -1) & (s == -1)).astype(np.uint8) << b)
    return out


def to_soa(state):
    return np.ascontiguousarray(state[:, :, 1:-1, :].transpose(3, 2, 1, 0))  # [a][z][y][x]


def from_soa(soa, shape):
    s = np.zeros(shape)
    s[:, :, 1:-1, :] = soa.transpose(3, 2, 1, 0)
    return s


@pytest.mark.parametrize("calls", [(4, 6), (3, 5)])
@pytest.mark.parametrize("textured", [False, True])
def test_noalloc_matches_context_entry_point(textured, calls):
    torch = pytest.importorskip("torch")
    L = dnslbm.lib()
    L.dnslbm_step_f64_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int, ctypes.c_int,
                                          ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_void_p,
                                          ctypes.c_int, ctypes.c_long, ctypes.c_void_p, ctypes.c_void_p,
                                          ctypes.c_char_p, ctypes.c_size_t]
    nx, ny, nz, omega, gx = 40, 24, 12, 1.75, 3e-5
    flags = inputs.flags_longitudinal(nx, ny, nz, 3, 3) if textured else inputs.flags_smooth(nx, ny, nz)
    s0 = inputs.laminar_state(nx, ny, nz, 0.08, 0.1, 21)
    # two calls in a row; an odd first call leaves the second one a state in
    # the swapped (parity 1) layout, and the sum is even, so the final state
    # is in the natural layout

    with dnslbm.Channel(nx, ny, nz, omega, gx=gx, force_mode=dnslbm.CONST_G, precision=64) as ch:
        ch.set_flags(flags)
        ch.load_state(s0)
        for n in calls:
            ch.step(n)
        want_state = ch.store_state()
        want_logs = ch.logs()

    pop = torch.from_numpy(to_soa(s0)).cuda()
    mask = torch.from_numpy(wall_bits(flags)).cuda() if textured else None
    err = ctypes.create_string_buffer(256)
    got_logs = []
    parity = 0
    for n in calls:
        logs = torch.zeros((n, 9), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        rc = L.dnslbm_step_f64_noalloc(pop.data_ptr(), nx * ny * nz, nx, ny, nz, omega, gx,
                                       mask.data_ptr() if textured else None, parity, n, logs.data_ptr(), None,
                                       err, len(err))
        assert rc == 0, err.value.decode()
        torch.cuda.synchronize()
        parity = (parity + n) % 2
        got_logs.append(logs.cpu().numpy())
    got_state = from_soa(pop.cpu().numpy(), s0.shape)
    got_logs = np.concatenate(got_logs)
    np.testing.assert_array_equal(got_state, want_state)
    np.testing.assert_allclose(got_logs, want_logs, rtol=1e-11, atol=1e-15)

    ref = s0.copy()
    ref_logs = oracle.run(ref, flags, omega, gx=gx, const_g=True, nsteps=sum(calls))
    np.testing.assert_array_equal(got_state, ref)
    np.testing.assert_allclose(got_logs, ref_logs, rtol=1e-11, atol=1e-15)


def test_noalloc_rejects_oversized_grid():
    L = dnslbm.lib()
    L.dnslbm_step_f64_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int, ctypes.c_int,
                                          ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_void_p,
                                          ctypes.c_int, ctypes.c_long, ctypes.c_void_p, ctypes.c_void_p,
                                          ctypes.c_char_p, ctypes.c_size_t]
    err = ctypes.create_string_buffer(256)
    # 628 x 4 x 3000 cells (7.5M, a valid grid) need about 54 doubles of
    # scratch per wall-normal plane: more than the 1 MiB array holds.  A dummy
    # aligned address: the size check fails before anything touches it.
    rc = L.dnslbm_step_f64_noalloc(ctypes.c_void_p(256), 628 * 4 * 3000, 628, 4, 3000, 1.5, 0.0, None,
                                   0, 1, None, None, err, len(err))
    assert rc == dnslbm.ERR_ARG and b"scratch" in err.value
