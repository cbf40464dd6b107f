"""On-device time averages of the plane statistics (dnslbm_stats_*): the
average of samples taken at several steps and both AA parities equals the
average of the same samples read one by one with dnslbm_statistics (means
averaged, rms pooled as the root of the mean square, the rule of the
reference's TKE-budget/postprocessing/time_stats.c), to 1e-12 relative."""
import numpy as np
import pytest

import dnslbm
import inputs

pytestmark = pytest.mark.gpu

RMS_ROWS = (3, 4, 5, 8)


@pytest.mark.parametrize("prec", [64, 32])
def test_device_average_equals_host_average(prec):
    nx, ny, nz = 40, 18, 14
    with dnslbm.Channel(nx, ny, nz, 1.8, gx=2e-5, precision=prec) as ch:
        ch.set_flags(inputs.flags_longitudinal(nx, ny, nz, 3, 3))
        ch.load_state(inputs.turbulent_state(nx, ny, nz, 0.06, 0.2, 2))
        samples = []
        for n in (0, 3, 4, 7, 1):
            ch.step(n)
            ch.stats_accumulate()
            samples.append(ch.statistics())
        avg, count = ch.stats_average()
        assert count == len(samples)
        sq = np.array(samples)
        want = sq.mean(axis=0)
        want[list(RMS_ROWS)] = np.sqrt((sq[:, list(RMS_ROWS)] ** 2).mean(axis=0))
        np.testing.assert_allclose(avg, want, rtol=1e-12, atol=1e-18)
        ch.stats_reset()
        avg, count = ch.stats_average()
        assert count == 0 and not avg.any()
        ch.stats_accumulate()
        avg, count = ch.stats_average()
        assert count == 1
        np.testing.assert_allclose(avg, ch.statistics(), rtol=1e-12, atol=1e-18)
