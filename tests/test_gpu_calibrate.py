"""The gather-rate calibration behind the sweep's gather bound
(net_measure_gather): random 4-byte loads per second from a device array,
from each SM's shared memory and from a cluster's shared memory."""
from __future__ import annotations

import pytest

import knappnet_b200 as K

pytestmark = pytest.mark.gpu


def test_gather_rates_are_measured_for_every_source():
    l2 = K.measure_gather(0, 1 << 24)
    smem = K.measure_gather(1)
    cluster = [K.measure_gather(c) for c in (2, 4, 8)]
    # whole-GPU rates: far above a billion per second, far below the
    # shared-memory bank limit of 148 SMs x 32 banks x 2 GHz
    for r in [l2, smem, *cluster]:
        assert 1e9 < r < 148 * 32 * 2.5e9
    # an SM's own shared memory serves random words faster than L2
    assert smem > l2
    # a larger array is no faster to gather from than one that fits in L2
    assert K.measure_gather(0, 1 << 28) < 1.2 * l2
