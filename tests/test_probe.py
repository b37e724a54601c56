"""The gather-bandwidth probe the search kernel's roofline divides by
(sg_probe_gather): random 16 B and 32 B loads over an L2-sized working set
and over one several times larger than L2."""
import pytest

import smina_b200 as sb

pytestmark = pytest.mark.gpu


def test_gather_probe_rates_are_plausible():
    e = sb.Engine(0, sb.PREC_FP32)
    try:
        l2_16 = e.probe_gather(64 << 20, 16)
        l2_32 = e.probe_gather(64 << 20, 32)
        hbm_32 = e.probe_gather(2 << 30, 32)
    finally:
        e.close()
    for g in (l2_16, l2_32, hbm_32):
        assert 100 < g < 100_000, g
    # from L2, a 32 B gather moves at least as many bytes per second as from HBM
    assert l2_32 > 0.8 * hbm_32
    e = sb.Engine(0, sb.PREC_FP32)
    try:
        with pytest.raises(sb.SminaError):
            e.probe_gather(64 << 20, 24)
    finally:
        e.close()
