"""GPU: the L2 read-bandwidth probe (ptiB200ProbeL2ReadBandwidth) that the
bench's gather roofline divides by: it runs, reports a rate far above the
HBM copy rate (the buffer stays in L2), and repeats within a factor of two."""
import pytest

from hiparti_b200 import ffi

pytestmark = pytest.mark.gpu


def test_l2_probe_reports_a_cache_rate(lib, cuda):
    gb = ffi.new("double *")
    rates = []
    for _ in range(3):
        assert lib.ptiB200ProbeL2ReadBandwidth(64 << 20, 20, gb) == 0
        rates.append(gb[0])
    assert min(rates) > 8000.0           # GB/s: an L2-resident stream on B200 (HBM copies reach about 6500)
    assert max(rates) < 2.0 * min(rates)
