"""BD-rate / BD-PSNR (mars_b200.rd) against the properties the reference's own tests hold
(crates/mars-bench/src/bdrate.rs:205-337, pchip.rs tests): self-comparison is zero, a rate
scaling by k gives (k - 1) * 100 % exactly, a PSNR shift by delta gives delta exactly, the
interval is the PSNR overlap, and short, disjoint or non-monotonic curves are refused."""
import pytest

from mars_b200 import rd

BPPS = [0.125, 0.25, 0.5, 1.0, 2.0]
PSNRS = [26.1, 29.4, 32.8, 36.0, 39.7]


def sample():
    return list(zip(BPPS, PSNRS))


def test_self_is_zero():
    r = rd.bd_metrics(sample(), sample())
    assert abs(r.bd_rate_pct) < 1e-6 and abs(r.bd_psnr_db) < 1e-12


@pytest.mark.parametrize("k", [0.5, 0.8, 1.0, 1.25, 2.0])
def test_scaled_rate_is_analytic(k):
    r = rd.bd_metrics(sample(), [(b * k, p) for b, p in sample()])
    assert abs(r.bd_rate_pct - (k - 1.0) * 100.0) < 1e-6


@pytest.mark.parametrize("delta", [-1.5, 0.0, 0.75])
def test_shifted_psnr_is_analytic(delta):
    r = rd.bd_metrics(sample(), [(b, p + delta) for b, p in sample()])
    assert abs(r.bd_psnr_db - delta) < 1e-12


def test_interval_is_the_psnr_overlap():
    a = list(zip([0.1, 0.2, 0.4, 0.8], [25.0, 28.0, 31.0, 34.0]))
    b = list(zip([0.2, 0.4, 0.8, 1.6], [27.0, 30.0, 33.0, 36.0]))
    r = rd.bd_metrics(a, b)
    assert r.psnr_interval_db == (27.0, 34.0)
    assert 0.0 < r.bpp_interval[0] < r.bpp_interval[1]


def test_refusals():
    with pytest.raises(rd.BdError, match="at least 4"):
        rd.bd_metrics(list(zip([0.1, 0.2, 0.4], [25.0, 28.0, 31.0])), sample())
    with pytest.raises(rd.BdError, match="no overlapping PSNR"):
        rd.bd_metrics(list(zip([0.1, 0.2, 0.3, 0.4], [20.0, 21.0, 22.0, 23.0])),
                      list(zip([4.0, 5.0, 6.0, 7.0], [40.0, 41.0, 42.0, 43.0])))
    with pytest.raises(rd.BdError, match="monotonically"):
        rd.bd_metrics(list(zip([0.1, 0.2, 0.4, 0.8], [25.0, 28.0, 27.0, 34.0])), sample())


def test_pchip_knots_lines_and_shape():
    p = rd.Pchip([0.0, 1.0, 2.5, 4.0], [1.0, 3.0, 2.0, 5.0])
    for x, y in zip([0.0, 1.0, 2.5, 4.0], [1.0, 3.0, 2.0, 5.0]):
        assert abs(p.eval(x) - y) < 1e-12
    line = rd.Pchip([0.0, 1.0, 2.0, 3.0], [0.0, 2.0, 4.0, 6.0])
    assert abs(line.integrate(0.0, 3.0) - 9.0) < 1e-12
    assert abs(line.integrate(0.5, 1.5) - 2.0) < 1e-12
    step = rd.Pchip([0.0, 1.0, 2.0, 3.0, 4.0], [0.0, 0.0, 0.0, 1.0, 1.0])
    assert all(-1e-12 <= step.eval(i / 100.0) <= 1.0 + 1e-12 for i in range(401))
    with pytest.raises(rd.BdError, match="strictly increasing"):
        rd.Pchip([0.0, 2.0, 1.0], [0.0, 1.0, 2.0])
    assert rd.bpp(1000, 100, 80) == 1.0
