"""Texture-filtering rate of the device against how far apart the lanes of a warp sample
(hpm_measure_tex_rate): the roof of the half-sweep's NCC sampling, whose lanes hold the planes of
neighbouring pixels and so sample apart.  The rate must fall as the lanes move apart, and the
table is printed for the kernel notes."""
import pytest

import hpm_b200

pytestmark = pytest.mark.gpu


def test_texture_rate_falls_as_lanes_sample_apart():
    rates = {j: hpm_b200.measure_tex_rate(0, hpm_b200.TEX_F32, j) for j in (0.0, 2.0, 4.0, 8.0, 16.0)}
    print("\n| lane offsets up to (px) | Gfetch/s |\n|---|---|")
    for j, r in rates.items():
        print(f"| {j:g} | {r:.0f} |")
    assert rates[0.0] == pytest.approx(hpm_b200.measure_tex_peak(0, hpm_b200.TEX_F32), rel=0.1)
    assert rates[16.0] < 0.8 * rates[0.0]
    assert all(rates[b] <= 1.05 * rates[a] for a, b in ((0.0, 2.0), (2.0, 4.0), (4.0, 8.0), (8.0, 16.0)))
    with pytest.raises(hpm_b200.HPMError):
        hpm_b200.measure_tex_rate(0, hpm_b200.TEX_F32, -1.0)
