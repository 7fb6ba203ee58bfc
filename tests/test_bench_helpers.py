"""Host-side helpers of the bench line, on the CPU: the SM-bound arithmetic of the
Gray-Scott forward (over the lattice and over the rows the multi-cluster kernel
computes, ghost rows included), the roofline note naming the kernel's layout, and the
peak lookup with its fallback."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


@pytest.fixture(scope="module")
def bench():
    import bench as b
    return b


def _mc_kernel(n=256, clusters=4, ghost=8):
    return {"variant": 41, "name": f"k_gs_forward_mc<{n},{clusters},{ghost},5>", "clusters": clusters,
            "ghost_rows": ghost, "sms": 16 * clusters, "rows_per_step": n + 2 * ghost * clusters}


def test_sm_bound_of_the_multicluster_forward(bench):
    """18 FP32 operations per cell-step over 64 SMs x 128 lanes at 1965 MHz: 0.0733 us
    per step for the 256 x 256 lattice, 0.0916 us over the 320 rows computed."""
    k = _mc_kernel()
    steps = 10_000
    per_step = 0.585e-6
    sb = bench.sm_bound(per_step * steps, steps, 256, 1965.0, k)
    bound = 256 * 256 * 18 / (64 * 128 * 1965e6)
    assert sb["sms_used"] == 64 and sb["rows_computed_per_step"] == 320
    assert sb["bound_us_per_step"] == pytest.approx(bound * 1e6)
    assert sb["achieved_us_per_step"] == pytest.approx(0.585)
    assert sb["frac"] == pytest.approx(bound / per_step)
    assert sb["frac_with_ghost_rows"] == pytest.approx(bound * 320 / 256 / per_step)


def test_sm_bound_of_the_single_cluster_forward(bench):
    k = {"variant": 18, "name": "k_gs_forward_rr<256,8>", "clusters": 1, "ghost_rows": 0, "sms": 16,
         "rows_per_step": 256}
    sb = bench.sm_bound(7.4e-3, 10_000, 256, None, k)      # no clock sample: 1965 MHz
    assert sb["sm_clock_hz"] == pytest.approx(1965e6)
    assert sb["frac"] == pytest.approx(sb["frac_with_ghost_rows"])
    assert sb["bound_us_per_step"] == pytest.approx(256 * 256 * 18 / (16 * 128 * 1965e6) * 1e6)


def test_kernel_note_names_the_layout(bench):
    note = bench.kernel_note(_mc_kernel())
    assert "4 16-CTA clusters" in note and "64 of 148 SMs" in note and "8 ghost rows" in note
    single = bench.kernel_note({"clusters": 1, "ghost_rows": 0})
    assert "one 16-CTA cluster" in single and "ghost" not in single


def test_peaks_fall_back_without_the_measured_file(bench, tmp_path, monkeypatch):
    monkeypatch.setattr(bench, "ROOT", str(tmp_path))
    assert bench.load_peaks() == (6650.0, "fallback")
    (tmp_path / "MEASURED_PEAKS.json").write_text('{"hbm_gbs": 6457.7, "bf16_tflops": 1590}')
    assert bench.load_peaks() == (6457.7, "measured")
