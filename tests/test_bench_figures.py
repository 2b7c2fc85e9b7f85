"""The bench reads per-launch ncu figures from the committed profile summaries
only for the rasterizer form it ran: a figure taken on another form names
other kernels (another tile edge, batch depth, launch shape or backward) and
must not stand in for the one timed."""

from __future__ import annotations

import types

import bench


def _opts(**kw):
    base = dict(tile_size=16, batch_depth=256, persistent_raster=True, grouped_backward=False,
                forward_pixels_per_thread=2, backward_pixels_per_thread=2)
    base.update(kw)
    return types.SimpleNamespace(**base)


def test_form_key_names_every_kernel_choice():
    keys = {bench.form_key(_opts(**kw)) for kw in (
        {}, {"tile_size": 32}, {"batch_depth": 128}, {"persistent_raster": False}, {"grouped_backward": True},
        {"forward_pixels_per_thread": 1}, {"backward_pixels_per_thread": 1})}
    assert len(keys) == 7


def test_figures_of_another_form_are_not_used(tmp_path, monkeypatch):
    (tmp_path / "profiles").mkdir()
    form = bench.form_key(_opts())
    other = bench.form_key(_opts(grouped_backward=True))
    (tmp_path / "profiles" / "x.md").write_text(
        f"traffic backward [{other}]: 111\n"
        f"traffic backward: 222\n"
        f"traffic backward [{form}]: 333 bytes\n"
        f"instructions backward [{other}]: 444\n")
    monkeypatch.setattr(bench, "ROOT", tmp_path)
    assert bench.measured_traffic("backward", form) == 333
    assert bench.measured_traffic("backward", other) == 111
    assert bench.profile_figure("instructions", "backward", form) is None
    assert bench.profile_figure("instructions", "backward", other) == 444
