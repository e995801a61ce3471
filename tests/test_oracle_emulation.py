"""The oracle's emulation of the mixed step (accuracy studies only).

``oracle.kks_oracle.run(update=...)`` replaces the reference's FP64 update by
the mixed CUDA step's increment form with single-precision transforms
("mixed"), or by the same with the Cahn-Hilliard chain in FP64 ("mixed_ch64").
The default stays the reference's update (pinned by test_oracle_golden.py).
On the reference's small set-up the emulated mixed step's X error is of the
FP32 round-off's order and the FP64 Cahn-Hilliard chain removes most of it.
"""

import tempfile

import numpy as np
import pytest

from conftest import rel_l2, small_config, three_precipitates


def _run(cfg, state, update):
    from oracle import kks_oracle

    with tempfile.TemporaryDirectory() as d:
        return kks_oracle.run(cfg, *[np.array(a) for a in state], cfg.material_tables, out_dir=d, write_logs=False,
                              save_maps=False, update=update)


def test_emulated_mixed_errors():
    cfg = small_config(n_steps=30)
    state = three_precipitates(cfg)
    ref = _run(cfg, state, "fp64")
    mixed = _run(cfg, state, "mixed")
    ch64 = _run(cfg, state, "mixed_ch64")
    e_mixed, x_mixed = rel_l2(mixed.eta, ref.eta), rel_l2(mixed.X, ref.X)
    e_ch64, x_ch64 = rel_l2(ch64.eta, ref.eta), rel_l2(ch64.X, ref.X)
    assert 1e-9 < x_mixed < 1e-6
    assert x_ch64 < x_mixed / 3
    assert e_mixed < 1e-9 and e_ch64 < 1e-9


def test_update_is_checked():
    from oracle import kks_oracle

    cfg = small_config(n_steps=2)
    with pytest.raises(ValueError):
        kks_oracle.run(cfg, *three_precipitates(cfg), cfg.material_tables, write_logs=False, save_maps=False,
                       update="fp16")
