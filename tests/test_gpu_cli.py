"""``pf-kks-run`` on the GPU against the reference's own command line.

The fixture ``golden/reference_cli.npz`` holds everything ``pf_kks.cli.main``
wrote for a small case (``golden/make_cli_fixture.py``: 48 x 40 cell, three
sharp precipitates read from a file, 12 fixed-dt steps, three map saves).
Here ``python -m pf_kks_gpu.cli`` runs the same TOML in a child process and
its outputs are compared file by file: config.json byte for byte, every
array of history.npz, the map names, keys (in order) and contents, and the
two logs byte for byte. Fields are held to the FP64 step's bar (1e-10
relative L2), histories to rtol 1e-9.
"""

import importlib.util
import json
import os
import subprocess
import sys

import numpy as np
import pytest

from conftest import GOLDEN, PKG, rel_l2

FIELDS = ("X", "X_al", "X_th", "eta")


def _fixture_module():
    spec = importlib.util.spec_from_file_location("make_cli_fixture", os.path.join(GOLDEN, "make_cli_fixture.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _cli(args, cwd):
    env = dict(os.environ)
    env["PYTHONPATH"] = PKG + os.pathsep + env.get("PYTHONPATH", "")
    return subprocess.run([sys.executable, "-m", "pf_kks_gpu.cli", *args], cwd=cwd, env=env, capture_output=True,
                          text=True, timeout=600)


def test_print_config_matches_reference(tmp_path):
    """--print-config needs no GPU: the resolved configuration as the
    reference prints it (the same JSON the reference's config.json holds)."""
    g = np.load(os.path.join(GOLDEN, "reference_cli.npz"))
    toml = _fixture_module().write_case(str(tmp_path / "case"))
    out = _cli([toml, "--print-config", "--fft-threads", "1"], cwd=str(tmp_path))
    assert out.returncode == 0, out.stderr
    assert json.loads(out.stdout) == json.loads(str(g["config_json"]))


def test_console_script_is_declared():
    import tomllib

    with open(os.path.join(PKG, "pyproject.toml"), "rb") as f:
        project = tomllib.load(f)["project"]
    assert project["scripts"]["pf-kks-run"] == "pf_kks_gpu.cli:entry"
    from pf_kks_gpu import cli

    assert callable(cli.entry)


@pytest.mark.gpu
def test_cli_outputs_match_reference_cli(tmp_path):
    g = np.load(os.path.join(GOLDEN, "reference_cli.npz"))
    toml = _fixture_module().write_case(str(tmp_path / "case"))
    out_dir = tmp_path / "out"
    run = _cli([toml, "--out", str(out_dir), "--quiet", "--fft-threads", "1"], cwd=str(tmp_path))
    assert run.returncode == 0, run.stderr

    assert (out_dir / "config.json").read_text() == str(g["config_json"])
    assert (out_dir / "log.txt").read_text() == str(g["log_txt"])
    assert (out_dir / "dtime.txt").read_text() == str(g["dtime_txt"])

    with np.load(out_dir / "history.npz") as h:
        ref_keys = sorted(k[5:] for k in g.files if k.startswith("hist_"))
        assert sorted(h.files) == ref_keys
        assert int(h["good_step"]) == int(g["hist_good_step"])
        for key in ref_keys:
            a, b = h[key], g[f"hist_{key}"]
            assert a.shape == b.shape, key
            np.testing.assert_allclose(a.astype(np.float64), b.astype(np.float64), rtol=1e-9, atol=1e-13,
                                       equal_nan=True, err_msg=key)

    maps = sorted(os.listdir(out_dir / "saved_maps"))
    assert maps == list(g["maps"])
    for i, name in enumerate(maps):
        with np.load(out_dir / "saved_maps" / name) as m:
            assert list(m.files) == list(g[f"map{i}_keys"])
            for key in m.files:
                a, b = m[key], g[f"map{i}_{key}"]
                assert a.dtype == b.dtype and a.shape == b.shape, key
                if key in FIELDS:
                    assert rel_l2(a, b) <= 1e-10, (name, key)
                else:
                    np.testing.assert_allclose(a, b, rtol=1e-9, atol=1e-13, err_msg=f"{name}:{key}")
