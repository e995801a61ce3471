"""Generate ``reference_cli.npz`` by running the reference's own command line
(``pf_kks.cli.main``, the ``pf-kks-run`` console script) on a small case.

    NUMBA_CACHE_DIR=/tmp/numba python tests/golden/make_cli_fixture.py REF

REF is a checkout of the reference (or set $PF_KKS_REFERENCE); it is read,
never written. The case (``CASE_TOML`` below, with the precipitates of
``CIRCLES`` and the material tables shipped in pf_kks_gpu/data) is a 48 x 40
cell with three sharp precipitates, 12 fixed-dt steps (x_equilibrium = 0 never
arms the adaptive scheme) and three map saves. The fixture keeps everything
the CLI writes:

* ``config_json``: the text of config.json;
* ``hist_<key>``: every array of history.npz (good_step and ttime included);
* ``maps``: the map file names; ``map<i>_<key>``: every array of each map;
* ``log_txt`` / ``dtime_txt``: the two log files.
"""

import os
import shutil
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
TABLES = os.path.join(HERE, "..", "..",
                      "extended-kim-kim-suzuki-kks--phase-field-model-for-prediction-of-materials-properties_b200",
                      "pf_kks_gpu", "data", "final_export.npz")

CASE_TOML = """
[grid]
nx = 48
ny = 40
nz = 1
dx = 0.5e-9

[heat_treatment]
schedule_time = [0, 1350]
schedule_temperature = [400, 850]

[microstructure]
precipitates = "circles.npz"
x_equilibrium = 0.0

[material]
material_tables = "tables.npz"
c_eps0 = 0.25
c_Meta = 0.6

[output]
n_steps = 12
n_map_saves = 3
n_surface_samples = 4
"""

# ox, oy, oz, r [m]
CIRCLES = np.array([[6.0e-9, 7.5e-9, 0.0, 3.0e-9],
                    [15.5e-9, 12.0e-9, 0.0, 2.0e-9],
                    [21.0e-9, 3.0e-9, 0.0, 2.5e-9]])


def write_case(directory):
    """Write the case's TOML, precipitates and tables into ``directory``;
    returns the TOML path."""
    os.makedirs(directory, exist_ok=True)
    np.savez(os.path.join(directory, "circles.npz"), ox_cyl=CIRCLES[:, 0], oy_cyl=CIRCLES[:, 1],
             oz_cyl=CIRCLES[:, 2], r_cyl=CIRCLES[:, 3])
    shutil.copyfile(TABLES, os.path.join(directory, "tables.npz"))
    path = os.path.join(directory, "case.toml")
    with open(path, "w") as f:
        f.write(CASE_TOML)
    return path


def collect(out_dir):
    """Everything the CLI wrote into ``out_dir``, in the fixture's layout."""
    data = {}
    with open(os.path.join(out_dir, "config.json")) as f:
        data["config_json"] = np.array(f.read())
    with np.load(os.path.join(out_dir, "history.npz")) as h:
        for key in h.files:
            data[f"hist_{key}"] = h[key]
    maps = sorted(os.listdir(os.path.join(out_dir, "saved_maps")))
    data["maps"] = np.array(maps)
    for i, name in enumerate(maps):
        with np.load(os.path.join(out_dir, "saved_maps", name)) as m:
            data[f"map{i}_keys"] = np.array(m.files)
            for key in m.files:
                data[f"map{i}_{key}"] = m[key]
    for name in ("log.txt", "dtime.txt"):
        with open(os.path.join(out_dir, name)) as f:
            data[name.replace(".", "_")] = np.array(f.read())
    return data


def main(ref_root):
    sys.path.insert(0, ref_root)
    from pf_kks import cli

    tmp = tempfile.mkdtemp()
    try:
        toml = write_case(os.path.join(tmp, "case"))
        out = os.path.join(tmp, "out")
        assert cli.main([toml, "--out", out, "--quiet", "--fft-threads", "1"]) == 0
        path = os.path.join(HERE, "reference_cli.npz")
        np.savez_compressed(path, **collect(out))
        print("wrote", path)
    finally:
        shutil.rmtree(tmp, ignore_errors=True)


if __name__ == "__main__":
    _ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("PF_KKS_REFERENCE")
    if not _ref:
        sys.exit(f"usage: python {os.path.basename(__file__)} REFERENCE_CHECKOUT (or set PF_KKS_REFERENCE)")
    main(_ref)
