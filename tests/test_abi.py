"""The C-ABI library: it loads, exports every function include/kks.h declares,
its ctypes mirror matches the C layout, and without a usable GPU it fails
loudly instead of computing on the CPU. No compute call is made here."""

import ctypes
import os
import re
import shutil
import subprocess

import pytest

from conftest import REPO

from pf_kks_gpu import _lib as L

HEADER = os.path.join(REPO, "include", "kks.h")


def declared_functions():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^(?:int|const char\*)\s+(kks_\w+)\s*\(", text, flags=re.M)))


def test_library_exports_every_declared_function():
    lib = L.load()
    names = declared_functions()
    assert len(names) >= 13
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert sorted(L.EXPORTS) == names
    assert b"sm_100a" in lib.kks_version()


@pytest.mark.skipif(shutil.which("gcc") is None, reason="gcc not available")
def test_ctypes_layout_matches_c(tmp_path):
    exe = tmp_path / "abi_sizes"
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(REPO, "include"), os.path.join(REPO, "tests", "abi_sizes.c"),
                    "-o", str(exe)], check=True)
    out = dict((ln.split()[0], [int(v) for v in ln.split()[1:]])
               for ln in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.splitlines())
    assert out["kks_params"] == [ctypes.sizeof(L.KksParams), L.KksParams.n_sched.offset, L.KksParams.sched_time.offset,
                                 L.KksParams.table.offset]
    assert out["kks_record"] == [ctypes.sizeof(L.KksRecord), L.KksRecord.T.offset, L.KksRecord.energy_s.offset]
    assert out["kks_step_row"] == [ctypes.sizeof(L.KksStepRow)]
    assert out["kks_run_state"] == [ctypes.sizeof(L.KksRunState), L.KksRunState.t.offset,
                                    L.KksRunState.error_dtime_s.offset]
    assert out["kks_gen_args"] == [ctypes.sizeof(L.KksGenArgs), L.KksGenArgs.w.offset, L.KksGenArgs.rng_state.offset,
                                   L.KksGenArgs.pc_ratio.offset]


def _gpu_present():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_gpu_present(), reason="checks the behaviour without a GPU")
def test_create_fails_loudly_without_gpu():
    from conftest import small_config

    from pf_kks_gpu import solver
    from pf_kks_gpu.materials import MaterialTables

    cfg = small_config()
    t = MaterialTables.from_npz(cfg.material_tables)
    with pytest.raises(L.KksError, match="kks_create"):
        solver.Cell(cfg, t)


def test_invalid_arguments_are_rejected_before_any_device_call():
    lib = L.load()
    h = ctypes.c_void_p()
    assert lib.kks_create(None, 0, 0, 0, None, 0, ctypes.byref(h)) == -1
    p = L.KksParams()
    p.nx, p.ny, p.n_sched, p.n_table = 1, 8, 1, 1
    assert lib.kks_create(ctypes.byref(p), 0, 0, 0, None, 0, ctypes.byref(h)) == -1
    assert b"np.gradient" in lib.kks_last_error()
    p.nx = 8
    assert lib.kks_create(ctypes.byref(p), 7, 0, 0, None, 0, ctypes.byref(h)) == -1
    assert b"precision" in lib.kks_last_error()
