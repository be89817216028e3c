"""The C-ABI library loads, exports every entry point include/emerge_cuda.h declares, and its
struct layouts match the ctypes mirrors (checked against a C compilation of the header)."""
import ctypes
import os
import re
import subprocess
import tempfile

import pytest

from emerge_engine_b200 import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "emerge_cuda.h")
ORACLE_HEADER = os.path.join(ROOT, "oracle", "emerge_oracle.h")


def declared_functions(path):
    src = open(path).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(emerge_cuda_\w+)\s*\(", src)))


def test_library_exports_every_declared_symbol(cuda_lib):
    names = declared_functions(HEADER)
    assert len(names) >= 25
    lib = ctypes.CDLL(abi.LIB_PATH)
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # and the ctypes table covers them all
    table = {n for n, _, _ in abi.ABI_FUNCTIONS}
    assert set(names) <= table, sorted(set(names) - table)


C_STRUCTS = {
    "emerge_particle": abi.Particle,
    "emerge_sim_config": abi.SimConfigC,
    "emerge_material_params": abi.MaterialParamsC,
    "emerge_spawn_region": abi.SpawnRegionC,
    "emerge_body_state": abi.BodyStateC,
    "emerge_step_timing": abi.StepTimingC,
    "emerge_stats": abi.StatsC,
    "emerge_closure_stats": abi.ClosureStatsC,
    "emerge_closure_train_config": abi.ClosureTrainConfigC,
    "emerge_closure_train_report": abi.ClosureTrainReportC,
    "emerge_batch_tune_report": abi.BatchTuneReportC,
}


def c_layout(header, structs):
    """sizeof and offsetof of every field, from gcc."""
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{header}"', "int main(void) {"]
    for cname, cls in structs.items():
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, _ in cls._fields_:
            cf = "lambda" if fname == "lambda_" else fname
            lines.append(f'printf("{cname}.{fname} %zu\\n", offsetof({cname}, {cf}));')
    lines.append("return 0; }")
    with tempfile.TemporaryDirectory() as d:
        src, exe = os.path.join(d, "l.c"), os.path.join(d, "l")
        open(src, "w").write("\n".join(lines))
        subprocess.run(["gcc", "-o", exe, src], check=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
    res = {}
    for line in out.splitlines():
        k, v = line.rsplit(" ", 1) if " size " not in line else (line.split(" size ")[0] + "#size", line.split(" size ")[1])
        res[k] = int(v)
    return res


def test_struct_layouts_match_header():
    lay = c_layout(HEADER, C_STRUCTS)
    for cname, cls in C_STRUCTS.items():
        assert lay[cname + "#size"] == ctypes.sizeof(cls), cname
        for fname, _ in cls._fields_:
            assert lay[f"{cname}.{fname}"] == getattr(cls, fname).offset, (cname, fname)
    assert lay["emerge_particle#size"] == 128        # particle.rs:144
    assert lay["emerge_material_params#size"] == 96  # params.rs:214


def test_oracle_structs_share_the_layout():
    names = {"oracle_particle": abi.Particle, "oracle_config": abi.SimConfigC,
             "oracle_spawn": abi.SpawnRegionC, "oracle_body_state": abi.BodyStateC}
    lay = c_layout(ORACLE_HEADER, names)
    for cname, cls in names.items():
        assert lay[cname + "#size"] == ctypes.sizeof(cls), cname
        for fname, _ in cls._fields_:
            assert lay[f"{cname}.{fname}"] == getattr(cls, fname).offset, (cname, fname)


def test_create_without_gpu_fails_loudly(cuda_lib):
    """No CPU fallback: without a usable CUDA device, create returns an error code."""
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if has_gpu:
        pytest.skip("a GPU is present")
    from emerge_engine_b200 import SimConfig, Simulation
    with pytest.raises(abi.EmergeError) as ei:
        Simulation(SimConfig.standard(64, 0.05, (0.0, -1.0)))
    assert ei.value.status == abi.ERR_CUDA


def test_invalid_config_is_rejected_before_any_device_work(cuda_lib):
    cfg = abi.SimConfigC()  # all zero: grid_res < 4
    out = ctypes.c_void_p()
    st = cuda_lib.emerge_cuda_create(ctypes.byref(cfg), 0, ctypes.byref(out))
    assert st == abi.ERR_INVALID_ARG
    assert b"grid_res" in cuda_lib.emerge_cuda_last_global_error()
