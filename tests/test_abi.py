"""The C-ABI: the ctypes mirror matches include/efsi.h byte for byte, and the
built library exports every entry point the header declares (no GPU needed)."""
import ctypes as C
import os
import re
import subprocess
import tempfile

import pytest

from eulerianfsi_b200 import _abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "efsi.h")

STRUCTS = {
    "efsi_bc_side": _abi.BCSide, "efsi_bc_setup": _abi.BCSetup, "efsi_mesh": _abi.Mesh,
    "efsi_models": _abi.Models, "efsi_numerics": _abi.Numerics, "efsi_config": _abi.Config,
    "efsi_step_report": _abi.StepReportC, "efsi_projection_result": _abi.ProjectionResultC,
    "efsi_stats": _abi.Stats, "efsi_diag_config": _abi.DiagConfig, "efsi_tensor_region": _abi.TensorRegion,
    "efsi_diagnostics": _abi.Diagnostics, "efsi_gradient": _abi.GradientC,
}


def _c_layout():
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"', "int main(void) {"]
    for cname, py in STRUCTS.items():
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            lines.append(f'printf("{cname}.{fname} %zu\\n", offsetof({cname}, {fname}));')
    lines.append("return 0; }")
    with tempfile.TemporaryDirectory() as d:
        src, exe = os.path.join(d, "l.c"), os.path.join(d, "l")
        open(src, "w").write("\n".join(lines))
        subprocess.run(["gcc", "-std=c99", src, "-o", exe], check=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
    res = {}
    for line in out.splitlines():
        k, v = line.rsplit(" ", 1)
        res[k] = int(v)
    return res


def test_struct_layout_matches_header():
    lay = _c_layout()
    for cname, py in STRUCTS.items():
        assert C.sizeof(py) == lay[f"{cname} size"], cname
        for fname, _ in py._fields_:
            assert getattr(py, fname).offset == lay[f"{cname}.{fname}"], (cname, fname)


def declared_entry_points():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"EFSI_API\s+[\w\s\*]*?\b(efsi_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib_path = _abi.LIBRARY_PATH
    if not os.path.exists(lib_path):
        from eulerianfsi_b200 import build
        build.build()
    out = subprocess.run(["nm", "-D", "--defined-only", lib_path], check=True, capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (efsi_\w+)", out))
    declared = declared_entry_points()
    assert len(declared) >= 15
    missing = [d for d in declared if d not in exported]
    assert not missing, missing


def test_library_loads_without_gpu():
    lib = _abi.load_library()
    for name in declared_entry_points():
        assert hasattr(lib, name)


def test_create_without_device_reports_cuda_error():
    """On a machine without a GPU the library loads and efsi_create fails cleanly."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    import eulerianfsi_b200 as ef
    from eulerianfsi_b200 import workloads
    w = workloads.cavity_disk(N=8)
    with pytest.raises(ef.CUDAError):
        ef.build_imex_context(w.metrics, w.bcs, w.models, numerics=w.numerics)
