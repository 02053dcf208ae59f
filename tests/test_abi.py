"""The C-ABI library loads on a CPU-only host and exports every declared symbol."""
import ctypes
import os

import pytest

from ibis_b200 import build, lib


def test_library_exports_every_declared_symbol():
    path = build.build()          # no-op when the in-tree library is current
    assert os.path.exists(path)
    so = ctypes.CDLL(path)
    names = lib.declared_symbols()
    assert "ibis_step_f32" in names and "ibis_step_f64" in names
    for name in names:
        assert hasattr(so, name), name
    assert set(names) <= set(lib.SIGNATURES), set(names) - set(lib.SIGNATURES)


def test_loader_sets_prototypes():
    L = lib.load()
    assert L.ibis_step_f32.restype is ctypes.c_int
    assert len(L.ibis_step_f32.argtypes) == 11


def _c_layout(tmp_path, body):
    import subprocess
    src = tmp_path / "probe.c"
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "ibis_b200.h"\nint main(void){' + body + 'return 0;}\n')
    exe = tmp_path / "probe"
    subprocess.run(["gcc", "-std=c99", "-I", os.path.join(lib.REPO, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()
    return [int(x) for x in out]


def test_struct_layouts_match_ctypes(tmp_path):
    from ibis_b200.params import IbisParamsC
    E = lib.IbisEnsembleC
    names = [f[0] for f in E._fields_]
    body = 'printf("%zu %zu ", sizeof(IbisParams), sizeof(IbisEnsemble));'
    body += "".join(f'printf("%zu ", offsetof(IbisEnsemble, {n}));' for n in names)
    got = _c_layout(tmp_path, body)
    assert got[0] == ctypes.sizeof(IbisParamsC)
    assert got[1] == ctypes.sizeof(E)
    assert got[2:] == [getattr(E, n).offset for n in names]


def test_day_params_layout_matches_ctypes(tmp_path):
    from ibis_b200.params import IbisDayParamsC
    names = [f[0] for f in IbisDayParamsC._fields_]
    body = 'printf("%zu ", sizeof(IbisDayParams));'
    body += "".join(f'printf("%zu ", offsetof(IbisDayParams, {n}));' for n in names)
    got = _c_layout(tmp_path, body)
    assert got[0] == ctypes.sizeof(IbisDayParamsC)
    assert got[1:] == [getattr(IbisDayParamsC, n).offset for n in names]


def test_ensemble_daily_layout_matches_ctypes(tmp_path):
    E = lib.IbisEnsembleDailyC
    names = [f[0] for f in E._fields_]
    body = 'printf("%zu ", sizeof(IbisEnsembleDaily));'
    body += "".join(f'printf("%zu ", offsetof(IbisEnsembleDaily, {n}));' for n in names)
    got = _c_layout(tmp_path, body)
    assert got[0] == ctypes.sizeof(E)
    assert got[1:] == [getattr(E, n).offset for n in names]


@pytest.mark.parametrize("struct,cname", [("IbisWetlandBuilderC", "IbisWetlandBuilder"), ("IbisForestC", "IbisForest")])
def test_wetland_layouts_match_ctypes(tmp_path, struct, cname):
    E = getattr(lib, struct)
    names = [f[0] for f in E._fields_]
    body = f'printf("%zu ", sizeof({cname}));'
    body += "".join(f'printf("%zu ", offsetof({cname}, {n}));' for n in names)
    got = _c_layout(tmp_path, body)
    assert got[0] == ctypes.sizeof(E)
    assert got[1:] == [getattr(E, n).offset for n in names]


def test_launch_configuration_table():
    """The configuration table is read from the library without a GPU: the
    default long configuration (6: fused, block 224, accumulators on chip), the
    two-kernel ones, and the staged fused form (11) with the same block."""
    cfgs = lib.configs()
    assert len(cfgs) == lib.load().ibis_num_configs() == 12
    assert cfgs[6]["form"] == "fused" and cfgs[6]["block"] == 224 and not cfgs[6]["staged"]
    assert cfgs[11]["form"] == "fused" and cfgs[11]["staged"]
    assert (cfgs[11]["block"], cfgs[11]["min_blocks"]) == (cfgs[6]["block"], cfgs[6]["min_blocks"])
    assert [c["id"] for c in cfgs if c["form"] == "split"] == [8, 9, 10]
    form = ctypes.c_int()
    assert lib.load().ibis_config_info(11, ctypes.byref(form), None, None, None, None) == 0 and form.value == 2
    assert lib.load().ibis_config_info(12, None, None, None, None, None) < 0
