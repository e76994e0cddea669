"""The C-ABI library loads without a GPU and exports every entry point the header declares;
the ctypes mirror matches the C structure layouts (checked with the system C compiler)."""
import ctypes as C
import os
import re
import subprocess
import tempfile

import pytest

from jd_lepic_b200 import _capi, build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "lepic_gpu.h")


def header_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(lepic_(?:gpu|cnn)_\w+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    build.build()
    return C.CDLL(build.LIB)


def test_header_symbols_exported(lib):
    names = header_functions()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), n


def test_ctypes_prototypes_cover_header():
    assert sorted(_capi.PROTOTYPES) == header_functions()


def test_abi_version_without_gpu(lib):
    lib.lepic_gpu_abi_version.restype = C.c_int32
    assert lib.lepic_gpu_abi_version() == 4


def test_struct_layouts_match_c():
    structs = {"lepic_config": _capi.LepicConfig, "lepic_xs_tables": _capi.LepicXsTables,
               "lepic_solve_stats": _capi.LepicSolveStats, "lepic_push_stats": _capi.LepicPushStats,
               "lepic_mcc_stats": _capi.LepicMccStats, "lepic_load_spec": _capi.LepicLoadSpec,
               "lepic_cnn_config": _capi.LepicCnnConfig, "lepic_cnn_stats": _capi.LepicCnnStats,
               "lepic_source_config": _capi.LepicSourceConfig, "lepic_source_tally": _capi.LepicSourceTally,
               "lepic_tallies": _capi.LepicTallies, "lepic_options": _capi.LepicOptions,
               "lepic_zloss_config": _capi.LepicZlossConfig,
               "lepic_secondary_config": _capi.LepicSecondaryConfig}
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"', "int main(void){"]
    for cname, py in structs.items():
        lines.append(f'printf("{cname} %zu\\n", sizeof({cname}));')
        for f, _t in py._fields_:
            lines.append(f'printf("{cname}.{f} %zu\\n", offsetof({cname}, {f}));')
    lines.append("return 0;}")
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "p.c")
        exe = os.path.join(d, "p")
        open(src, "w").write("\n".join(lines))
        subprocess.run(["gcc", src, "-o", exe], check=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
    got = dict(l.rsplit(" ", 1) for l in out.strip().splitlines())
    for cname, py in structs.items():
        assert int(got[cname]) == C.sizeof(py), cname
        for f, _t in py._fields_:
            assert int(got[f"{cname}.{f}"]) == getattr(py, f).offset, f"{cname}.{f}"


def test_create_without_gpu_fails_cleanly(lib):
    """Without a device the library returns an error code instead of aborting."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    L = _capi.load_library()
    cfg = _capi.LepicConfig()
    ctx = C.c_void_p()
    rc = L.lepic_gpu_create(C.byref(cfg), None, None, None, None, C.byref(ctx))
    assert rc == _capi.EINVAL
