"""The C-ABI library: it loads, exports every entry point that
include/mdacp_b200.h declares, and its structs match the ctypes mirrors.
No compute calls (these run without a GPU)."""
from __future__ import annotations

import ctypes
import pathlib
import re
import subprocess

import pytest

import mdacp_b200 as M

ROOT = pathlib.Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "mdacp_b200.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(mdg_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = M.load_library()
    names = declared_functions()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_bindings_cover_header():
    assert set(declared_functions()) == set(M.SIGNATURES)


def _c_layout(struct, fields, tmp_path):
    src = tmp_path / "layout.c"
    body = "".join(f'  printf("{f} %zu\\n", offsetof({struct}, {f}));\n' for f in fields)
    src.write_text(
        f'#include <stdio.h>\n#include <stddef.h>\n#include "mdacp_b200.h"\nint main(void){{\n'
        f'  printf("size %zu\\n", sizeof({struct}));\n{body}  return 0;\n}}\n')
    exe = tmp_path / "layout"
    subprocess.check_call(["gcc", "-I", str(ROOT / "include"), str(src), "-o", str(exe)])
    out = subprocess.check_output([str(exe)], text=True)
    return dict((k, int(v)) for k, v in (line.split() for line in out.splitlines()))


@pytest.mark.parametrize("struct,cls", [("mdg_params", M.Params), ("mdg_info", M.Info)])
def test_struct_layout_matches_c(struct, cls, tmp_path):
    fields = [f for f, _ in cls._fields_]
    lay = _c_layout(struct, fields, tmp_path)
    assert lay["size"] == ctypes.sizeof(cls)
    for f in fields:
        assert lay[f] == getattr(cls, f).offset, f


def test_default_params_are_reference_defaults():
    lib = M.load_library()
    p = M.Params()
    lib.mdg_default_params(ctypes.byref(p))
    # SimulationInfo ctor defaults, src/simulationinfo.cc:5-51; CUTOFF_LENGTH 3.0
    assert p.cutoff == 3.0 and p.buffer_length == 0.3 and p.time_step == 0.001
    assert p.heatbath_tau == 0.1 and p.heatbath_gamma == 0.1 and p.aimed_temperature == 1.0
    assert p.check_list_length == 500


def test_status_strings():
    lib = M.load_library()
    for code in M.STATUS_NAMES:
        assert lib.mdg_status_string(code)
    assert b"sm_100a" in lib.mdg_version()


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="checks the no-device path")
def test_create_without_device_fails_cleanly():
    with pytest.raises(M.MdgError) as e:
        M.System([12.0, 12.0, 12.0], cutoff=2.5, capacity=10)
    assert e.value.status == -10
