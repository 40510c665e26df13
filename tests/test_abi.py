"""The C ABI library loads without a GPU and exports every entry point
include/lapstack_b200.h declares; compute entry points fail loudly (no CPU
fallback) when no CUDA device is present. CPU only."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import lapstack_b200 as L
from lapstack_b200 import _lib

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "lapstack_b200.h")


def declared():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(lsb_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_the_boundary():
    names = declared()
    for must in ["lsb_abi", "lsb_engine_create", "lsb_stack_begin", "lsb_stack_push_u16", "lsb_stack_push_f32",
                 "lsb_stack_shares", "lsb_stack_finish", "lsb_result_free", "lsb_free_str", "lsb_engine_destroy",
                 "lsb_depth_from_slices", "lsb_wls_solve", "lsb_align_pair", "lsb_warp_cost"]:
        assert must in names


def test_library_exports_every_declared_symbol():
    lib = L.load()
    for name in declared():
        assert hasattr(lib, name), name
    assert set(declared()) == set(_lib.SIGNATURES), "the ctypes table covers the header exactly"
    assert lib.lsb_abi() == _lib.ABI_VERSION


def test_header_is_plain_c_and_links(tmp_path):
    """A C99 caller (cgo, bindgen, a C host) includes the header and links the library as is."""
    import shutil
    import subprocess
    if shutil.which("gcc") is None:
        pytest.skip("no gcc")
    src = tmp_path / "abi.c"
    src.write_text('#include "lapstack_b200.h"\n#include <stdio.h>\n'
                   'int main(void) { printf("%u\\n", (unsigned)lsb_abi()); return 0; }\n')
    exe = tmp_path / "abi"
    libdir = os.path.dirname(_lib.LIB_PATH)
    cc = subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-pedantic", "-Werror", "-I", os.path.dirname(HEADER),
                         str(src), "-L", libdir, "-llapstack_b200", f"-Wl,-rpath,{libdir}", "-o", str(exe)],
                        capture_output=True, text=True)
    assert cc.returncode == 0, cc.stderr
    run = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    assert run.returncode == 0, run.stderr
    assert int(run.stdout) == _lib.ABI_VERSION


def header_arity():
    src = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    out = {}
    for name, args in re.findall(r"\b(lsb_[a-z0-9_]+)\s*\(([^()]*)\)\s*;", src):
        args = args.strip()
        out[name] = 0 if args in ("", "void") else args.count(",") + 1
    return out


def test_rust_binding_in_the_guide_matches_the_header():
    """Every `pub fn` of the Rust extern block in INTEGRATION.md is declared in the header with as many arguments."""
    guide = open(os.path.join(os.path.dirname(HEADER), "..", "INTEGRATION.md")).read()
    block = re.search(r'extern "C" \{(.*?)\n\}', guide, flags=re.S).group(1)
    block = re.sub(r"//[^\n]*", "", block)
    fns = re.findall(r"pub fn (lsb_[a-z0-9_]+)\(([^()]*)\)", block)
    assert len(fns) >= 15
    arity = header_arity()
    for name, args in fns:
        assert name in arity, name
        n = 0 if not args.strip() else args.strip().rstrip(",").count(",") + 1
        assert n == arity[name], (name, n, arity[name])


def test_ctypes_table_matches_the_header_arity():
    arity = header_arity()
    for name, (_res, args) in _lib.SIGNATURES.items():
        assert len(args) == arity[name], (name, len(args), arity[name])


def test_ctypes_structs_have_the_header_layout(tmp_path):
    """Size and every field offset of the ctypes mirrors, against what a C compiler makes of the header."""
    import shutil
    import subprocess
    if shutil.which("gcc") is None:
        pytest.skip("no gcc")
    structs = {"lsb_config": _lib.Config, "lsb_fuse_params": _lib.FuseParamsC, "lsb_align_params": _lib.AlignParamsC,
               "lsb_depth_params": _lib.DepthParamsC, "lsb_result": _lib.Result, "lsb_tuning": _lib.Tuning,
               "lsb_synth_desc": _lib.SynthDesc, "lsb_wav_params": _lib.WavParamsC}
    rename = {"lam": "lambda"}
    body, want = [], []
    for cname, cls in structs.items():
        body.append(f'printf("%zu\\n", sizeof({cname}));')
        want.append(C.sizeof(cls))
        for fname, *_ in cls._fields_:
            body.append(f'printf("%zu\\n", offsetof({cname}, {rename.get(fname, fname)}));')
            want.append(getattr(cls, fname).offset)
    src = tmp_path / "layout.c"
    src.write_text('#include "lapstack_b200.h"\n#include <stdio.h>\n#include <stddef.h>\nint main(void) {\n'
                   + "\n".join(body) + "\nreturn 0;\n}\n")
    exe = tmp_path / "layout"
    cc = subprocess.run(["gcc", "-std=c99", "-I", os.path.dirname(HEADER), str(src), "-o", str(exe)],
                        capture_output=True, text=True)
    assert cc.returncode == 0, cc.stderr
    got = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True, timeout=60).stdout.split()]
    assert got == want


def test_no_cpu_fallback_without_a_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    with pytest.raises(L.LsbError, match="CUDA"):
        L.Engine()


def test_host_synthetic_stack_is_seeded():
    a, ta = L.synth_stack(L.SynthSpec(96, 64, 3, seed=7))
    b, tb = L.synth_stack(L.SynthSpec(96, 64, 3, seed=7))
    c, _ = L.synth_stack(L.SynthSpec(96, 64, 3, seed=8))
    assert a.shape == (3, 64, 96, 3) and a.dtype == np.uint16
    assert np.array_equal(a, b) and np.array_equal(ta, tb)
    assert not np.array_equal(a, c)
    m = a.astype(np.float64) / 65535
    assert 0.35 < m.mean() < 0.55 and 0.05 < m.std() < 0.3


def test_warped_synthetic_stack_records_its_transforms():
    _, t = L.synth_stack(L.SynthSpec(96, 64, 4, warp=True, mag_step=0.0))
    assert np.allclose(t[0], [1, 0, 0, 0])
    assert np.all(np.abs(t[1:, 0] - 1) <= 0.004 + 1e-12) and np.all(np.abs(t[1:, 2:]) <= 8.0)
