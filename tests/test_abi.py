"""The C-ABI library loads without a GPU and exports every function include/*.h declares;
the ctypes struct matches the C layout; calls that need no device work on the CPU."""
import ctypes
import glob
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT

DECL = re.compile(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_ \*]*?\b(oco_[a-z0-9_]+)\s*\(", re.M)


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = re.sub(r"/\*.*?\*/", "", open(h).read(), flags=re.S)
        names.update(m.group(1) for m in DECL.finditer(text))
    return sorted(names)


def test_every_declared_symbol_is_exported():
    from ocotillo_b200 import load_library
    lib = load_library()
    names = declared_functions()
    assert len(names) >= 12
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_params_struct_layout_matches_c(tmp_path):
    from ocotillo_b200.engine import OcoParams
    src = tmp_path / "sz.c"
    src.write_text('#include <stddef.h>\n#include <stdio.h>\n#include "oco.h"\nint main(void){printf("%zu %zu %zu %zu\\n",'
                   'sizeof(oco_params), offsetof(oco_params,dz), offsetof(oco_params,lgrey), offsetof(oco_params,reserved));return 0;}\n')
    exe = tmp_path / "sz"
    subprocess.check_call(["gcc", "-I", os.path.join(ROOT, "include"), "-o", str(exe), str(src)])
    size, off_dz, off_lgrey, off_res = map(int, subprocess.check_output([str(exe)]).split())
    assert ctypes.sizeof(OcoParams) == size
    assert OcoParams.dz.offset == off_dz and OcoParams.lgrey.offset == off_lgrey and OcoParams.reserved.offset == off_res


def test_calc_wavelength_without_gpu():
    from ocotillo_b200 import calc_wavelength
    assert list(calc_wavelength(5000.0, 3000.0, 5)) == [3000.0, 3500.0, 4000.0, 4500.0, 5000.0]
    assert list(calc_wavelength(5000.0, 3000.0, 1)) == [3000.0]


def test_create_fails_cleanly_without_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from ocotillo_b200 import Engine, OcoError
    with pytest.raises(OcoError) as e:
        Engine(0)
    assert e.value.code == -5


def test_no_alloc_rejects_bad_sizes_before_touching_a_device():
    from ocotillo_b200.engine import load_library, OcoParams
    lib = load_library()
    prm = OcoParams(1, 1, 1, 8, 1e13, 0.4, 2e4, 0, 0, 0, 0)  # nz = 1
    assert lib.oco_solve_block_noalloc(ctypes.byref(prm), None, ctypes.c_void_p(1), ctypes.c_void_p(1),
                                       ctypes.c_void_p(1), None, None, None, None, None) == -1
