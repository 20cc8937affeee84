"""The C-ABI library loads without a GPU and exports every function include/*.h declares;
every ctypes struct and signature matches the header; calls that need no device work on the
CPU, and argument checks refuse before any device work."""
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
    from ocotillo_b200 import OcoError
    for nw in (0, -3):
        with pytest.raises(OcoError) as e:
            calc_wavelength(5000.0, 3000.0, nw)
        assert e.value.code == -1


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


@pytest.mark.parametrize("dims,dz,msg", [((2**31 - 1, 2**31 - 1, 4096, 4096), 1e13, b"exceeds 2^56"),
                                         ((2**20, 2**20, 4096, 4096), 1e13, b"exceeds 2^56"),
                                         ((1, 1, 8, 8), float("inf"), b"finite"),
                                         ((1, 1, 8, 8), float("nan"), b"finite")])
def test_no_alloc_rejects_oversized_blocks_and_bad_dz(dims, dz, msg):
    """Element counts beyond 2^56 (which would wrap int64 index arithmetic) and a non-finite dz
    are refused before any device work."""
    from ocotillo_b200.engine import load_library, OcoParams
    lib = load_library()
    prm = OcoParams(*dims, dz, 0.4, 2e4, 0, 0, 0, 0)
    one = ctypes.c_void_p(1)
    assert lib.oco_solve_block_noalloc(ctypes.byref(prm), None, one, one, one, None, None, None, None, None) == -1
    assert msg in lib.oco_noalloc_last_error()


def test_no_alloc_rejects_bad_wavelengths_before_touching_a_device():
    from ocotillo_b200.engine import load_library, OcoParams
    lib = load_library()
    prm = OcoParams(1, 1, 8, 4, 1e13, 0.4, 2e4, 0, 0, 0, 0)
    one = ctypes.c_void_p(1)
    for bad in (0.0, -5000.0, float("nan"), float("inf")):
        wa = np.array([3000.0, 4000.0, bad, 6000.0])
        assert lib.oco_solve_block_noalloc(ctypes.byref(prm), wa.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                           one, one, one, None, None, None, None, None) == -1
        assert b"wavelength 2" in lib.oco_noalloc_last_error()


def test_every_ctypes_struct_matches_its_c_layout(tmp_path):
    """Each ctypes mirror in engine.py has the C struct's size and every field's offset."""
    from ocotillo_b200 import engine
    pairs = {"oco_params": engine.OcoParams, "oco_batch_column": engine.OcoBatchColumn,
             "oco_batch_info": engine.OcoBatchInfo, "oco_server_config": engine.OcoServerConfig,
             "oco_job": engine.OcoJob, "oco_job_status": engine.OcoJobStatus,
             "oco_deck_info": engine.OcoDeckInfo}
    lines = []
    for cname, cls in pairs.items():
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for f in cls._fields_:
            lines.append(f'printf("{cname} {f[0]} %zu\\n", offsetof({cname}, {f[0]}));')
    src = tmp_path / "layout.c"
    src.write_text('#include <stddef.h>\n#include <stdio.h>\n#include "oco.h"\nint main(void){'
                   + "".join(lines) + "return 0;}\n")
    exe = tmp_path / "layout"
    subprocess.check_call(["gcc", "-I", os.path.join(ROOT, "include"), "-o", str(exe), str(src)])
    c = {}
    for ln in subprocess.check_output([str(exe)]).decode().splitlines():
        s, f, v = ln.split()
        c[(s, f)] = int(v)
    for cname, cls in pairs.items():
        assert ctypes.sizeof(cls) == c[(cname, "size")], cname
        for f in cls._fields_:
            assert getattr(cls, f[0]).offset == c[(cname, f[0])], (cname, f[0])


def test_dense_batch_offsets_are_prefix_sums():
    from ocotillo_b200 import dense_batch_offsets
    nz = [2, 512, 37, 1024]
    nw = [1, 256, 3, 17]
    o = dense_batch_offsets(nz, nw)
    in_off, u_off, kv_off, f_off = [0], [0], [0], [0]
    for a, b in zip(nz, nw):
        in_off.append(in_off[-1] + a)
        u_off.append(u_off[-1] + (a + 6) * b)
        kv_off.append(kv_off[-1] + a * b)
        f_off.append(f_off[-1] + b)
    assert list(o["in_off"]) == in_off[:-1] and o["n_in"] == in_off[-1]
    assert list(o["u_off"]) == u_off[:-1] and o["n_u"] == u_off[-1]
    assert list(o["kv_off"]) == kv_off[:-1] and o["n_kv"] == kv_off[-1]
    assert list(o["flux_off"]) == f_off[:-1] and o["n_flux"] == f_off[-1]
    one = dense_batch_offsets([5], [4])
    assert list(one["u_off"]) == [0] and one["n_u"] == 44 and one["n_flux"] == 4


def test_batch_offsets_of_a_caller_packing():
    from ocotillo_b200 import batch_offsets, dense_batch_offsets
    nz, nw = [2, 512, 37], [1, 256, 3]
    d = dense_batch_offsets(nz, nw)
    same = batch_offsets(nz, nw, d["in_off"], d["u_off"], d["kv_off"], d["flux_off"])
    assert all(np.array_equal(same[k], d[k]) if k.endswith("_off") else same[k] == d[k] for k in d)
    # reverse order with gaps: every total is the furthest end, not the sum
    o = batch_offsets(nz, nw, [700, 100, 0], [10, 0, 200000], [0, 5, 1000], [9, 4, 0])
    assert o["n_in"] == 702 and o["n_u"] == 200000 + 43 * 3 and o["n_kv"] == 5 + 512 * 256
    assert o["n_flux"] == 4 + 256
    with pytest.raises(ValueError):
        batch_offsets(nz, nw, [0, 1], [0, 0, 0], [0, 0, 0], [0, 0, 0])


def _c_kind(t):
    t = t.strip()
    if "*" in t:
        return "ptr"
    t = re.sub(r"\bconst\b", "", t).split()[0]
    return {"int": "i32", "int32_t": "i32", "int64_t": "i64", "double": "f64", "void": "void"}[t]


def _py_kind(t):
    if t is None:
        return "void"
    if t in (ctypes.c_void_p, ctypes.c_char_p) or isinstance(t, type(ctypes.POINTER(ctypes.c_int))):
        return "ptr"
    return {ctypes.c_int32: "i32", ctypes.c_int64: "i64", ctypes.c_double: "f64"}[t]


def test_ctypes_signatures_match_the_header():
    """Every function the header declares has a ctypes signature in the binding with the same
    number of arguments and the same kind (pointer, int32, int64, double) of each, and the same
    return kind: a mismatch would pass garbage through the ABI without any error."""
    from ocotillo_b200 import load_library
    lib = load_library()
    text = re.sub(r"/\*.*?\*/", "", open(os.path.join(ROOT, "include", "oco.h")).read(), flags=re.S)
    proto = re.compile(r"^\s*((?:const\s+)?[A-Za-z_][A-Za-z0-9_]*\s*\**)\s*(oco_[a-z0-9_]+)\s*\(([^)]*)\)\s*;", re.M)
    seen = 0
    for m in proto.finditer(text):
        ret, name, params = m.group(1), m.group(2), m.group(3)
        params = [] if params.strip() in ("", "void") else params.split(",")
        want = [_c_kind(re.sub(r"\b[A-Za-z_][A-Za-z0-9_]*\s*$", "", p) if "*" not in p.split()[-1] else p)
                for p in params]
        f = getattr(lib, name)
        assert f.argtypes is not None, f"{name}: no ctypes signature"
        assert [_py_kind(a) for a in f.argtypes] == want, name
        assert _py_kind(f.restype) == _c_kind(ret), name
        seen += 1
    assert seen == len(declared_functions())


def test_server_create_refuses_bad_config_and_fails_cleanly_without_gpu():
    from ocotillo_b200 import OcoError, Server
    for kw in ({"max_jobs": 0}, {"max_nz": -1}, {"budget_bytes": -1.0}, {"chunk_points": -5},
               {"reserve_bytes": -1.0}):
        with pytest.raises(OcoError) as e:
            Server(0, **kw)
        assert e.value.code == -1, kw
    import torch
    if not torch.cuda.is_available():
        with pytest.raises(OcoError) as e:
            Server(0, max_jobs=2)
        assert e.value.code == -5
