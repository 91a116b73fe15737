"""The C-ABI library loads, exports every declared symbol, matches the header's
struct layout and rejects bad input before touching a GPU (no GPU needed)."""
import ctypes
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

from west_b200 import lib as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "west_b200.h")


def _declared():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"\b(wb_[a-z_]+)\s*\(", txt)))


def test_header_declares_binding_exports():
    assert sorted(L.EXPORTS) == _declared()


def test_library_exports_every_declared_symbol():
    lib = L.load()
    for name in _declared():
        assert hasattr(lib, name), name
    assert lib.wb_version() >= 100
    out = subprocess.run(["nm", "-D", "--defined-only", L.LIB_PATH], capture_output=True, text=True).stdout
    for name in _declared():
        assert re.search(rf"\bT {name}\b", out), name


def test_struct_layout_matches_header():
    """Size and field offsets of every struct of the header as a C compiler sees them."""
    structs = {"wb_system": L.WbSystem, "wb_stats": L.WbStats, "wb_davidson_params": L.WbDavidsonParams,
               "wb_davidson_info": L.WbDavidsonInfo, "wb_tuning": L.WbTuning}
    src = "#include <stdio.h>\n#include <stddef.h>\n#include \"west_b200.h\"\nint main(){\n"
    expect = []
    for cname, py in structs.items():
        src += f'printf("%zu\\n", sizeof({cname}));\n'
        expect.append(ctypes.sizeof(py))
        for f, _ in py._fields_:
            src += f'printf("%zu\\n", offsetof({cname}, {f}));\n'
            expect.append(getattr(py, f).offset)
    src += "return 0;}\n"
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "t.c"); exe = os.path.join(d, "t")
        open(c, "w").write(src)
        subprocess.run(["gcc", "-I", os.path.dirname(HEADER), c, "-o", exe], check=True)
        vals = [int(x) for x in subprocess.run([exe], capture_output=True, text=True).stdout.split()]
    assert vals == expect


def _sys_struct(tiny, **over):
    keep = {}
    s = L.WbSystem()
    s.npw = s.npwx = tiny.npw
    s.nr1, s.nr2, s.nr3 = tiny.nrs
    s.nbnd_occ = tiny.nbnd_occ
    s.nkb = tiny.nkb
    s.n_dfpt_maxiter = 250
    s.gstart = 2
    arrs = dict(nl=(tiny.nl + 1).astype(np.int32), nlm=(tiny.nlm + 1).astype(np.int32), g2kin=tiny.g2kin,
                vrs=tiny.vrs, evc=np.asfortranarray(tiny.evc), et=tiny.et, occupation=tiny.occupation,
                vkb=np.asfortranarray(tiny.vkb), deeq=np.asfortranarray(tiny.deeq), sqvc=tiny.sqvc)
    for k, v in arrs.items():
        keep[k] = v
        setattr(s, k, v.ctypes.data)
    s.alpha_pv = tiny.alpha_pv; s.omega = tiny.omega; s.wk = tiny.wk
    for k, v in over.items():
        setattr(s, k, v)
    return s, keep


@pytest.mark.parametrize("over,code,msg", [
    (dict(npw=0), L.WB_ERR_ARG, "npw"),
    (dict(nr3=22), L.WB_ERR_UNSUPPORTED, "prime factor above 7"),
    (dict(nr1=17, nr2=17, nr3=17), L.WB_ERR_UNSUPPORTED, "FFT edge"),
    (dict(gstart=1), L.WB_ERR_UNSUPPORTED, "gstart"),
    (dict(nbnd_occ=0), L.WB_ERR_ARG, "nbnd_occ"),
    (dict(omega=0.0), L.WB_ERR_ARG, "omega"),
    (dict(evc=None), L.WB_ERR_ARG, "null"),
])
def test_ctx_create_rejects_bad_input(tiny, over, code, msg):
    lib = L.load()
    s, keep = _sys_struct(tiny, **over)
    ctx = ctypes.c_void_p()
    rc = lib.wb_ctx_create(ctypes.byref(ctx), ctypes.byref(s), 0)
    assert rc == code
    assert msg in lib.wb_last_error().decode()
    assert not ctx.value


def test_null_context_calls_fail_cleanly():
    lib = L.load()
    assert lib.wb_apply_operator(None, 1, None, 1, None, 1, 1e-10, 1, None) == L.WB_ERR_ARG
    assert lib.wb_set_precision(None, 0) == L.WB_ERR_ARG
    assert lib.wb_set_batch(None, 4) == L.WB_ERR_ARG
    assert lib.wb_set_graphs(None, 1) == L.WB_ERR_ARG
    assert lib.wb_set_autotune(None, 1) == L.WB_ERR_ARG
    assert lib.wb_get_tuning(None, None) == L.WB_ERR_ARG
    assert lib.wb_apply_operator_multi(1, None, None, None, None, None, None, 1e-10, 1, None, 0) == L.WB_ERR_ARG
    assert lib.wb_ctx_destroy(None) == L.WB_OK
