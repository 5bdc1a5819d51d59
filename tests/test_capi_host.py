"""Host-side checks of the C ABI library (no GPU needed): it loads, exports every
function include/*.h declares, and rejects unsupported parameter blocks before any CUDA
call, as get_parameters' checks do (Model_rot.f90:336-362)."""
import ctypes
import glob
import os
import re

import pytest

from pip_b200 import build, capi, ics
from pip_b200.params import PIP_ABI_VERSION

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names.update(re.findall(r"\b(pip_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


@pytest.fixture(scope="module")
def lib():
    build.build()
    return capi.lib()


def test_exports_every_declared_symbol(lib):
    names = declared_functions()
    assert "pip_run" in names and "pip_ctx_create" in names
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(names) == set(capi.EXPORTS)


def test_strerror(lib):
    assert capi.strerror(0) == "ok"
    assert "NaN" in capi.strerror(capi.PIP_ERR_NAN)


def _create(s, **field):
    p, keep = s.to_params()
    for k, v in field.items():
        setattr(p, k, v)
    h = ctypes.c_void_p()
    st = capi.lib().pip_ctx_create(ctypes.byref(p), ctypes.byref(h))
    assert not h.value
    return st


@pytest.mark.parametrize("field", [
    dict(abi_version=PIP_ABI_VERSION + 1), dict(ndim=3), dict(flag_sch=1), dict(flag_hll=0),
    dict(s_order=1), dict(t_order=4), dict(flag_time=1), dict(flag_col=0), dict(flag_col=8),
    dict(flag_col=3, precision=1), dict(flag_col=2, beta=0.0), dict(flag_col=6, beta=-1.0),
    dict(nvar_m=9), dict(flag_ir=4), dict(precision=7), dict(flag_pip_imp=2),
])
def test_rejects_unsupported_parameters(lib, field):
    s, _, _ = ics.brio_wu(64)
    assert _create(s, **field) == capi.PIP_ERR_PARAM


def test_rejects_unsupported_boundaries(lib):
    s, _, _ = ics.orszag_tang(16)
    p, keep = s.to_params()
    p.flag_bnd[2] = 20   # custom boundary type 20 is outside the path
    h = ctypes.c_void_p()
    assert capi.lib().pip_ctx_create(ctypes.byref(p), ctypes.byref(h)) == capi.PIP_ERR_PARAM


def test_null_arguments(lib):
    h = ctypes.c_void_p()
    assert capi.lib().pip_ctx_create(None, ctypes.byref(h)) == capi.PIP_ERR_NULL
    assert capi.lib().pip_upload(None, None, None) == capi.PIP_ERR_NULL
    assert capi.lib().pip_run(None, 1, 0.0, None, None) == capi.PIP_ERR_NULL


def test_parameter_block_layout_matches_the_header(tmp_path):
    """The ctypes pip_params has the C struct's size and field offsets (include/pip_gpu.h,
    compiled by the host C compiler), so a Fortran or Python caller and the library agree
    on every field."""
    from pip_b200.params import PipParams
    import shutil
    import subprocess
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no host C compiler")
    names = [f[0] for f in PipParams._fields_]
    src = ["#include <stdio.h>", "#include <stddef.h>",
           '#include "%s"' % os.path.join(ROOT, "include", "pip_gpu.h"),
           "int main(void) {", '  printf("size %zu\\n", sizeof(pip_params));']
    src += ['  printf("%s %%zu\\n", offsetof(pip_params, %s));' % (n, n) for n in names]
    src += ["  return 0;", "}"]
    c = tmp_path / "layout.c"
    c.write_text("\n".join(src) + "\n")
    exe = tmp_path / "layout"
    subprocess.run([cc, "-std=c11", "-o", str(exe), str(c)], check=True)
    out = dict(line.split() for line in subprocess.run([str(exe)], check=True,
                                                       capture_output=True, text=True).stdout.splitlines())
    assert int(out["size"]) == ctypes.sizeof(PipParams)
    for n in names:
        assert int(out[n]) == getattr(PipParams, n).offset, n
