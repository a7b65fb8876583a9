"""C-ABI library checks that need no GPU: it loads, exports every function
include/shygpu.h declares, computes geometry, and fails loudly (no CPU
fallback) when a compute entry has no device."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

import shygpu
import shyref

ROOT = Path(__file__).resolve().parents[1]


def declared_functions():
    text = (ROOT / "include" / "shygpu.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?[a-z_0-9]+\s*\*?\s*([a-z_0-9]+)\s*\(", text, flags=re.M)
    return sorted(set(n for n in names if n not in ("if", "while")))


def test_library_exports_every_declared_symbol():
    lib = shygpu.lib()
    names = declared_functions()
    assert "system_solve_" in names and "shygpu_run" in names
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    C.c_int.in_dll(lib, "shy_zeta_system")      # the element-data struct is exported too


def test_set_ev_matches_oracle(channel):
    ev32 = shygpu.set_ev(channel)
    ev64 = shyref.set_ev(channel)
    # b, c and aj in single precision (the library stores ev as real like the reference)
    assert np.allclose(ev32[:, 3:10], ev64[:, 3:10], rtol=2e-6, atol=1e-12)
    assert np.allclose(ev32[:, 16:19], ev64[:, 16:19], rtol=1e-6)


def test_no_cpu_fallback_without_device(channel):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    with pytest.raises(shygpu.ShyError) as ei:
        shygpu.Model(channel)
    assert ei.value.code == 2          # SHY_ECUDA


def test_footprint_positive(small3d):
    assert shygpu.footprint([small3d]) > 0


def test_header_is_plain_c99(tmp_path):
    """include/shygpu.h is a C ABI: it compiles as strict C99 (a Fortran
    iso_c_binding or cgo host includes it from C)."""
    import shutil
    import subprocess
    from pathlib import Path
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    src = tmp_path / "use.c"
    src.write_text('#include "shygpu.h"\nint main(void) { return shygpu_last_error() == 0; }\n')
    inc = Path(__file__).resolve().parents[1] / "include"
    r = subprocess.run([cc, "-std=c99", "-Wall", "-Wextra", "-pedantic", "-Werror", "-fsyntax-only",
                        "-I", str(inc), str(src)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
