"""The C-ABI library loads and exports every symbol include/*.h declares (no GPU needed)."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent


def _declared():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        names |= set(re.findall(r"FOMO_API\s+[\w\s\*]+?\b(fomo_\w+)\s*\(", h.read_text()))
    return names


def test_library_exports_every_declared_symbol(fomo):
    from fomo_b200 import _lib

    L = _lib.lib()
    declared = _declared()
    assert declared, "no FOMO_API declarations found"
    for name in declared:
        assert hasattr(L, name), name
    assert set(_lib.EXPORTS) == declared


def test_version_matches_header(fomo):
    from fomo_b200 import _lib

    hdr = (ROOT / "include" / "fomo_b200.h").read_text()
    v = int(re.search(r"#define FOMO_ABI_VERSION (\d+)", hdr).group(1))
    assert _lib.lib().fomo_version() == v


@pytest.mark.parametrize("order", [2, 4, 6, 8, 10])
@pytest.mark.parametrize("centered", [0, 1])
def test_cfl_bound_matches_reference_formula(fomo, order, centered):
    from fomo_b200 import _lib
    from fomo_b200.api import get_centered_d2, get_fd_coefficients

    vmax, dh = np.float32(4500.0), np.float32(5.0)
    if centered:  # utils/checks.jl:61-70
        c0, d2 = get_centered_d2(order)
        lam = np.float32(abs(c0) + np.float32(2.0) * np.float32(np.sum(np.abs(d2), dtype=np.float32)))
        want = np.float32(2.0) * dh / (vmax * np.sqrt(np.float32(2.0) * lam))
    else:  # utils/checks.jl:39-48
        a = get_fd_coefficients(order)
        want = dh / (vmax * np.sqrt(np.float32(2.0)) * np.float32(np.sum(np.abs(a), dtype=np.float32)))
    got = C.c_float()
    rc = _lib.lib().fomo_check_numerics(float(vmax), float(dh), 1e-6, order, centered, C.byref(got))
    assert rc == 0
    assert abs(got.value - float(want)) <= 2e-7 * float(want)
    rc = _lib.lib().fomo_check_numerics(float(vmax), float(dh), 1.0, order, centered, C.byref(got))
    assert rc == _lib.FOMO_EARG


def test_bad_arguments_return_codes_without_a_device(fomo):
    from fomo_b200 import _lib

    L = _lib.lib()
    assert L.fomo_check_numerics(3000.0, 10.0, 1e-3, 7, 0, None) == _lib.FOMO_EARG
    assert L.fomo_last_error(None) == b"null context"
    # solver entry points reject a NULL context instead of crashing
    assert L.fomo_elastic2d_batch(None, None, None, None, None, None, None, None, None, None) != 0
    assert L.fomo_coupled2d(None, None, None, None, 0.0, 3.0, None, 0, None, None, None, None,
                            None, None) == _lib.FOMO_EARG
    assert L.fomo_debug_coupled_medium(None, 4, 4, 2, 8, 10.0, 3.0, None, None,
                                       None) == _lib.FOMO_EARG


def test_create_without_device_fails_cleanly(fomo):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    from fomo_b200 import _lib

    h = C.c_void_p()
    assert _lib.lib().fomo_create(C.byref(h), 0) == _lib.FOMO_ECUDA
    assert not h.value


_STRUCTS = [("Grid2D", "fomo_grid2d"), ("Acq", "fomo_acq"), ("Grid3D", "fomo_grid3d"),
            ("Acq3D", "fomo_acq3d"), ("Shot2D", "fomo_shot2d"), ("Opts", "fomo_opts"),
            ("Stats", "fomo_stats")]


def test_ctypes_struct_layouts_match_header(fomo, tmp_path):
    """Every ctypes mirror has the size and field offsets of its C struct."""
    import shutil
    import subprocess

    from fomo_b200 import _lib as L

    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    inc = Path(__file__).resolve().parents[1] / "include"
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "fomo_b200.h"',
             "int main(void) {"]
    want = []
    for py, c in _STRUCTS:
        cls = getattr(L, py)
        lines.append(f'  printf("%zu\\n", sizeof({c}));')
        want.append(C.sizeof(cls))
        for name, _ in cls._fields_:
            lines.append(f'  printf("%zu\\n", offsetof({c}, {name}));')
            want.append(getattr(cls, name).offset)
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run([cc, "-I", str(inc), "-o", str(exe), str(src)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], check=True, capture_output=True,
                                          text=True).stdout.split()]
    assert got == want
