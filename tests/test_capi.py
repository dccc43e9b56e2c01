"""The C ABI: libxac.so loads, exports every function include/xac.h declares, and the ctypes structs
match the header's layout. No compute calls (runs without a GPU)."""
import re
import subprocess
import ctypes as C
from pathlib import Path

import pytest

from xadvcool_b200 import _capi

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "xac.h"


def declared_functions():
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    return sorted(set(re.findall(r"\b(xac_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_entry_points():
    names = declared_functions()
    assert "xac_lattice_step" in names and "xac_stream" in names
    assert len(names) >= 30


def test_library_exports_every_declared_symbol():
    lib = _capi.load()
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, f"declared in xac.h but not exported: {missing}"


def test_ctypes_signatures_cover_header():
    names = set(declared_functions()) - {"xac_last_error", "xac_version"}
    assert names <= set(_capi.SIGNATURES), sorted(names - set(_capi.SIGNATURES))


def test_struct_layout_matches_header(tmp_path):
    src = tmp_path / "layout.c"
    src.write_text(f'''
#include <stdio.h>
#include <stddef.h>
#include "{HEADER}"
int main(void) {{
  printf("%zu %zu %zu %zu %zu %zu\\n", sizeof(xac_desc), offsetof(xac_desc, tau_fluid), offsetof(xac_desc, precision),
         sizeof(xac_scalar_params), sizeof(xac_run_opts), sizeof(xac_run_result));
  printf("%zu %zu %zu %zu %zu\\n", offsetof(xac_run_result, u_inlet_final), offsetof(xac_run_result, last_stats),
         sizeof(xac_design_spec), offsetof(xac_design_spec, background), offsetof(xac_design_spec, hot));
  return 0;
}}''')
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-o", str(exe), str(src)], check=True)
    a, b = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")[:2]
    got = [int(v) for v in a.split()] + [int(v) for v in b.split()]
    want = [C.sizeof(_capi.Desc), _capi.Desc.tau_fluid.offset, _capi.Desc.precision.offset,
            C.sizeof(_capi.ScalarParams), C.sizeof(_capi.RunOpts), C.sizeof(_capi.RunResult),
            _capi.RunResult.u_inlet_final.offset, _capi.RunResult.last_stats.offset, C.sizeof(_capi.DesignSpec),
            _capi.DesignSpec.background.offset, _capi.DesignSpec.hot.offset]
    assert got == want


def test_constants_match_header():
    text = HEADER.read_text()
    assert f"#define XAC_NSTATS {_capi.NSTATS}" in text
    assert f"#define XAC_NSCALARS {_capi.NSCALARS}" in text


def test_invalid_arguments_are_reported_without_touching_the_gpu():
    lib = _capi.load()
    h = C.c_void_p()
    rc = lib.xac_lattice_create(None, C.byref(h), None)
    assert rc == _capi.XAC_EINVAL
    assert b"null descriptor" in lib.xac_last_error()
    with pytest.raises(_capi.XacError):
        _capi.check(rc)
    rc = lib.xac_equilibrium(None, None, None, 0, 1, 1, None)
    assert rc == _capi.XAC_EINVAL and b"positive" in lib.xac_last_error()


def test_autotune_cache_is_keyed_on_the_library_build(tmp_path, monkeypatch):
    """Launch shapes timed on one build of libxac.so are not reused by another: the cache key holds a hash of the
    library file, so a rebuilt kernel or a new population layout is timed afresh."""
    import shutil
    from xadvcool_b200 import autotune
    first = autotune._lib_id()
    assert re.fullmatch(r"[0-9a-f]{12}", first) and autotune._lib_id() == first
    copy = tmp_path / "libxac.so"
    shutil.copyfile(_capi.LIB_PATH, copy)
    with open(copy, "ab") as f:
        f.write(b"\0")  # another build
    monkeypatch.setattr(_capi, "LIB_PATH", copy)
    monkeypatch.setattr(autotune, "_LIB_ID", None)
    assert autotune._lib_id() != first
