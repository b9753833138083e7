"""The C ABI library: builds for sm_100a, loads, exports every declared
entry point, fails cleanly without a GPU; the C++ drop-in header compiles."""
from __future__ import annotations

import ctypes as C
import re
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
PKG = ROOT / "3dfilteredbackprojection-public_b200"
HEADER = ROOT / "include" / "fbp_b200.h"


def declared_symbols() -> list[str]:
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(fbp\w+)\s*\(", text, re.M)))


@pytest.fixture(scope="module")
def lib():
    import build as B
    B.build()
    import fbp_b200
    return fbp_b200.library()


def test_header_declares_the_pipeline():
    syms = declared_symbols()
    for name in ("fbp_create", "fbp_apply_fdk_weights_to_projections", "fbp_apply_filter_to_projections",
                 "fbp_project_backward_cone_fdk_from_projections", "fbp_read_volume", "fbp_last_error",
                 "fbp2d_project_backward", "fbp_fft_rows"):
        assert name in syms


def test_library_exports_every_declared_symbol(lib):
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_python_mirror_covers_the_header():
    import fbp_b200
    assert set(declared_symbols()) == set(fbp_b200.SIGNATURES)


def test_build_targets_sm100a_only():
    import build as B
    assert B.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]


def test_null_context_is_an_error(lib):
    assert lib.fbp_synchronize(None) == -1
    assert b"null context" in lib.fbp_last_error(None)


def test_create_without_gpu_reports_error(lib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = C.c_void_p()
    rc = lib.fbp_create(C.byref(h), 0)
    assert rc != 0 and not h.value
    assert lib.fbp_last_error(None)


def test_cpp_dropin_header_compiles(tmp_path):
    src = tmp_path / "use.cpp"
    src.write_text(
        '#include "fbp_b200.hpp"\n'
        "int main() {\n"
        "  fbp::FBP3D solver;\n"
        "  solver.upload_projections(nullptr, 8, 8, 4);\n"
        "  solver.apply_fdk_weights_to_projections(730.87f, 669.04f, 409.60f);\n"
        "  solver.apply_filter_to_projections(fbp::FBP2D::FilterType::SHEPP_LOGAN);\n"
        "  solver.project_backward_cone_fdk_from_projections(730.87f, 669.04f, 409.60f, 213.84f, 1, 8, 8, 0);\n"
        "  float slice[64];\n  solver.load_volume_slice_y(0, slice);\n"
        "  solver.generate_blank_sinograms(8, 8, 4);\n"
        "  solver.store_projection_to_sinograms(slice, 2);\n"
        "  solver.load_projection_from_sinograms(2, slice);\n"
        "  fbp::FBP2D f2;\n  f2.set_precision(FBP_PRECISION_MIXED);\n"
        "  return 0;\n}\n")
    r = subprocess.run(["g++", "-std=c++17", "-fsyntax-only", f"-I{ROOT / 'include'}", f"-I{PKG}", str(src)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_cpp_dropin_links_against_library(tmp_path):
    src = tmp_path / "link.cpp"
    src.write_text('#include "fbp_b200.hpp"\nint main(){ try { fbp::FBP3D s; } catch (const fbp::Error&) {} return 0; }\n')
    exe = tmp_path / "link"
    r = subprocess.run(["g++", "-std=c++17", f"-I{ROOT / 'include'}", f"-I{PKG}", str(src), "-o", str(exe),
                        f"-L{PKG}", "-lfbp_b200", f"-Wl,-rpath,{PKG}"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_projection_file_index_rule():
    """read_projections takes a file's projection index from the 4 characters
    before a 4-character extension (FBP3D.cpp:97-104); names without one are
    ignored. Host-only: no device is touched."""
    import fbp_b200 as F
    cases = {"dir/proj_0012.raw": 12, "a/b/0007.tif": 7, "scan1234.raw": 1234, "ab12cd.raw": 12,
             "img-001.raw": -1, "x.raw": -1, "abc": -1, "readme.txt": -1}
    for name, idx in cases.items():
        assert F.projection_file_index(name) == idx, name
