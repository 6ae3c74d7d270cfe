"""The C-ABI library loads and exports every symbol the headers in include/
declare (no compute calls: runs without a GPU)."""
import os
import re
import subprocess

from hmfem_b200 import gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    inc = os.path.join(ROOT, "include")
    src = "".join(open(os.path.join(inc, f)).read()
                  for f in sorted(os.listdir(inc)) if f.endswith(".h"))
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = set(re.findall(r"\b([A-Za-z_]\w*)\s*\(", src))
    names -= {"if", "for", "while", "return", "sizeof"}
    names |= set(re.findall(r"extern\s+int\s+(\w+)\s*;", src))
    return sorted(names)


def test_header_declares_the_bridge_and_device_layer():
    names = declared_symbols()
    for s in ("compute", "solve_linsys", "_device_linear_operator",
              "_device_jacobi", "_device_matrix_conversion", "hmfem_solve"):
        assert s in names


def test_library_exports_every_declared_symbol():
    L = gpu.lib()
    missing = [s for s in declared_symbols() if not hasattr(L, s)]
    assert missing == []
    assert gpu.missing_exports() == []


def test_cxx_names_for_the_g_plus_plus_built_application():
    out = subprocess.run(["nm", "-D", "--defined-only", gpu.LIB_PATH],
                         capture_output=True, text=True, check=True).stdout
    assert "_Z7computePiS_S_PdS0_S0_" in out
    assert "_Z12solve_linsysP9ELEstructP5IndexPdS3_9Dimension" in out


def test_struct_layouts_match_reference():
    import ctypes as C
    assert C.sizeof(gpu.Ele) == 56 and C.sizeof(gpu.Ind) == 28
    assert C.sizeof(gpu.Dim) == 32
