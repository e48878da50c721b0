"""The C-ABI library loads on a machine without a GPU and exports every symbol include/*.h declares."""
import os
import re
import subprocess

from pcbroute_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_pcbg():
    src = open(os.path.join(ROOT, "include", "pcbg.h")).read()
    return sorted(set(re.findall(r"\b(pcbg_[a-z_0-9]+)\s*\(", src)))


def test_library_loads_and_exports_pcbg_h():
    lib = _lib.load()
    names = _declared_pcbg()
    assert "pcbg_solve" in names and "pcbg_solve_batch" in names
    for n in names:
        getattr(lib, n)  # raises AttributeError if missing
    assert _lib.exported_symbols() == []


def test_gpu_h_symbols_are_exported_with_cpp_linkage():
    """The router objects (src/router.cpp built with -DPCB_GPU) resolve exactly these mangled names."""
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True).stdout
    demangled = subprocess.run(["c++filt"], input=out, capture_output=True, text=True).stdout
    for sig in ["gpu_available()", "gpu_configure(int, unsigned long)",
                "gpu_solve(GpuQuery const&, GpuOut&, bool)", "GpuOut::~GpuOut()", "GpuOut::reserve(unsigned long)",
                "GpuOut::operator()(long) const"]:
        assert sig in demangled, sig


def test_struct_layouts_match_the_header():
    """ctypes mirrors of pcbg_query / pcbg_result / pcbg_search agree with the C compiler's layout."""
    import ctypes as C
    import tempfile
    prog = r'''
#include <stdio.h>
#include <stddef.h>
#include "pcbg.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu %zu %zu\n", sizeof(pcbg_query), offsetof(pcbg_query, tbit), offsetof(pcbg_query, mlf),
         sizeof(pcbg_result), offsetof(pcbg_result, ub), sizeof(pcbg_search), offsetof(pcbg_search, best));
  return 0;
}
'''
    with tempfile.TemporaryDirectory() as d:
        c, exe = os.path.join(d, "l.c"), os.path.join(d, "l")
        open(c, "w").write(prog)
        subprocess.run(["gcc", "-I" + os.path.join(ROOT, "include"), c, "-o", exe], check=True)
        got = [int(x) for x in subprocess.run([exe], capture_output=True, text=True).stdout.split()]
    want = [C.sizeof(_lib.Query), _lib.Query.tbit.offset, _lib.Query.mlf.offset, C.sizeof(_lib.Result),
            _lib.Result.ub.offset, C.sizeof(_lib.Search), _lib.Search.best.offset]
    assert got == want


def test_no_device_reports_unavailable_without_crashing():
    import torch
    if torch.cuda.is_available():
        return
    assert _lib.load().pcbg_available() == 0
