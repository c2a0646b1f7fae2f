"""CPU tests of the C ABI: the library loads, exports every declared symbol,
and its struct layout matches the header.  No compute calls."""
import os
import re
import subprocess
import tempfile

import pytest

from conftest import ROOT, gpu_available
from flowlb_b200 import engine as E

HEADER = os.path.join(ROOT, "include", "flowlb.h")


def declared_functions(path=HEADER):
    text = open(path).read()
    return sorted(set(re.findall(r"FLB_API\s+[\w\s\*]+?\b(flb_\w+)\s*\(", text)))


def exported_symbols(lib):
    out = subprocess.run(["nm", "-D", "--defined-only", lib], capture_output=True, text=True, check=True).stdout
    return {line.split()[-1] for line in out.splitlines() if " T " in line}


def test_library_exports_every_declared_function():
    assert os.path.exists(E.LIB_PATH), "engine library not built"
    declared = declared_functions()
    assert len(declared) >= 20
    exported = exported_symbols(E.LIB_PATH)
    missing = [f for f in declared if f not in exported]
    assert not missing, missing
    assert sorted(E.EXPORTS) == declared


def test_library_exports_nothing_else():
    exported = exported_symbols(E.LIB_PATH)
    ours = {s for s in exported if s.startswith("flb_")}
    assert ours == set(declared_functions())


def test_library_loads_and_reports_version():
    L = E.load_library()
    assert b"sm_100a" in L.flb_version()
    assert L.flb_status_string(0) == b"ok"
    assert L.flb_status_string(7) == b"no CUDA device"


def test_case_desc_layout_matches_header():
    """Compiles a C probe against the header and compares field offsets with
    the ctypes mirror used by the Python binding."""
    fields = [f for f, _ in E.CaseDesc._fields_]
    src = '#include <stdio.h>\n#include <stddef.h>\n#include "flowlb.h"\nint main(void){\n'
    src += 'printf("size %zu\\n", sizeof(flb_case_desc));\n'
    for f in fields:
        src += f'printf("{f} %zu\\n", offsetof(flb_case_desc, {f}));\n'
    src += "return 0;}\n"
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "probe.c")
        exe = os.path.join(d, "probe")
        open(c, "w").write(src)
        subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), c, "-o", exe], check=True)
        out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout
    got = dict(line.split() for line in out.strip().splitlines())
    import ctypes
    assert int(got["size"]) == ctypes.sizeof(E.CaseDesc)
    for f in fields:
        assert int(got[f]) == getattr(E.CaseDesc, f).offset, f


def test_case_desc_defaults():
    L = E.load_library()
    d = E.CaseDesc()
    L.flb_case_desc_init(d)
    assert d.precision == 32 and d.mass_precision == 64
    assert d.bounce_back == E.BB_HALFWAY and d.fs_mode == E.FS_CONSERVATIVE
    assert d.device == -1 and abs(d.tau - 0.6) < 1e-7


def test_create_rejects_bad_arguments_before_touching_a_device():
    import ctypes
    import numpy as np
    L = E.load_library()
    flags = np.ones((8, 8), np.uint8)
    d = E.CaseDesc()
    L.flb_case_desc_init(d)
    d.nx, d.ny, d.flags = 8, 8, flags.ctypes.data
    h = ctypes.c_void_p()
    d.tau = 0.4
    assert L.flb_create(d, h) == 1
    d.tau = 0.6
    d.precision = 12
    assert L.flb_create(d, h) == 1
    d.precision = 64
    d.mass_precision = 32
    assert L.flb_create(d, h) == 4
    d.precision, d.mass_precision = 16, 64
    d.f16_scale = 3.0
    assert L.flb_create(d, h) == 1
    d.f16_scale = 0.0
    d.nx = 2
    assert L.flb_create(d, h) == 1
    assert L.flb_create(None, h) == 1


@pytest.mark.skipif(gpu_available(), reason="checks the no-device path")
def test_create_without_device_reports_no_device():
    import numpy as np
    with pytest.raises(E.FlowLBError) as ei:
        E.Solver(np.ones((8, 8), np.uint8))
    assert ei.value.status == 7


def test_null_handle_calls_fail_cleanly():
    import ctypes
    L = E.load_library()
    t = ctypes.c_uint64()
    assert L.flb_step(None, 1) == 1
    assert L.flb_get_time(None, t) == 1
    assert L.flb_destroy(None) == 1
    assert L.flb_last_error(None) == b"null handle"


@pytest.mark.parametrize("lang", ["c99", "c++17"])
def test_header_builds_pedantic_and_links(lang):
    """A host written in C or C++ (FlowLB itself is C++17) includes the header
    with -Wall -Wextra -pedantic -Werror, links against libflowlb.so and calls
    the device-free entry points."""
    src = ('#include <string.h>\n#include "flowlb.h"\n'
           "int main(void) {\n"
           "  flb_case_desc d;\n"
           "  flb_case_desc_init(&d);\n"
           "  if (d.nx != 0 || d.flags) return 1;\n"
           "  if (strcmp(flb_status_string(FLB_ERR_NONFINITE), \"non-finite populations\") != 0) return 2;\n"
           "  if (!flb_version() || !flb_version()[0]) return 3;\n"
           "  if (flb_create(0, 0) != FLB_ERR_INVALID_ARGUMENT) return 4;\n"
           "  return 0;\n}\n")
    libdir = os.path.join(ROOT, "flowlb_b200")
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "host.c" if lang == "c99" else "host.cpp")
        exe = os.path.join(d, "host")
        open(path, "w").write(src)
        cc = ["gcc", "-std=c99"] if lang == "c99" else ["g++", "-std=c++17"]
        subprocess.run(cc + ["-Wall", "-Wextra", "-pedantic", "-Werror", "-I", os.path.join(ROOT, "include"), path,
                             "-L", libdir, "-lflowlb", f"-Wl,-rpath,{libdir}", "-o", exe], check=True)
        assert subprocess.run([exe]).returncode == 0
