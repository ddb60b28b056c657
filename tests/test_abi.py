"""CPU tests of the drop-in boundary: libgalpha.so loads, exports every entry
point the public headers declare (including the reference's C++ symbols), the
headers compile as C and C++, and without a GPU every entry point fails with a
status instead of falling back to the CPU."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

import galpha_b200 as G

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INC = os.path.join(ROOT, "include")
LIB = os.path.join(ROOT, "galpha_b200", "lib", "libgalpha.so")


def declared_functions():
    names = set()
    for h in ("gpudt.h", "galpha.h"):
        src = open(os.path.join(INC, h)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^\s*[A-Za-z_][\w\s\*]*?\b([A-Za-z_]\w*)\s*\([^;{]*\)\s*;", src, flags=re.M):
            names.add(m.group(1))
    return names


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(LIB):
        from galpha_b200 import build

        build.build()
    return G.load()


def exported():
    out = subprocess.run(["nm", "-D", "--defined-only", LIB], capture_output=True, text=True).stdout
    return {ln.split()[-1] for ln in out.splitlines() if " T " in ln}


def test_exports_every_declared_symbol(lib):
    exp = exported()
    decl = declared_functions()
    cpp = {"gpudtComputeDT": "_Z14gpudtComputeDTP11GPUDTPARAMS",
           "gpudtReleaseDTOutput": "_Z20gpudtReleaseDTOutputP11GPUDTOUTPUT"}
    assert decl, "header parse found nothing"
    for name in decl:
        assert cpp.get(name, name) in exp, name


def test_headers_compile_as_c_and_cpp(tmp_path):
    src = tmp_path / "use.c"
    src.write_text('#include "gpudt.h"\n#include "galpha.h"\n#include <stdio.h>\n'
                   'int main(void){GPUDTPARAMS p; GPUDTOUTPUT o; gpudtStatus s;\n'
                   'double xy[6]={0,0,1,0,0,1}; p.minX=0;p.minY=0;p.maxX=1;p.maxY=1;p.nPoints=3;'
                   'p.points=(gpudtVertex*)xy;p.nConstraints=0;p.constraints=0;p.fboSize=256;\n'
                   'int r = gpudtComputeDTEx(&p,&o,&s); printf("%d\\n", r); return 0;}\n')
    exe = tmp_path / "use"
    subprocess.run(["gcc", "-I", INC, str(src), "-o", str(exe), LIB, "-Wl,-rpath," + os.path.dirname(LIB)], check=True)
    subprocess.run(["g++", "-x", "c++", "-I", INC, "-c", str(src), "-o", str(tmp_path / "use.o")], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0
    code = int(r.stdout.strip().splitlines()[-1])
    try:
        import torch

        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    assert code == (0 if has_gpu else -7)


def test_struct_layouts_match_c(lib, tmp_path):
    """ctypes mirrors must have the C compiler's sizes and offsets."""
    from galpha_b200.api import ALPHA_DTYPE, QueryResult, Status, _AlphaOut, _MasterOut, _Output, _Params

    src = tmp_path / "sz.c"
    src.write_text('#include "gpudt.h"\n#include "galpha.h"\n#include <stdio.h>\n#include <stddef.h>\n'
                   'int main(void){printf("%zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu\\n", sizeof(GPUDTPARAMS), '
                   'sizeof(GPUDTOUTPUT), sizeof(gpudtStatus), sizeof(GAlphaOutput), sizeof(gpudtTriangle), '
                   'sizeof(galphaEdgeInterval), sizeof(galphaPointInterval), offsetof(GPUDTPARAMS, fboSize), '
                   'offsetof(gpudtStatus, ms), sizeof(galphaQueryResult), offsetof(galphaQueryResult, nTris), '
                   'sizeof(galphaAlpha), sizeof(GAlphaMasterList)); return 0;}\n')
    exe = tmp_path / "sz"
    subprocess.run(["gcc", "-I", INC, str(src), "-o", str(exe)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True).stdout.split()]
    mine = [ctypes.sizeof(_Params), ctypes.sizeof(_Output), ctypes.sizeof(Status), ctypes.sizeof(_AlphaOut),
            G.TRIANGLE_DTYPE.itemsize, G.EDGE_INTERVAL_DTYPE.itemsize, G.POINT_INTERVAL_DTYPE.itemsize,
            _Params.fboSize.offset, Status.ms.offset, ctypes.sizeof(QueryResult), QueryResult.nTris.offset,
            ALPHA_DTYPE.itemsize, ctypes.sizeof(_MasterOut)]
    assert got == mine


def test_no_device_fails_loudly(lib):
    try:
        import torch

        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except Exception:
        pass
    with pytest.raises(G.GpudtError) as e:
        G.Engine()
    assert e.value.code == -7


def test_reads_reference_input_format(tmp_path):
    f = tmp_path / "pts.txt"
    f.write_text("3\n0 1.5 2\n2 -1 0.25\n1 3 4\n")
    p = G.read_points_file(str(f))
    assert np.array_equal(p, np.array([[1.5, 2], [3, 4], [-1, 0.25]]))
