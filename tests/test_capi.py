"""CPU checks of the drop-in boundary: libexcfv loads, exports every entry point
declared in include/excfv.h, and the ctypes mirror of struct excfv_static has
the C layout (compiled with gcc from the header).  No compute call is made."""
import ctypes as C
import os
import re
import subprocess
import tempfile

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "excfv.h")


def _declared():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(excfv_[a-z0-9_]+)\s*\(", src)))


@pytest.fixture(scope="module")
def lib():
    from exciting_b200 import lib as L
    if not os.path.exists(L.LIB_PATH):
        from exciting_b200.build import build_library
        build_library()
    return L.load()


def test_header_declares_the_reference_entry_points():
    names = _declared()
    for n in ["excfv_match", "excfv_hamiltonandoverlapsetup", "excfv_solvewithlapack",
              "excfv_seceqnfv", "excfv_seceqn", "excfv_set_static"]:
        assert n in names


def test_library_exports_every_declared_symbol(lib):
    from exciting_b200 import lib as L
    for name in _declared():
        assert hasattr(lib, name), name
        assert name in L.SIGNATURES, f"{name} has no ctypes signature"


@pytest.mark.parametrize("pyname,cname", [("ExcfvStatic", "excfv_static"), ("ExcfvMtrad", "excfv_mtrad"),
                                           ("ExcfvRhoset", "excfv_rhoset"), ("ExcfvBfield", "excfv_bfield"),
                                           ("ExcfvBfieldNc", "excfv_bfield_nc")])
def test_struct_layout_matches_c(lib, pyname, cname):
    from exciting_b200 import lib as L
    cls = getattr(L, pyname)
    fields = [f for f, _ in cls._fields_]
    prog = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"', "int main(void){",
            f'printf("%zu\\n", sizeof({cname}));']
    for f in fields:
        prog.append(f'printf("%zu\\n", offsetof({cname}, {f}));')
    prog.append("return 0;}")
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "t.c")
        exe = os.path.join(d, "t")
        open(c, "w").write("\n".join(prog))
        subprocess.run(["gcc", "-O0", "-o", exe, c], check=True)
        out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split()
    vals = [int(x) for x in out]
    assert vals[0] == C.sizeof(cls)
    for f, off in zip(fields, vals[1:]):
        assert getattr(cls, f).offset == off, f


def test_status_codes_match_header():
    from exciting_b200 import lib as L
    src = open(HEADER).read()
    for name in ["EXCFV_OK", "EXCFV_ERR_ARG", "EXCFV_ERR_UNSUPPORTED", "EXCFV_ERR_CUDA",
                 "EXCFV_ERR_ALLOC", "EXCFV_ERR_STATE", "EXCFV_ERR_TIMEOUT", "EXCFV_ERR_NOCONV",
                 "EXCFV_PREC_FP64", "EXCFV_PREC_MIXED"]:
        m = re.search(rf"#define {name} \(?(-?\d+)\)?", src)
        assert m, name
        assert int(m.group(1)) == getattr(L, name)


def test_create_without_gpu_fails_cleanly(lib):
    """On a machine without a GPU the handle cannot be created and the call says so."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = C.c_void_p()
    rc = lib.excfv_create(0, C.byref(h))
    assert rc < 0
    assert lib.excfv_last_error()
