"""The C-ABI boundary without a GPU: every function include/tis_b200.h declares
is exported by the built library and bound in tis_b200.abi, and the ctypes
structs match the C layout field for field (compiled here with gcc)."""
import ctypes as C
import os
import re
import subprocess

import pytest

from tis_b200 import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "tis_b200.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^[A-Za-z_][\w\s\*]*?\b(tis_\w+)\s*\(", src, flags=re.M)))


def test_header_declares_the_path():
    names = declared_functions()
    for must in ("tis_init", "tis_neighbor", "tis_force_sumup", "tis_energy_sumup", "tis_time_integral_pre",
                 "tis_step", "tis_replica_exchange", "tis_set_noise", "tis_status", "tis_destroy"):
        assert must in names


def test_binding_list_matches_header():
    assert sorted(abi.EXPORTED) == declared_functions()


@pytest.fixture(scope="module")
def built_library():
    from tis_b200 import build
    build.build()
    return C.CDLL(abi.library_path())


def test_library_exports_every_declared_symbol(built_library):
    missing = [n for n in declared_functions() if not hasattr(built_library, n)]
    assert not missing, missing


def test_loader_declares_signatures(built_library):
    lib = abi.load_library()
    for n in abi.EXPORTED:
        assert getattr(lib, n).argtypes is not None, n


def _c_layout(struct, fields, tmp_path):
    prog = ["#include <stdio.h>", "#include <stddef.h>", f'#include "{HEADER}"', "int main(void) {",
            f'  printf("%zu\\n", sizeof({struct}));']
    for f in fields:
        prog.append(f'  printf("%zu\\n", offsetof({struct}, {f}));')
    prog += ["  return 0;", "}"]
    c = tmp_path / "layout.c"
    c.write_text("\n".join(prog))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c99", "-o", str(exe), str(c)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()
    return int(out[0]), [int(v) for v in out[1:]]


@pytest.mark.parametrize("py,cname", [(abi.Topology, "tis_topology"), (abi.Params, "tis_params"),
                                      (abi.Status, "tis_status_t")])
def test_struct_layout_matches_header(py, cname, tmp_path):
    fields = [f for f, _ in py._fields_]
    size, offs = _c_layout(cname, fields, tmp_path)
    assert C.sizeof(py) == size
    assert [getattr(py, f).offset for f in fields] == offs


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    monkeypatch.setattr(abi, "_LIB", None)
    monkeypatch.setattr(abi, "library_path", lambda: str(tmp_path / "absent.so"))
    with pytest.raises(RuntimeError):
        abi.load_library()
