"""CPU tests of the drop-in boundary: the C-ABI library loads and exports
every entry point declared in include/symprop.h; host-only helpers work
without a GPU (no compute call is made here)."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

import symprop_b200 as sp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "symprop.h")).read()
    return sorted(set(re.findall(r"\b(symprop_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    L = sp.lib()
    names = declared_symbols()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    assert set(sp.exported_symbols()) <= set(names)


def test_status_strings_and_host_helpers():
    L = sp.lib()
    assert L.symprop_status_string(0) == b"ok"
    assert L.symprop_status_string(2) == b"unsupported order"
    assert sp.symtens_size(16, 3) == 816
    c = sp.symtens_coeff(3, 3)
    assert c.sum() == 27


def test_headers_compile_as_c_and_cpp(tmp_path):
    src = tmp_path / "t.c"
    src.write_text('#include "symprop.h"\nint main(void){return SYMPROP_OK;}\n')
    subprocess.run(["gcc", "-std=c99", "-I", os.path.join(ROOT, "include"), "-c", str(src), "-o",
                    str(tmp_path / "t.o")], check=True)
    cpp = tmp_path / "t.cpp"
    cpp.write_text('#include "symtucker.hpp"\nint main(){symprop::Config c; return (int)c.rank - 2;}\n')
    # the reference's API and this library's additions compile as a caller writes them
    api = tmp_path / "api.cpp"
    api.write_text('''#include "symtucker.hpp"
using namespace symprop;
int use(const char *path) {
  SpSymtensor X = SpSymtensor::load(path);
  X.save_spt("x.spt");
  std::vector<real_t> U(X.dim() * 4), Y(X.dim() * symtens_size(4, X.order() - 1)), C(4 * 4);
  X.S3TTMc(Y, U, 4, true);
  matrix::gemmtn(C, U, U, X.dim(), 4, 4);
  matrix::qr(U, X.dim(), 4);
  std::vector<real_t> coeff = symtens_coeff(4, X.order() - 1), F((size_t)X.dim() * X.dim());
  matrix::symgemm(F, Y, Y, coeff, X.dim(), X.dim());
  Config c;
  c.rank = 4;
  SymTuckerDecomp d = X.TuckerHOOI(c);
  d.print(std::cout);
  FunctionTimer::printTimes();
  return (int)X.size();
}
''')
    subprocess.run(["/usr/bin/g++", "-std=c++20", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), "-c",
                    str(api), "-o", str(tmp_path / "api.o")], check=True)
    subprocess.run(["/usr/bin/g++", "-std=c++20", "-I", os.path.join(ROOT, "include"), "-c",
                    str(cpp), "-o", str(tmp_path / "t2.o")], check=True)


def test_cli_help_and_unknown_flag():
    cli = sp.CLI_PATH
    r = subprocess.run([cli, "-h"], capture_output=True, text=True)
    assert r.returncode == 1 and "-f <input_file>" in r.stdout
    r = subprocess.run([cli, "-zz"], capture_output=True, text=True)
    assert r.returncode == 1 and "Option -zz is not defined" in r.stdout


def test_symtens_ttmc_usage_and_open_failure(tmp_path):
    """examples/symtens_ttmc.cpp:12-27: fewer than two arguments print the
    usage line, an unreadable file the open error; both exit 1 before any
    device work."""
    exe = sp.TTMC_PATH
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 1 and r.stderr == f"Usage: {exe} <input_file> <R>\n"
    r = subprocess.run([exe, "only-one"], capture_output=True, text=True)
    assert r.returncode == 1 and r.stderr.startswith("Usage: ")
    missing = str(tmp_path / "none.tns")
    r = subprocess.run([exe, missing, "4"], capture_output=True, text=True, cwd=tmp_path)
    assert r.returncode == 1 and r.stderr == f"Error opening file: {missing}\n"
    assert not (tmp_path / "ttmc.out").exists()
