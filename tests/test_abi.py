"""The C ABI: the library loads without a GPU and exports every entry point
that include/pulsesuite_b200.h declares; the numpy struct layouts match the
C structs (checked with the host compiler)."""

import ctypes
import os
import re
import subprocess

import pytest

from pulsesuite_b200 import abi, build

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(REPO, "include", "pulsesuite_b200.h")


def declared():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(psb_\w+)\s*\(", src)))


def test_header_declares_entry_points():
    names = declared()
    for n in ["psb_abi_version", "psb_last_error", "psb_coulomb_vint", "psb_coulomb_k0",
              "psb_chi1d", "psb_screen_f64", "psb_rhs_f64", "psb_rk4_f64", "psb_leapfrog_f64"]:
        assert n in names


def test_library_exports_all_declared_symbols():
    lib = ctypes.CDLL(build.build())
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing
    assert lib.psb_abi_version() == abi.PSB_ABI_VERSION


def test_ctypes_signatures_cover_header():
    from pulsesuite_b200 import _lib

    assert set(declared()) <= set(_lib._SIGNATURES)


def test_struct_layouts_match_c(tmp_path):
    prog = r'''
#include <stdio.h>
#include <stddef.h>
#include "pulsesuite_b200.h"
int main(void) {
  printf("%zu %zu %zu\n", sizeof(PsbTable), sizeof(PsbWire), sizeof(PsbModel));
  printf("%zu %zu %zu %zu %zu %zu\n", offsetof(PsbWire, gap), offsetof(PsbWire, t),
         offsetof(PsbWire, amp), offsetof(PsbWire, p_off), offsetof(PsbWire, status),
         offsetof(PsbWire, steps));
  printf("%zu %zu\n", offsetof(PsbTable, L), offsetof(PsbTable, dens_max));
  printf("%zu %zu %zu\n", sizeof(PsbFullParams), offsetof(PsbFullParams, dt),
         offsetof(PsbFullParams, lf));
  printf("%zu %zu %zu %zu %zu %zu %zu\n", sizeof(PsbFullMB), offsetof(PsbFullMB, vscale),
         offsetof(PsbFullMB, maps), offsetof(PsbFullMB, scratch), offsetof(PsbFullMB, dc_dk),
         offsetof(PsbFullMB, n_hw), offsetof(PsbFullMB, Y));
  return 0;
}
'''
    tmp = str(tmp_path / "abi_layout")
    with open(tmp + ".c", "w") as f:
        f.write(prog)
    r = subprocess.run(["gcc", "-I", os.path.join(REPO, "include"), "-o", tmp, tmp + ".c"],
                       capture_output=True, text=True)
    if r.returncode:
        pytest.skip("no host C compiler: " + r.stderr)
    out = subprocess.run([tmp], capture_output=True, text=True, check=True).stdout.split()
    vals = list(map(int, out))
    W = abi.WIRE_DTYPE
    assert vals[:3] == [abi.TABLE_DTYPE.itemsize, W.itemsize, abi.MODEL_DTYPE.itemsize]
    assert vals[3:9] == [W.fields[f][1] for f in ("gap", "t", "amp", "p_off", "status", "steps")]
    assert vals[9:11] == [abi.TABLE_DTYPE.fields["L"][1], abi.TABLE_DTYPE.fields["dens_max"][1]]
    F = abi.FULL_PARAMS_DTYPE
    assert vals[11:14] == [F.itemsize, F.fields["dt"][1], F.fields["lf"][1]]
    M = abi.FULL_MB_DTYPE
    assert vals[14:] == [M.itemsize] + [M.fields[f][1] for f in ("vscale", "maps", "scratch",
                                                                  "dc_dk", "n_hw", "Y")]
