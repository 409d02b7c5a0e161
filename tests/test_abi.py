"""The C-ABI library: loads, exports every symbol include/daw_b200.h declares,
host-side helpers agree with the oracle, and it refuses to run without a GPU
(no CPU fallback).  CPU only (no compute calls)."""
import ctypes
import subprocess

import numpy as np
import pytest


def test_exports_every_header_symbol(pkg):
    L = pkg.lib()
    names = pkg.header_symbols()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_nm_dynamic_exports(pkg):
    out = subprocess.run(["nm", "-D", "--defined-only", pkg.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    for n in pkg.header_symbols():
        assert n in exported, n


def test_hicks_tiles_match_oracle(pkg, O):
    for args in [(51, 51, 0), (1, 100, 0), (37, 12, 9), (100, 3, 4), (63, 77, 10), (5, 95, 1)]:
        assert np.array_equal(pkg.kws_tile(*args), O.kws_tile(*args)), args


def test_subsourcekws_matches_oracle(pkg, O):
    rng = np.random.default_rng(0)
    for _ in range(200):
        z, x = rng.uniform(0, 300), rng.uniform(0, 9000)
        h = float(rng.choice([4.0, 5.0, 12.5, 20.0]))
        for ofs in (0, 1):
            assert np.array_equal(pkg.subsourcekws(z, x, h, ofs), O.subsourcekws(z, x, h, ofs))


def test_no_cpu_fallback(pkg):
    # without a CUDA device daw_create must fail with DAW_ERR_NODEV
    try:
        rt = ctypes.CDLL("libcudart.so.12")
        n = ctypes.c_int(0)
        has = rt.cudaGetDeviceCount(ctypes.byref(n)) == 0 and n.value > 0
    except OSError:
        has = False
    if has:
        pytest.skip("a GPU is present")
    with pytest.raises(pkg.DawError) as e:
        pkg.Handle(0)
    assert e.value.code == -8


def test_driver_executable_exists(pkg):
    import os
    exe = os.path.join(os.path.dirname(pkg.LIB_PATH), "main_redatum_daw")
    assert os.access(exe, os.X_OK)


C_CLIENT = r"""
#include <math.h>
#include <stdio.h>
#include "daw_b200.h"

int main(void) {
  float tile[21 * 21];
  double sum = 0.0;
  int32_t loc[5];
  daw_handle* h = NULL;
  int rc;
  daw_hicks_tile(51, 51, 0, tile);           /* on-node monopole: sums to 1 */
  for (int i = 0; i < 21 * 21; ++i) sum += tile[i];
  daw_hicks_locate(40.0f, 100.0f, 20.0f, 1, loc);
  rc = daw_create(&h, 0);
  if (rc == DAW_OK) daw_destroy(h);
  printf("%.6f %d %d %d %d %d %d\n", sum, loc[0], loc[1], loc[2], loc[3], loc[4], rc);
  return 0;
}
"""


def test_header_is_plain_c(pkg, tmp_path):
    """include/daw_b200.h compiles as C99 and a C client links the library:
    the boundary a Fortran (ISO_C_BINDING) or any C-FFI caller binds."""
    import os
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    src = tmp_path / "client.c"
    src.write_text(C_CLIENT)
    exe = tmp_path / "client"
    libdir = os.path.dirname(pkg.LIB_PATH)
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-pedantic",
                    "-I", os.path.join(root, "include"), str(src), "-o", str(exe),
                    "-L", libdir, "-ldaw_b200", "-Wl,-rpath," + libdir, "-lm"],
                   check=True, capture_output=True, text=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()
    assert abs(float(out[0]) - 1.0) < 1e-5
    assert [int(v) for v in out[1:6]] == [3, 6, 51, 51, 8]  # subsourcekws on a grid node
    assert int(out[6]) in (0, -8)  # a handle on a GPU box, DAW_ERR_NODEV without one
