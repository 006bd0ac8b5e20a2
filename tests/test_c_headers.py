"""The C-ABI headers are plain C: a C99 program that includes every header in
include/, links librrtmg_b200.so and calls the entry points that need no GPU
(the per-step scalar helpers, argument checks, status strings) compiles with
gcc -std=c99 -Wall -Werror and runs."""

from __future__ import annotations

import shutil
import subprocess

import numpy as np
import pytest

from conftest import REPO

PROGRAM = r"""
#include <stdio.h>
#include "rrtmg_b200.h"
#include "rrtmg_surrogate.h"
#include "rrtmg_prologue.h"
#include "rrtmg_tendency.h"
#include "rrtmg_tables.h"

int main(void) {
    float declin = 0.0f, solcon = 0.0f;
    rrtmg_prologue_scalars sc;
    rrtmg_tendency_bounds tb = {0};
    if (rrtmg_radconst(172.3, &declin, &solcon) != RRTMG_OK) return 1;
    if (rrtmg_prologue_scalars_from_calendar(172.3, 195.0, 6.0, declin, &sc) != RRTMG_OK) return 2;
    if (rrtmg_radiation_tendency(&tb, NULL, NULL, NULL, NULL, NULL, 0, NULL, NULL, NULL) != RRTMG_BAD_ARG) return 3;
    if (rrtmg_lw_nlayers(5000.0, 50) != 63) return 4;
    printf("%.9g %.9g %.9g %d %d %.9g %.9g %s\n", declin, solcon, sc.tloctm0, sc.month_lo, sc.month_hi,
           sc.fact_lo, sc.fact_hi, rrtmg_status_string(RRTMG_UNSUPPORTED_OPTION));
    return 0;
}
"""


def test_headers_compile_as_c_and_link(pkg, tmp_path):
    from wrf_jax_b200 import _capi, prologue
    gcc = shutil.which("gcc")
    if gcc is None:
        pytest.skip("no C compiler")
    if not _capi.LIB_PATH.exists():
        pytest.skip("library not built")
    src = tmp_path / "abi.c"
    src.write_text(PROGRAM)
    exe = tmp_path / "abi"
    lib_dir = _capi.LIB_PATH.parent
    cmd = [gcc, "-std=c99", "-Wall", "-Wextra", "-Werror", f"-I{REPO / 'include'}", str(src), "-o", str(exe),
           f"-L{lib_dir}", "-lrrtmg_b200", f"-Wl,-rpath,{lib_dir}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    run = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    assert run.returncode == 0, (run.returncode, run.stderr)
    declin, solcon, t0, lo, hi, f1, f2, status = run.stdout.strip().split(maxsplit=7)
    ref_declin, ref_solcon = prologue.radconst(172.3)
    assert abs(float(declin) - ref_declin) <= 1e-6 and abs(float(solcon) - ref_solcon) <= 1e-3
    lo_, hi_, w1, w2 = prologue.ozone_month_weights(172.3)
    # nine significant digits round-trip binary32: the weights are exact
    assert (int(lo), int(hi)) == (lo_, hi_)
    assert np.float32(float(f1)) == np.float32(w1) and np.float32(float(f2)) == np.float32(w2)
    assert status == "unsupported option"
