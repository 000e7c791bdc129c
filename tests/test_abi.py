"""C ABI checks that need no GPU: the library builds and loads, exports every entry point
include/spgpu.h declares, its struct layouts match the ctypes mirror, it refuses to run
without a device (no CPU fallback), and its host-side filler routines reproduce the
reference's initializeFillers / scatterFillers."""
import ctypes as C
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

from superplace_b200 import abi, engine

from .conftest import ROOT, golden_small_db

HEADER = os.path.join(ROOT, "include", "spgpu.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?[a-z_0-9]+\*?\s+\**(spg_[a-z_0-9]+)\s*\(", src, re.M)))


def test_library_exports_every_declared_symbol():
    names = declared_functions()
    assert len(names) >= 30
    L = engine.lib()
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_struct_layouts_match_header():
    probe = r"""
#include <stdio.h>
#include <stddef.h>
#include "spgpu.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu\n", sizeof(spg_db_view), sizeof(spg_params), sizeof(spg_result),
         sizeof(spg_iter_metrics), sizeof(spg_filler_info));
  printf("%zu %zu %zu %zu\n", offsetof(spg_db_view, total_row_area), offsetof(spg_params, random_seed),
         offsetof(spg_iter_metrics, evaluations), offsetof(spg_iter_metrics, elapsed_ms));
  return 0;
}
"""
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "p.c")
        open(c, "w").write(probe)
        exe = os.path.join(d, "p")
        subprocess.run(["/usr/bin/gcc", "-I", os.path.join(ROOT, "include"), c, "-o", exe], check=True)
        out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split()
    sizes = [int(v) for v in out]
    mine = [C.sizeof(abi.DbView), C.sizeof(abi.Params), C.sizeof(abi.Result),
            C.sizeof(abi.IterMetrics), C.sizeof(abi.FillerInfo),
            abi.DbView.total_row_area.offset, abi.Params.random_seed.offset,
            abi.IterMetrics.evaluations.offset, abi.IterMetrics.elapsed_ms.offset]
    assert sizes == mine


def test_params_defaults_match_reference_config():
    p = abi.Params()
    engine.lib().spg_params_default(C.byref(p))
    q = abi.default_params()
    for name, _ in abi.Params._fields_:
        assert getattr(p, name) == getattr(q, name), name


def test_abi_version():
    assert engine.lib().spg_abi_version() == 3


@pytest.mark.skipif(engine.device_available(), reason="checks the no-device refusal")
def test_refuses_without_device():
    db, _ = golden_small_db(True)
    with pytest.raises(engine.SpgError) as e:
        engine.GpContext(db)
    assert e.value.code == abi.SPG_E_NO_DEVICE
    with pytest.raises(engine.SpgError):
        engine.PoissonBackend(64, 64, 1.0, 1.0)


def test_host_fillers_match_reference():
    """spg_fillers_plan + spg_fillers_scatter (host C++) vs the reference's fillers."""
    db, g = golden_small_db(False)
    info = engine.initialize_fillers(db, 1.0, 1002)
    ref = g["filler_info"]
    assert info.count == int(ref[0])
    assert np.float32(info.width) == np.float32(ref[1]) and info.height == ref[2]
    assert info.whitespace_area == ref[3] and info.node_area_scaled == ref[4]
    assert info.total_filler_area == ref[5]
    assert np.array_equal(db.node_x[db.num_nodes:], g["filler_x"])
    assert np.array_equal(db.node_y[db.num_nodes:], g["filler_y"])
