"""The pipeline of superplace_b200.flow (src/main.cpp's parse, init, gp, lg and the .pl write):
on CPU without the GP stage, on the GPU with it. The lg stage is the reference's own
legalizeCells (oracle/_ref), passed in as the flow's cell legaliser, as the reference's
LegalizeStage runs it after GP."""
import os

import numpy as np
import pytest

from oracle import ref
from superplace_b200 import bookshelf, flow, generator, qp

from .checks import ref_legalize_cells


@pytest.fixture
def small_aux(tmp_path):
    return bookshelf.write_bookshelf(str(tmp_path), "small", generator.small_design(1002))


def test_flow_without_gp(small_aux, tmp_path):
    out = str(tmp_path / "out.pl")
    db, rep = flow.place(small_aux, out_pl=out, stages=("parse", "init", "lg", "write"),
                         qp_params=qp.default_params(device=0), legalize_cells=ref_legalize_cells)
    names = [s["stage"] for s in rep["stages"]]
    assert names == ["parse", "init", "lg", "write"]
    lg = rep["stages"][2]
    assert lg["failed"] == 0 and lg["selfcheck_overlaps"] == 0 and lg["selfcheck_off_site"] == 0
    assert rep["stages"][1]["hpwl"] < rep["stages"][0]["hpwl"]  # QP pulls the nets in
    again = str(tmp_path / "again.pl")
    bookshelf.write_pl(again, db)
    assert open(out, "rb").read() == open(again, "rb").read()
    back = bookshelf.read_bookshelf(os.path.splitext(small_aux)[0] + ".aux")
    bookshelf.read_placement(out, back)
    assert np.array_equal(back.node_x, db.node_x[: db.num_nodes])


@pytest.mark.skipif(not os.path.exists(ref.CHECK_PATH), reason="oracle/_ref/superplace-check not built")
def test_flow_output_passes_the_reference_checker(small_aux, tmp_path):
    """The reference's own legality checker (tools/check/main.cpp) passes the legalised .pl
    and fails the overlapping start; its HPWL agrees with ours."""
    out = str(tmp_path / "out.pl")
    db, rep = flow.place(small_aux, out_pl=out, stages=("parse", "init", "lg", "write"),
                         qp_params=qp.default_params(device=0), legalize_cells=ref_legalize_cells)
    rc, text = ref.check_placement(small_aux, out)
    assert rc == 0 and "Result:         PASS" in text, text
    hpwl = float(text.split("HPWL:")[1].split()[0])
    assert hpwl == pytest.approx(rep["stages"][-1]["hpwl"], rel=1e-6)
    rc, text = ref.check_placement(small_aux)  # the design's own, overlapping .pl
    assert rc == 1 and "Result:         FAIL" in text


@pytest.mark.gpu
def test_flow_with_gp(small_aux, tmp_path):
    from superplace_b200 import abi
    db, rep = flow.place(small_aux, out_pl=str(tmp_path / "out.pl"), legalize_cells=ref_legalize_cells,
                         params=abi.default_params(gp_bin_dim=64))  # split-BF16 needs 128-multiples
    st = {s["stage"]: s for s in rep["stages"]}
    assert "stopped" not in rep and list(st) == ["parse", "init", "gp", "lg", "write"]
    assert st["init"]["device"] == 1
    assert st["gp"]["overflow"] <= 0.10 and st["gp"]["iterations"] > 0
    assert st["lg"]["failed"] == 0 and st["lg"]["selfcheck_overlaps"] == 0
    assert st["lg"]["hpwl"] < 1.2 * st["gp"]["hpwl"]
    if os.path.exists(ref.CHECK_PATH):
        rc, text = ref.check_placement(small_aux, str(tmp_path / "out.pl"))
        assert rc == 0, text
