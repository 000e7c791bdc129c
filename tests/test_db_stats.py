"""The design summary (CPU) against the reference's own DbStats::compute and toString
(src/db/db_stats.cpp, compiled into oracle/_ref): every value exactly and the text byte for byte."""
import os

import pytest

from oracle import ref
from superplace_b200 import bookshelf, generator
from superplace_b200.stats import db_stats, summary_text

from .test_bookshelf import corner_design

needs_ref = pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")


def check(db):
    s = db_stats(db)
    v, hist, text = ref.db_stats(ref.RefDb(db))
    mine = [s.core_lx, s.core_ly, s.core_hx, s.core_hy, s.row_height, s.row_count, s.site_step, s.core_area,
            s.movable_area, s.fixed_area, s.fixed_area_in_core, s.total_row_area, s.max_net_degree, s.degree_over]
    assert mine == v
    assert list(s.degree_histogram) == hist
    assert summary_text(s) == text
    return s


@needs_ref
def test_generated_designs():
    s = check(generator.small_design(1002))
    assert s.node_count + s.fixed_count == s.object_count and sum(s.degree_count) + s.degree_over == s.net_count
    check(generator.mixed_design(5, n_cells=20_000, n_nets=21_000))


@needs_ref
def test_bookshelf_corner_design(tmp_path):
    os.makedirs(tmp_path / "c")
    db = bookshelf.read_bookshelf(corner_design(str(tmp_path / "c")))
    s = check(db)
    assert s.fixed_count == 4 and s.macro_count == 3 and s.degree_histogram[0] == 1
