"""BookShelf I/O parity (CPU): superplace_b200.bookshelf against the reference's own
BookshelfReader / BookshelfWriter (src/io/bookshelf_reader.cpp, src/io/bookshelf_writer.cpp),
built from its sources into oracle/_ref.

The designs are written here as text: a hand-made one that walks the format's corner cases
(comments, CRLF, tabs, glued "Key:value", a row without End, unnamed nets, terminal and
terminal_NI nodes, /FIXED in the .pl, names missing from the .pl, "12.000000" integers, a .wts
with unknown names, duplicate names, corners that fall half-way between two 6-decimal values) and seeded random ones with non-integer sizes, offsets
and positions. Every array must match the reference reader bit for bit, and the .pl writer's
output byte for byte. The round-trip checks restate test/test_roundtrip.cpp.
"""
import os

import numpy as np
import pytest

from oracle import ref
from superplace_b200 import bookshelf
from superplace_b200.engine import SpgError
from superplace_b200.placedb import F_FIXED, F_MACRO, F_NI

needs_ref = pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")

ARRAYS = ("node_x", "node_y", "node_w", "node_h", "node_flags", "node_orient", "pin_offset_x",
          "pin_offset_y", "pin2node", "pin2net", "net2pin_start", "flat_net2pin", "node2pin_start",
          "flat_node2pin", "net_weight", "row_ly", "row_height", "row_lx", "row_step", "row_num_sites")


def _write(d, name, text):
    with open(os.path.join(d, name), "w", newline="") as f:
        f.write(text)


CORNER = {
    "c.aux": "# design\nRowBasedPlacement :  c.nodes  c.nets c.wts c.pl   c.scl\n",
    "c.scl": (
        "UCLA scl 1.0\n# rows\n\nNumRows : 5\n"
        "CoreRow Horizontal\r\n  Coordinate : 0\r\n  Height : 12\r\n  Sitewidth : 1\r\n"
        "  Sitespacing : 1\r\n  SubrowOrigin : 0\tNumSites : 100\r\nEnd\r\n"
        "CoreRow Horizontal\n Coordinate :12\n Height : 12\n Sitewidth : 2\n Sitespacing : 0\n"
        " SubrowOrigin : 4 NumSites : 48.000000\nEnd\n"
        "CoreRow Horizontal\n\tCoordinate\t:\t24\n\tHeight\t:\t16\n\tSitewidth\t:\t1\n"
        "\tSubrowOrigin:2 NumSites:98\nEnd\n"
        "CoreRow Horizontal\n Coordinate : 40\n Height : 16\n Sitespacing : 0.5\n"
        " SubrowOrigin : 0.25 NumSites : 200\n"
        "End\nEnd\n"
        "CoreRow Horizontal\n Coordinate : 56\n Height : 12\n SubrowOrigin : 0 NumSites : 100\n"
    ),
    "c.nodes": (
        "UCLA nodes 1.0\n# comment\n\nNumNodes : 14\nNumTerminals : 3\n"
        "\ta0\t4\t12\n\ta1\t2.5\t12\n\tbig\t20\t40\n\tt0\t10\t10\tterminal\n"
        "\ta2 6 12.000000\n\tni\t0\t0\tterminal_NI\n\ta3\t3\t12\r\n"
        "\ta4\t8\t24\n\tt1\t5\t50\tterminal\n\tonly2\t5\n\ta5\t1e1\t12\n"
        "\ttall\t4\t18.5\n\ta6\t7.75\t12\tsomething\n\ta0\t9\t9\n"
    ),
    "c.nets": (
        "UCLA nets 1.0\n\nNumNets : 7\nNumPins : 20\n\n"
        "NetDegree : 3   n_first\n\ta0\tI : 1.5\t-2\n\tbig O : 0 0\n\tt0 B : -5 5\n"
        "NetDegree : 2\n\ta1 I : 0.25 0.125\n\ta2\n"
        "NetDegree:2 glued\n\ta3 I : 1\n\tni I : 0 0\n"
        "# inner comment\n"
        "NetDegree : 4 wide\n\ta4 I : 1 1\n\ta5 O : -1 -1\n\ttall I : 0.5 2\n\ta0 I : -1.25 3\n"
        "\tzzz I : 9 9\n"
        "NetDegree : 1 single\n\tt1 I : 0 -20\n"
        "NetDegree : 2 dup\n\ta6 : 2 2\n\ta0 I : 0 0\n"
        "NetDegree : 3 last\n\ta1\tI :\t0\t0\n\ta4 I : 2.0e-1 3\n\tt0 I : 1 1\n"
    ),
    "c.pl": (
        "UCLA pl 1.0\n\n"
        "a0\t10\t0\t: N\na1 20.5 12 : FS\nbig 40 12 : E\nt0\t60\t30\t: N /FIXED\n"
        "a2 0 0\nni 5 5 : N /FIXED_NI\na3 1 1 : W /FIXED\na4 30 24 :FN\n"
        "t1 70 0 : S\nunknown 1 2 : N\nshort 1\na5 12.0078125 36.0234375 : FW\ntall 3 3 : FE\n"
        "a1 21 12 : S\n"
    ),
    "c.wts": "UCLA wts 1.0\n\nwide 2.5\nnot_a_net 3\nsingle\nglued 0.5\nn1 4\n",
}


def corner_design(d):
    for k, v in CORNER.items():
        _write(d, k, v)
    return os.path.join(d, "c.aux")


def random_design(d, seed, n_nodes=600, n_nets=700, crlf=False, dyadic=False):
    """A seeded design with real-valued sizes, offsets and positions (with `dyadic`, sizes in
    quarters and positions in 64ths, which "%.6f" prints exactly)."""
    rng = np.random.default_rng(seed)
    eol = "\r\n" if crlf else "\n"
    heights = (9.0, 9.0, 12.0)
    rows = []
    y = 0.0
    for r in range(40):
        h = heights[r % 3]
        rows.append((y, h, float(rng.integers(0, 5)) * 0.5, float(rng.choice([1.0, 0.5, 2.0])),
                     int(rng.integers(50, 400))))
        y += h
    scl = ["UCLA scl 1.0", "", f"NumRows : {len(rows)}"]
    for ly, h, lx, st, ns in rows:
        scl += ["CoreRow Horizontal", f" Coordinate : {ly!r}", f" Height : {h!r}", f" Sitewidth : {st!r}",
                f" Sitespacing : {st!r}", f" SubrowOrigin : {lx!r}\tNumSites : {ns}", "End"]
    names = [f"o{i}" for i in range(n_nodes)]
    term = rng.random(n_nodes) < 0.08
    ni = term & (rng.random(n_nodes) < 0.3)
    w = np.round(rng.uniform(0.5, 30.0, n_nodes).astype(np.float32), 3)
    h = np.where(rng.random(n_nodes) < 0.1, rng.uniform(10, 60, n_nodes), 9.0).astype(np.float32)
    q = (lambda v, s: np.round(np.asarray(v) * s) / s) if dyadic else (lambda v, s: v)
    w, h = q(w, 4).astype(np.float32), q(h, 4).astype(np.float32)
    nodes = ["UCLA nodes 1.0", "", f"NumNodes : {n_nodes}", f"NumTerminals : {int(term.sum())}"]
    for i in range(n_nodes):
        kind = ("\tterminal_NI" if ni[i] else "\tterminal") if term[i] else ""
        nodes.append(f"\t{names[i]}\t{float(w[i])!r}\t{float(h[i])!r}{kind}")
    nets = ["UCLA nets 1.0", "", f"NumNets : {n_nets}"]
    for k in range(n_nets):
        deg = int(min(rng.geometric(0.35) + 1, 40))
        nets.append(f"NetDegree : {deg}" + (f"   net_{k}" if rng.random() < 0.9 else ""))
        for nd in rng.integers(0, n_nodes, deg):
            ox, oy = rng.normal(0, 3, 2).astype(np.float32)
            nets.append(f"\t{names[nd]}\t{rng.choice(['I', 'O', 'B'])} : {float(ox)!r}\t{float(oy)!r}")
    pl = ["UCLA pl 1.0", ""]
    for i in rng.permutation(n_nodes):
        if rng.random() < 0.03:
            continue  # stays at the origin
        o = bookshelf.ORIENTS[int(rng.integers(0, 8))]
        fx = " /FIXED" if (term[i] or rng.random() < 0.02) else ""
        pl.append(f"{names[i]}\t{float(np.float32(q(rng.uniform(0, 3000), 64)))!r}\t"
                  f"{float(np.float32(q(rng.uniform(0, 360), 64)))!r}\t: {o}{fx}")
    wts = ["UCLA wts 1.0", ""] + [f"net_{k}\t{float(np.float32(rng.uniform(0.5, 4)))!r}"
                                  for k in range(0, n_nets, 7)]
    aux = f"RowBasedPlacement : r.nodes r.nets r.wts r.pl r.scl"
    for name, lines in (("r.scl", scl), ("r.nodes", nodes), ("r.nets", nets), ("r.pl", pl), ("r.wts", wts),
                        ("r.aux", [aux])):
        _write(d, name, eol.join(lines) + eol)
    return os.path.join(d, "r.aux")


def assert_same_arrays(db, want):
    assert db.num_movable == want["num_movable"]
    assert db.num_nodes == want["num_nodes"]
    for k in ARRAYS:
        a, b = np.asarray(getattr(db, k)), want[k]
        assert a.dtype == b.dtype or a.dtype.itemsize == b.dtype.itemsize, k
        assert a.shape == b.shape, (k, a.shape, b.shape)
        assert np.array_equal(a.view(np.uint8), b.view(np.uint8)), k  # bit for bit
    assert db.node_names == want["node_names"]
    assert db.net_names == want["net_names"]
    assert db.core == pytest.approx(want["core"], abs=0)
    assert np.float32(db.row_height_mode) == np.float32(want["row_height_mode"])
    assert db.total_row_area == want["total_row_area"]


def design_cases(tmp_path):
    out = [("corner", corner_design(str(tmp_path / "corner")) if os.makedirs(tmp_path / "corner") is None else None)]
    for seed, crlf in ((1, False), (2, True), (3, False)):
        d = tmp_path / f"rand{seed}"
        os.makedirs(d)
        out.append((f"rand{seed}", random_design(str(d), seed, crlf=crlf)))
    return out


@needs_ref
def test_reader_matches_reference(tmp_path):
    for name, aux in design_cases(tmp_path):
        db = bookshelf.read_bookshelf(aux)
        want = ref.bookshelf_arrays(ref.bookshelf_read(aux))
        assert_same_arrays(db, want)


def test_corner_design_semantics(tmp_path):
    """What the corner design must read as, independent of the reference build."""
    os.makedirs(tmp_path / "c")
    db = bookshelf.read_bookshelf(corner_design(str(tmp_path / "c")))
    names = db.node_names
    assert db.num_nodes == 13 and names.count("a0") == 2  # "only2" is skipped, duplicates kept
    fixed = {names[i] for i in range(db.num_nodes) if db.node_flags[i] & F_FIXED}
    assert fixed == {"t0", "ni", "a3", "t1"}  # terminals plus /FIXED in the .pl
    assert names[db.num_movable:] == ["t0", "ni", "a3", "t1"]  # file order inside each segment
    i = names.index("ni")
    assert db.node_flags[i] & F_NI
    # row heights 12, 12, 16, 16, 12: mode 12, macros are movable nodes taller than 18
    macros = {names[i] for i in range(db.num_nodes) if db.node_flags[i] & F_MACRO}
    assert macros == {"big", "a4", "tall"}
    assert db.row_height_mode == 12.0 and db.row_ly.shape[0] == 5  # a last row without End counts
    assert list(db.row_step) == [1.0, 2.0, 1.0, 0.5, 1.0]
    # keys are matched on the first token, so "SubrowOrigin:2 ..." is not a SubrowOrigin line,
    # and a value glued to a lone ':' at the end of a line is not read (valueAfterColon,
    # src/io/bookshelf_reader.cpp:101-116)
    assert list(db.row_num_sites) == [100, 48, 0, 200, 100]
    assert list(db.row_ly) == [0.0, 0.0, 24.0, 40.0, 56.0] and list(db.row_lx) == [0.0, 4.0, 0.0, 0.25, 0.0]
    i = names.index("a1")  # the last .pl line for a node wins
    assert (db.node_x[i], db.node_y[i], db.node_orient[i]) == (22.25, 18.0, 2)  # S
    i = names.index("a4")  # ":FN" glued is no orientation
    assert db.node_orient[i] == 0
    i = names.index("a2")
    assert (db.node_x[i], db.node_y[i]) == (3.0, 6.0)
    # nets: the unnamed one is "n<index>"; "NetDegree:2 glued" is no NetDegree line, so it and
    # its pins fall past the previous net's degree and are skipped, as is the extra "zzz" pin
    assert db.net_names == ["n_first", "n1", "wide", "single", "dup", "last"]
    assert list(np.diff(db.net2pin_start)) == [3, 2, 4, 1, 2, 3]
    assert list(db.net_weight) == [1.0, 4.0, 2.5, 1.0, 1.0, 1.0]
    a0 = names.index("a0")  # the first of the duplicate names owns the pins
    assert set(db.pin2node[db.flat_node2pin[db.node2pin_start[a0]:db.node2pin_start[a0 + 1]]]) == {a0}
    assert db.node2pin_start[a0 + 1] - db.node2pin_start[a0] == 3


@needs_ref
def test_write_pl_matches_reference_bytes(tmp_path):
    for name, aux in design_cases(tmp_path):
        db = bookshelf.read_bookshelf(aux)
        mine, theirs = str(tmp_path / f"{name}.mine.pl"), str(tmp_path / f"{name}.ref.pl")
        bookshelf.write_pl(mine, db)
        ref.write_pl(ref.bookshelf_read(aux), theirs)
        assert open(mine, "rb").read() == open(theirs, "rb").read(), name


def test_pl_roundtrip(tmp_path):
    """test/test_roundtrip.cpp: write the .pl, read it back, positions and flags unchanged; two
    writes are byte-identical."""
    d = tmp_path / "rt"
    os.makedirs(d)
    aux = random_design(str(d), 7, dyadic=True)
    db = bookshelf.read_bookshelf(aux)
    bookshelf.write_pl(str(d / "r.pl"), db)
    back = bookshelf.read_bookshelf(aux)
    assert np.array_equal(back.node_x, db.node_x) and np.array_equal(back.node_y, db.node_y)
    assert np.array_equal(back.node_flags, db.node_flags)
    assert np.array_equal(back.node_orient, db.node_orient)
    bookshelf.write_pl(str(d / "again.pl"), back)
    assert open(d / "r.pl", "rb").read() == open(d / "again.pl", "rb").read()


def test_write_bookshelf_roundtrip(tmp_path):
    for name, aux in design_cases(tmp_path):
        db = bookshelf.read_bookshelf(aux)
        if name == "corner":
            continue  # duplicate node names do not survive a rewrite
        out = bookshelf.write_bookshelf(str(tmp_path / f"{name}_out"), "w", db)
        back = bookshelf.read_bookshelf(out)
        for k in ARRAYS:
            if k in ("node_x", "node_y"):
                continue  # the .pl holds 6 decimals
            assert np.array_equal(getattr(back, k), getattr(db, k)), (name, k)
        assert back.node_names == db.node_names and back.net_names == db.net_names
        assert np.allclose(back.node_x, db.node_x, atol=1e-3) and np.allclose(back.node_y, db.node_y, atol=1e-3)


ERRORS = {
    "no_scl": ({"c.aux": "RowBasedPlacement : c.nodes c.nets c.pl\n"}, "aux file missing required entries"),
    "missing_file": ({"c.aux": "RowBasedPlacement : c.nodes c.nets c.pl gone.scl\n"}, "cannot open"),
    "unknown_pin_node": ({"c.nets": "NetDegree : 2 x\n a0 I : 0 0\n nobody I : 0 0\n"},
                         "net references unknown node: nobody"),
    "bad_float": ({"c.nodes": "NumNodes : 1\n a0 x4 12\n"}, "bad float: x4"),
    "trailing_text": ({"c.nodes": "NumNodes : 1\n a0 4x 12\n"}, "net references unknown node: big"),
    "bad_count": ({"c.nodes": "NumNodes : many\n a0 4 12\n"}, "bad integer: many"),
    "no_rows": ({"c.scl": "NumRows : 0\n"}, "no CoreRow found in"),
    "bad_degree": ({"c.nets": "NetDegree\n"}, "malformed NetDegree line"),
}


@pytest.mark.parametrize("case", sorted(ERRORS))
def test_errors_match_reference(tmp_path, case):
    files, msg = ERRORS[case]
    d = str(tmp_path)
    corner_design(d)
    for k, v in files.items():
        _write(d, k, v)
    aux = os.path.join(d, "c.aux")
    with pytest.raises(SpgError) as e:
        bookshelf.read_bookshelf(aux)
    assert msg in str(e.value)
    if ref.available():
        with pytest.raises(RuntimeError) as r:
            ref.bookshelf_read(aux)
        assert str(e.value).split("] ", 1)[1] == str(r.value)


@pytest.fixture(scope="module")
def large_bookshelf(tmp_path_factory):
    """The 211k-cell synthetic design written as BookShelf (about 59 MB): every file above the
    reader's piece size, so it is parsed in pieces on several threads."""
    from superplace_b200 import generator
    d = tmp_path_factory.mktemp("large")
    return bookshelf.write_bookshelf(str(d), "large", generator.large_design(1002))


@needs_ref
def test_reader_matches_reference_full_size(large_bookshelf, tmp_path):
    db = bookshelf.read_bookshelf(large_bookshelf)
    r = ref.bookshelf_read(large_bookshelf)
    assert_same_arrays(db, ref.bookshelf_arrays(r))
    mine, theirs = str(tmp_path / "mine.pl"), str(tmp_path / "ref.pl")
    bookshelf.write_pl(mine, db)
    ref.write_pl(r, theirs)
    assert open(mine, "rb").read() == open(theirs, "rb").read()


def test_first_error_across_pieces(large_bookshelf, tmp_path):
    """Two bad pin lines far apart in the .nets file: the one earlier in the file is reported,
    whichever piece reaches its line first."""
    src = os.path.dirname(large_bookshelf)
    for ext in (".aux", ".nodes", ".pl", ".scl", ".wts"):
        with open(os.path.join(src, "large" + ext), "rb") as f:
            data = f.read()
        with open(tmp_path / ("large" + ext), "wb") as f:
            f.write(data)
    lines = open(os.path.join(src, "large.nets")).read().split("\n")
    at = (int(len(lines) * 0.3), int(len(lines) * 0.8))
    for i, bad in zip(at, ("ghost_early", "ghost_late")):
        while not lines[i].startswith("\t"):
            i += 1
        lines[i] = f"\t{bad}\tI : 0 0"
    with open(tmp_path / "large.nets", "w") as f:
        f.write("\n".join(lines))
    aux = str(tmp_path / "large.aux")
    with pytest.raises(SpgError, match="unknown node: ghost_early"):
        bookshelf.read_bookshelf(aux)
    if ref.available():
        with pytest.raises(RuntimeError, match="unknown node: ghost_early"):
            ref.bookshelf_read(aux)


@needs_ref
def test_read_placement_matches_reference(tmp_path):
    """A second .pl over a design already read (main.cpp's --pl): positions, orientations and
    /FIXED flags as the reference's readPlacement leaves them, nodes not reordered."""
    for name, aux in design_cases(tmp_path):
        db = bookshelf.read_bookshelf(aux)
        r = ref.bookshelf_read(aux)
        rng = np.random.default_rng(len(name))
        lines = ["UCLA pl 1.0", "# second placement", ""]
        for i in rng.permutation(db.num_nodes)[: db.num_nodes * 3 // 4]:
            fx = " /FIXED" if rng.random() < 0.1 else ""
            o = f" : {bookshelf.ORIENTS[int(rng.integers(0, 8))]}" if rng.random() < 0.8 else ""
            lines.append(f"{db.node_names[i]}\t{rng.uniform(-5, 500):.4f}\t{rng.uniform(0, 90):.3f}{o}{fx}")
        lines += ["nobody 1 2 : N", f"{db.node_names[0]} 7 8 : FE"]
        pl = str(tmp_path / f"{name}.second.pl")
        _write(str(tmp_path), f"{name}.second.pl", "\n".join(lines) + "\n")
        bookshelf.read_placement(pl, db)
        ref.read_placement(r, pl)
        want = ref.bookshelf_arrays(r)
        for k in ("node_x", "node_y", "node_flags", "node_orient"):
            assert np.array_equal(getattr(db, k).view(np.uint8), want[k].view(np.uint8)), (name, k)
        assert db.node_orient[0] == 5
