"""BookShelf placement files <-> PlaceDB.

`read_bookshelf` is BookshelfReader::read (src/io/bookshelf_reader.cpp:433-463),
`read_placement` is BookshelfReader::readPlacement (src/io/bookshelf_reader.cpp:367-401) and
`write_pl` is BookshelfWriter::writePl (src/io/bookshelf_writer.cpp:16-37); all run in the engine
library's host code (spg_bookshelf_*, no device work). The returned PlaceDB carries the I/O
side arrays of the reference's PlaceDB (src/db/place_db.h:30-43) as attributes: node_names,
net_names (lists of str), node_orient (uint8 codes, ORIENTS order) and net_weight (float32).

`write_bookshelf` writes a whole design (.aux, .nodes, .nets, .wts, .pl, .scl) that the reader
reads back to the same arrays; the reference has no writer for the files other than .pl.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import abi
from .engine import SpgError, lib
from .placedb import F_FIXED, F_NI, PlaceDB

ORIENTS = ("N", "E", "S", "W", "FN", "FE", "FS", "FW")


def _bs_check(rc):
    if rc != 0:
        raise SpgError(rc, lib().spg_bookshelf_last_error().decode())


def _split_names(buf: np.ndarray, count: int) -> list:
    names = bytes(buf).split(b"\0")[:count]
    return [n.decode() for n in names]


def _join_names(names) -> np.ndarray:
    blob = b"".join(str(n).encode() + b"\0" for n in names)
    return np.frombuffer(blob or b"\0", np.uint8).copy()


def read_bookshelf(aux_path: str) -> PlaceDB:
    """Reads the design named by a .aux file. Nodes come back as [movable | fixed] with
    centre coordinates; macros (movable, taller than 1.5 row heights) carry F_MACRO."""
    L = lib()
    h = C.c_void_p()
    _bs_check(L.spg_bookshelf_read(os.fsencode(aux_path), C.byref(h)))
    try:
        cnt = (C.c_int64 * 7)()
        _bs_check(L.spg_bookshelf_counts(h, cnt))
        num_movable, num_nodes, num_pins, num_nets, num_rows, node_bytes, net_bytes = (int(c) for c in cnt)
        db = PlaceDB()
        db.name = os.path.splitext(os.path.basename(aux_path))[0]
        db.num_movable, db.num_nodes, db.num_fillers = num_movable, num_nodes, 0
        f32 = lambda n: np.zeros(n, np.float32)  # noqa: E731
        i32 = lambda n: np.zeros(n, np.int32)  # noqa: E731
        db.node_x, db.node_y, db.node_w, db.node_h = (f32(num_nodes) for _ in range(4))
        db.node_flags = np.zeros(num_nodes, np.uint8)
        db.node_orient = np.zeros(num_nodes, np.uint8)
        node_names = np.zeros(max(node_bytes, 1), np.uint8)
        _bs_check(L.spg_bookshelf_nodes(h, abi.fptr(db.node_x), abi.fptr(db.node_y), abi.fptr(db.node_w),
                                        abi.fptr(db.node_h), abi.u8ptr(db.node_flags),
                                        abi.u8ptr(db.node_orient), node_names.ctypes.data))
        db.pin_offset_x, db.pin_offset_y = f32(num_pins), f32(num_pins)
        db.pin2node, db.pin2net, db.flat_net2pin, db.flat_node2pin = (i32(num_pins) for _ in range(4))
        db.net2pin_start, db.node2pin_start = i32(num_nets + 1), i32(num_nodes + 1)
        _bs_check(L.spg_bookshelf_pins(h, abi.fptr(db.pin_offset_x), abi.fptr(db.pin_offset_y),
                                       abi.iptr(db.pin2node), abi.iptr(db.pin2net),
                                       abi.iptr(db.net2pin_start), abi.iptr(db.flat_net2pin),
                                       abi.iptr(db.node2pin_start), abi.iptr(db.flat_node2pin)))
        db.net_weight = f32(num_nets)
        net_names = np.zeros(max(net_bytes, 1), np.uint8)
        _bs_check(L.spg_bookshelf_nets(h, abi.fptr(db.net_weight), net_names.ctypes.data))
        db.row_ly, db.row_height, db.row_lx, db.row_step = (f32(num_rows) for _ in range(4))
        db.row_num_sites = i32(num_rows)
        _bs_check(L.spg_bookshelf_rows(h, abi.fptr(db.row_ly), abi.fptr(db.row_height), abi.fptr(db.row_lx),
                                       abi.fptr(db.row_step), abi.iptr(db.row_num_sites)))
    finally:
        L.spg_bookshelf_destroy(h)
    db.node_names = _split_names(node_names, num_nodes)
    db.net_names = _split_names(net_names, num_nets)
    db.compute_regions()
    return db


def write_pl(path: str, db: PlaceDB, x=None, y=None) -> None:
    """Lower-left corners of the design's nodes (fillers excluded) as a .pl, in node order.
    x, y default to the PlaceDB's centres; fixed nodes get " /FIXED"."""
    n = db.num_nodes
    x = np.ascontiguousarray(db.node_x[:n] if x is None else np.asarray(x)[:n], np.float32)
    y = np.ascontiguousarray(db.node_y[:n] if y is None else np.asarray(y)[:n], np.float32)
    w = np.ascontiguousarray(db.node_w[:n], np.float32)
    h = np.ascontiguousarray(db.node_h[:n], np.float32)
    flags = np.ascontiguousarray(db.node_flags[:n], np.uint8)
    names = getattr(db, "node_names", None) or [f"o{i}" for i in range(n)]
    orient = getattr(db, "node_orient", None)
    orient = None if orient is None else np.ascontiguousarray(orient[:n], np.uint8)
    blob = _join_names(names[:n])
    _bs_check(lib().spg_bookshelf_write_pl(os.fsencode(path), n, blob.ctypes.data, abi.fptr(x), abi.fptr(y),
                                           abi.fptr(w), abi.fptr(h), abi.u8ptr(flags),
                                           None if orient is None else abi.u8ptr(orient)))


def read_placement(path: str, db: PlaceDB) -> None:
    """Applies a .pl to a PlaceDB read by read_bookshelf, in place (BookshelfReader::readPlacement,
    src/io/bookshelf_reader.cpp:367-401): centres from the lower-left corners, orientations, and
    F_FIXED for "/FIXED" lines. Nodes keep their order, so a node fixed here may sit in the
    movable segment, as after the reference's call."""
    n = db.num_nodes
    for k in ("node_x", "node_y", "node_w", "node_h"):
        setattr(db, k, np.ascontiguousarray(getattr(db, k), np.float32))
    db.node_flags = np.ascontiguousarray(db.node_flags, np.uint8)
    if getattr(db, "node_orient", None) is None:
        db.node_orient = np.zeros(db.node_x.shape[0], np.uint8)
    db.node_orient = np.ascontiguousarray(db.node_orient, np.uint8)
    names = getattr(db, "node_names", None) or [f"o{i}" for i in range(n)]
    blob = _join_names(names[:n])
    _bs_check(lib().spg_bookshelf_apply_pl(os.fsencode(path), n, blob.ctypes.data, abi.fptr(db.node_w),
                                           abi.fptr(db.node_h), abi.fptr(db.node_x), abi.fptr(db.node_y),
                                           abi.u8ptr(db.node_flags), abi.u8ptr(db.node_orient)))


def _num(v) -> str:
    """Shortest text that reads back to the same float32."""
    v = float(np.float32(v))
    return str(int(v)) if v.is_integer() and abs(v) < 1e15 else repr(v)


def write_bookshelf(directory: str, design: str, db: PlaceDB) -> str:
    """Writes `design`.aux/.nodes/.nets/.wts/.pl/.scl under `directory` from a PlaceDB (fillers
    excluded) and returns the .aux path. Pins are written net by net in CSR order, so the reader
    returns the same pin numbering when the PlaceDB's pins are in net order."""
    os.makedirs(directory, exist_ok=True)
    n = db.num_nodes
    names = getattr(db, "node_names", None) or [f"o{i}" for i in range(n)]
    nets = getattr(db, "net_names", None) or [f"n{k}" for k in range(db.num_nets)]
    weight = getattr(db, "net_weight", None)
    p = lambda ext: os.path.join(directory, design + ext)  # noqa: E731

    with open(p(".aux"), "w") as f:
        f.write(f"RowBasedPlacement : {design}.nodes {design}.nets {design}.wts {design}.pl {design}.scl\n")

    fixed = (db.node_flags[:n] & F_FIXED) != 0
    with open(p(".nodes"), "w") as f:
        f.write(f"UCLA nodes 1.0\n\nNumNodes : {n}\nNumTerminals : {int(fixed.sum())}\n")
        for i in range(n):
            kind = ""
            if fixed[i]:
                kind = "\tterminal_NI" if db.node_flags[i] & F_NI else "\tterminal"
            f.write(f"\t{names[i]}\t{_num(db.node_w[i])}\t{_num(db.node_h[i])}{kind}\n")

    with open(p(".nets"), "w") as f:
        f.write(f"UCLA nets 1.0\n\nNumNets : {db.num_nets}\nNumPins : {db.num_pins}\n\n")
        for k in range(db.num_nets):
            a, b = int(db.net2pin_start[k]), int(db.net2pin_start[k + 1])
            f.write(f"NetDegree : {b - a}\t{nets[k]}\n")
            for q in db.flat_net2pin[a:b]:
                f.write(f"\t{names[db.pin2node[q]]}\tI : {_num(db.pin_offset_x[q])}\t{_num(db.pin_offset_y[q])}\n")

    with open(p(".wts"), "w") as f:
        f.write("UCLA wts 1.0\n\n")
        if weight is not None:
            for k in range(db.num_nets):
                if weight[k] != 1.0:
                    f.write(f"{nets[k]}\t{_num(weight[k])}\n")

    write_pl(p(".pl"), db)

    with open(p(".scl"), "w") as f:
        f.write(f"UCLA scl 1.0\n\nNumRows : {db.row_ly.shape[0]}\n\n")
        for r in range(db.row_ly.shape[0]):
            f.write("CoreRow Horizontal\n"
                    f"  Coordinate    :  {_num(db.row_ly[r])}\n"
                    f"  Height        :  {_num(db.row_height[r])}\n"
                    f"  Sitewidth     :  {_num(db.row_step[r])}\n"
                    f"  Sitespacing   :  {_num(db.row_step[r])}\n"
                    "  Siteorient    :  1\n  Sitesymmetry  :  1\n"
                    f"  SubrowOrigin  :  {_num(db.row_lx[r])}\tNumSites  :  {int(db.row_num_sites[r])}\n"
                    "End\n")
    return p(".aux")
