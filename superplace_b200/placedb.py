"""Host-side PlaceDB: the reference's SoA + CSR layout (src/db/place_db.h:24-113) in numpy.

Nodes are kept in the reference's segment order [movable | fixed | filler]; coordinates
are node centres. `finalize_csr` and `compute_regions` restate PlaceDB::finalizeCSR
(src/db/place_db.cpp:67-95) and PlaceDB::computeRegions (src/db/place_db.cpp:97-127).
`view()` exposes the arrays as the C ABI's spg_db_view without copying.
"""
from __future__ import annotations

import numpy as np

from . import abi

F_MACRO, F_FIXED, F_FILLER, F_NI = abi.F_MACRO, abi.F_FIXED, abi.F_FILLER, abi.F_NI


class PlaceDB:
    def __init__(self):
        self.node_x = np.zeros(0, np.float32)
        self.node_y = np.zeros(0, np.float32)
        self.node_w = np.zeros(0, np.float32)
        self.node_h = np.zeros(0, np.float32)
        self.node_flags = np.zeros(0, np.uint8)
        self.pin_offset_x = np.zeros(0, np.float32)
        self.pin_offset_y = np.zeros(0, np.float32)
        self.pin2node = np.zeros(0, np.int32)
        self.pin2net = np.zeros(0, np.int32)
        self.net2pin_start = np.zeros(1, np.int32)
        self.flat_net2pin = np.zeros(0, np.int32)
        self.node2pin_start = np.zeros(1, np.int32)
        self.flat_node2pin = np.zeros(0, np.int32)
        self.row_ly = np.zeros(0, np.float32)
        self.row_height = np.zeros(0, np.float32)
        self.row_lx = np.zeros(0, np.float32)
        self.row_step = np.zeros(0, np.float32)
        self.row_num_sites = np.zeros(0, np.int32)
        self.num_movable = 0
        self.num_nodes = 0
        self.num_fillers = 0
        self.core = (0.0, 0.0, 0.0, 0.0)
        self.row_height_mode = 0.0
        self.total_row_area = 0.0
        self.name = "db"

    # ---------------------------------------------------------------- sizes
    @property
    def total_nodes(self) -> int:
        return self.num_nodes + self.num_fillers

    @property
    def num_pins(self) -> int:
        return int(self.pin2node.shape[0])

    @property
    def num_nets(self) -> int:
        return int(self.net2pin_start.shape[0] - 1)

    # ---------------------------------------------------------------- build
    def finalize_csr(self, pin_net: np.ndarray, num_nets: int) -> None:
        """Two-way CSR by counting sort; pins keep ascending index order inside each
        net and node (src/db/place_db.cpp:67-95)."""
        pin_net = np.asarray(pin_net, np.int32)
        self.pin2net = pin_net.copy()
        counts = np.bincount(pin_net, minlength=num_nets)
        self.net2pin_start = np.concatenate([[0], np.cumsum(counts)]).astype(np.int32)
        self.flat_net2pin = np.argsort(pin_net, kind="stable").astype(np.int32)
        n = self.num_nodes
        counts = np.bincount(self.pin2node, minlength=n)[:n] if n else np.zeros(0, np.int64)
        self.node2pin_start = np.concatenate([[0], np.cumsum(counts)]).astype(np.int32)
        self.flat_node2pin = np.argsort(self.pin2node, kind="stable").astype(np.int32)

    def compute_regions(self) -> None:
        """coreRegion = bounding box of all rows, rowHeight = most frequent row height
        (smallest on ties), totalRowArea in double (src/db/place_db.cpp:97-127)."""
        if self.row_ly.size == 0:
            self.core = (0.0, 0.0, 0.0, 0.0)
            self.row_height_mode = 0.0
            self.total_row_area = 0.0
            return
        hs, cnt = np.unique(self.row_height, return_counts=True)
        self.row_height_mode = float(hs[int(np.argmax(cnt))])
        hx = (self.row_lx + self.row_step * self.row_num_sites.astype(np.float32)).astype(np.float32)
        hy = (self.row_ly + self.row_height).astype(np.float32)
        self.core = (float(self.row_lx.min()), float(self.row_ly.min()),
                     float(hx.max()), float(hy.max()))
        widths = (hx - self.row_lx).astype(np.float64)
        self.total_row_area = float(np.sum(widths * self.row_height.astype(np.float64)))

    def extend_node2pin(self) -> None:
        """Fillers own no pins: extend node2pin_start to total+1 (src/gp/filler.cpp:130)."""
        need = self.total_nodes + 1
        if self.node2pin_start.shape[0] < need:
            pad = np.full(need - self.node2pin_start.shape[0], self.num_pins, np.int32)
            self.node2pin_start = np.concatenate([self.node2pin_start, pad]).astype(np.int32)
        elif self.node2pin_start.shape[0] > need:
            self.node2pin_start = self.node2pin_start[:need].copy()

    def set_fillers(self, count: int, width: float, height: float, x, y) -> None:
        """Replace the filler segment with `count` fillers of one size."""
        keep = self.num_nodes
        self.node_x = np.concatenate([self.node_x[:keep], np.asarray(x, np.float32)])
        self.node_y = np.concatenate([self.node_y[:keep], np.asarray(y, np.float32)])
        self.node_w = np.concatenate([self.node_w[:keep], np.full(count, width, np.float32)])
        self.node_h = np.concatenate([self.node_h[:keep], np.full(count, height, np.float32)])
        self.node_flags = np.concatenate([self.node_flags[:keep],
                                          np.full(count, F_FILLER, np.uint8)])
        self.num_fillers = int(count)
        self.extend_node2pin()

    def copy(self) -> "PlaceDB":
        o = PlaceDB()
        for k, v in self.__dict__.items():
            setattr(o, k, v.copy() if isinstance(v, np.ndarray) else v)
        return o

    # ---------------------------------------------------------------- queries
    def pin_xy(self):
        px = self.node_x[self.pin2node] + self.pin_offset_x
        py = self.node_y[self.pin2node] + self.pin_offset_y
        return px.astype(np.float32), py.astype(np.float32)

    def node_degree(self) -> np.ndarray:
        return np.diff(self.node2pin_start).astype(np.int32)

    # ---------------------------------------------------------------- ABI
    def _contig(self):
        for k in ("node_x", "node_y", "node_w", "node_h", "pin_offset_x", "pin_offset_y",
                  "row_ly", "row_height", "row_lx", "row_step"):
            setattr(self, k, np.ascontiguousarray(getattr(self, k), np.float32))
        for k in ("pin2node", "pin2net", "net2pin_start", "flat_net2pin", "node2pin_start",
                  "flat_node2pin", "row_num_sites"):
            setattr(self, k, np.ascontiguousarray(getattr(self, k), np.int32))
        self.node_flags = np.ascontiguousarray(self.node_flags, np.uint8)

    def view(self) -> abi.DbView:
        """spg_db_view over this object's arrays (valid while the arrays live)."""
        self._contig()
        self.extend_node2pin()
        v = abi.DbView()
        v.num_movable, v.num_nodes, v.num_fillers = self.num_movable, self.num_nodes, self.num_fillers
        v.node_x, v.node_y = abi.fptr(self.node_x), abi.fptr(self.node_y)
        v.node_w, v.node_h = abi.fptr(self.node_w), abi.fptr(self.node_h)
        v.node_flags = abi.u8ptr(self.node_flags)
        v.num_pins = self.num_pins
        v.pin_offset_x, v.pin_offset_y = abi.fptr(self.pin_offset_x), abi.fptr(self.pin_offset_y)
        v.pin2node, v.pin2net = abi.iptr(self.pin2node), abi.iptr(self.pin2net)
        v.num_nets = self.num_nets
        v.net2pin_start, v.flat_net2pin = abi.iptr(self.net2pin_start), abi.iptr(self.flat_net2pin)
        v.node2pin_start, v.flat_node2pin = abi.iptr(self.node2pin_start), abi.iptr(self.flat_node2pin)
        v.num_rows = int(self.row_ly.shape[0])
        v.row_ly, v.row_height = abi.fptr(self.row_ly), abi.fptr(self.row_height)
        v.row_lx, v.row_step = abi.fptr(self.row_lx), abi.fptr(self.row_step)
        v.row_num_sites = abi.iptr(self.row_num_sites)
        v.core_lx, v.core_ly, v.core_hx, v.core_hy = self.core
        v.row_height_mode = self.row_height_mode
        v.total_row_area = self.total_row_area
        v._keep = self  # keep the arrays alive with the view
        return v


def make_db(nodes, rows, nets=(), pin_offsets=None, name="db") -> PlaceDB:
    """Small-fixture builder in the style of the reference tests' makeDb helpers
    (test/test_density.cpp:24-54, test/test_wirelength.cpp:19-57).

    nodes: iterable of (cx, cy, w, h, flags); they are placed in segment order
           [movable | fixed | filler] preserving the given order inside each segment.
    rows:  iterable of (ly, height, lx, step, num_sites).
    nets:  iterable of node-index lists (indices into the reordered node list).
    pin_offsets: optional list of (ox, oy) per pin in net order.
    """
    nodes = list(nodes)

    def cls(f):
        f = int(f)
        return 2 if f & F_FILLER else (1 if f & F_FIXED else 0)

    order = [i for p in range(3) for i, n in enumerate(nodes) if cls(n[4]) == p]
    db = PlaceDB()
    db.name = name
    arr = np.array([nodes[i] for i in order], np.float64).reshape(-1, 5)
    db.node_x = arr[:, 0].astype(np.float32)
    db.node_y = arr[:, 1].astype(np.float32)
    db.node_w = arr[:, 2].astype(np.float32)
    db.node_h = arr[:, 3].astype(np.float32)
    db.node_flags = arr[:, 4].astype(np.uint8)
    classes = [cls(nodes[i][4]) for i in order]
    db.num_movable = classes.count(0)
    db.num_nodes = db.num_movable + classes.count(1)
    db.num_fillers = classes.count(2)
    pin2node, pin_net = [], []
    for k, net in enumerate(nets):
        for nd in net:
            pin2node.append(nd)
            pin_net.append(k)
    db.pin2node = np.array(pin2node, np.int32)
    if pin_offsets is None:
        db.pin_offset_x = np.zeros(len(pin2node), np.float32)
        db.pin_offset_y = np.zeros(len(pin2node), np.float32)
    else:
        po = np.array(pin_offsets, np.float32).reshape(-1, 2)
        db.pin_offset_x, db.pin_offset_y = po[:, 0].copy(), po[:, 1].copy()
    db.finalize_csr(np.array(pin_net, np.int32), len(list(nets)))
    r = np.array(list(rows), np.float64).reshape(-1, 5)
    db.row_ly = r[:, 0].astype(np.float32)
    db.row_height = r[:, 1].astype(np.float32)
    db.row_lx = r[:, 2].astype(np.float32)
    db.row_step = r[:, 3].astype(np.float32)
    db.row_num_sites = r[:, 4].astype(np.int32)
    db.compute_regions()
    db.extend_node2pin()
    return db
