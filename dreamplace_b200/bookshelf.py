"""Bookshelf (ISPD 2005 style) writer and reader for the synthetic designs.

Lets the reference's own ``Placer.py`` place exactly the designs this package
generates (on machines where the reference's ``place_io`` parser builds), and
lets this package read such files back.  Files follow the layout the
reference's parser accepts and its writer emits
(dreamplace/ops/place_io/src/BookshelfWriter.cpp): ``.aux`` listing
``.nodes .nets .wts .pl .scl``.  Conventions:

* pin offsets in ``.nets`` are relative to the node centre (Bookshelf); the
  in-memory offsets are relative to the lower-left corner;
* fixed macros are ``terminal`` nodes with ``/FIXED`` in ``.pl``; fillers are
  not written (the placer inserts them, dreamplace/PlaceDB.py:919-950);
* rows cover the die at the design's row height with unit sites.
"""
import os

import numpy as np

from . import synthetic


def _names(design):
    m, t = design.num_movable_nodes, design.num_terminals
    return ["o%d" % i for i in range(m)] + ["p%d" % i for i in range(t)]


def write_bookshelf(design, directory, name=None, positions=None):
    """Writes ``<name>.aux`` and its five files; returns the .aux path."""
    d = design
    name = name or d.name
    os.makedirs(directory, exist_ok=True)
    path = lambda ext: os.path.join(directory, name + ext)  # noqa: E731
    names = _names(d)
    m, nphys = d.num_movable_nodes, d.num_physical_nodes
    if positions is None:
        positions = d.initial_positions()
    n = d.num_nodes
    with open(path(".aux"), "w") as f:
        f.write("RowBasedPlacement : %s.nodes %s.nets %s.wts %s.pl %s.scl\n" % ((name,) * 5))
    with open(path(".nodes"), "w") as f:
        f.write("UCLA nodes 1.0\n\nNumNodes : %d\nNumTerminals : %d\n" % (nphys, d.num_terminals))
        for i in range(nphys):
            f.write("\t%s\t%.6g\t%.6g%s\n" % (names[i], d.node_size_x[i], d.node_size_y[i],
                                              "\tterminal" if i >= m else ""))
    with open(path(".nets"), "w") as f:
        f.write("UCLA nets 1.0\n\nNumNets : %d\nNumPins : %d\n" % (d.num_nets, d.num_pins))
        start = d.flat_net2pin_start_map
        for e in range(d.num_nets):
            f.write("NetDegree : %d n%d\n" % (start[e + 1] - start[e], e))
            for j in range(start[e], start[e + 1]):
                p = d.flat_net2pin_map[j]
                node = d.pin2node_map[p]
                xo = float(d.pin_offset_x[p]) - float(d.node_size_x[node]) / 2
                yo = float(d.pin_offset_y[p]) - float(d.node_size_y[node]) / 2
                f.write("\t%s\tI : %.6f\t%.6f\n" % (names[node], xo, yo))
    with open(path(".wts"), "w") as f:
        f.write("UCLA wts 1.0\n\n")
        for e in range(d.num_nets):
            if d.net_weights[e] != 1.0:
                f.write("\tn%d\t%.6g\n" % (e, d.net_weights[e]))
    with open(path(".pl"), "w") as f:
        f.write("UCLA pl 1.0\n\n")
        for i in range(nphys):
            f.write("%s\t%.6f\t%.6f\t: N%s\n" % (names[i], positions[i], positions[n + i],
                                                 "\t/FIXED" if i >= m else ""))
    rows = int(round((d.yh - d.yl) / d.row_height))
    with open(path(".scl"), "w") as f:
        f.write("UCLA scl 1.0\n\nNumRows : %d\n\n" % rows)
        for r in range(rows):
            f.write("CoreRow Horizontal\n  Coordinate :\t%d\n  Height :\t%d\n  Sitewidth :\t1\n"
                    "  Sitespacing :\t1\n  Siteorient :\t1\n  Sitesymmetry :\t1\n"
                    "  SubrowOrigin :\t%d\tNumSites :\t%d\nEnd\n"
                    % (d.yl + r * d.row_height, d.row_height, d.xl, int(d.xh - d.xl)))
    return path(".aux")


def _tokens(path):
    with open(path) as f:
        for line in f:
            line = line.split("#", 1)[0].strip()
            if line:
                yield line


def read_bookshelf(aux_path, num_bins=None, target_density=1.0):
    """Reads a Bookshelf design into a synthetic.Design (fillers and bins derived
    as the reference's PlaceDB does)."""
    directory = os.path.dirname(aux_path)
    files = open(aux_path).read().split(":", 1)[1].split()
    get = lambda ext: os.path.join(directory, next(x for x in files if x.endswith(ext)))  # noqa: E731
    names, sx, sy, term = [], [], [], []
    for line in _tokens(get(".nodes")):
        if line.startswith(("UCLA", "NumNodes", "NumTerminals")):
            continue
        p = line.split()
        names.append(p[0])
        sx.append(float(p[1]))
        sy.append(float(p[2]))
        term.append(len(p) > 3 and p[3].startswith("terminal"))
    term = np.array(term)
    order = np.r_[np.where(~term)[0], np.where(term)[0]]  # movable first, then terminals
    index = {names[i]: k for k, i in enumerate(order)}
    sx = np.array(sx, np.float32)[order]
    sy = np.array(sy, np.float32)[order]
    m = int((~term).sum())
    nphys = len(names)
    degrees, pin_node, offx, offy = [], [], [], []
    for line in _tokens(get(".nets")):
        if line.startswith(("UCLA", "NumNets", "NumPins")):
            continue
        if line.startswith("NetDegree"):
            degrees.append(0)
            continue
        p = line.replace(":", " ").split()
        node = index[p[0]]
        pin_node.append(node)
        offx.append(float(p[2]) + sx[node] / 2)
        offy.append(float(p[3]) + sy[node] / 2)
        degrees[-1] += 1
    starts = np.zeros(len(degrees) + 1, np.int64)
    np.cumsum(degrees, out=starts[1:])
    net_start = np.array(starts, np.int64)
    num_nets = len(net_start) - 1
    pin2node = np.array(pin_node, np.int32)
    px = np.zeros(nphys, np.float32)
    py = np.zeros(nphys, np.float32)
    for line in _tokens(get(".pl")):
        if line.startswith("UCLA"):
            continue
        p = line.split()
        k = index[p[0]]
        px[k], py[k] = float(p[1]), float(p[2])
    weights = np.ones(num_nets, np.float32)
    if any(x.endswith(".wts") for x in files):
        for line in _tokens(get(".wts")):
            if line.startswith("UCLA"):
                continue
            p = line.split()
            if p[0].startswith("n") and p[0][1:].isdigit():
                weights[int(p[0][1:])] = float(p[1])
    rows = []
    cur = {}
    for line in _tokens(get(".scl")):
        if line.startswith("Coordinate"):
            cur["y"] = float(line.split(":")[1])
        elif line.startswith("Height"):
            cur["h"] = float(line.split(":")[1])
        elif line.startswith("SubrowOrigin"):
            q = line.replace(":", " ").split()
            cur["x"], cur["n"] = float(q[1]), int(q[3])
        elif line.startswith("End"):
            rows.append(cur)
            cur = {}
    xl = min(r["x"] for r in rows)
    xh = max(r["x"] + r["n"] for r in rows)
    yl = min(r["y"] for r in rows)
    yh = max(r["y"] + r["h"] for r in rows)
    rh = rows[0]["h"]
    net_of_pin = np.repeat(np.arange(num_nets, dtype=np.int32), np.diff(net_start))
    d = synthetic._finish_from_arrays(
        os.path.splitext(os.path.basename(aux_path))[0], xl, yl, xh, yh, rh, sx[:m], sy[:m], px[m:], py[m:],
        sx[m:], sy[m:], pin2node, net_of_pin, net_start.astype(np.int32), np.array(offx, np.float32),
        np.array(offy, np.float32), weights, num_bins or 128, target_density)
    d.node_x[:m] = px[:m]
    d.node_y[:m] = py[:m]
    return d
