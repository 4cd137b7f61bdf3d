"""Bookshelf writer and reader: a synthetic design survives write + read; the
reader gives on the reference's place_io unit-test design what the reference's
own parser gives; the writer's lines have the reference's Bookshelf shapes."""
import re

import numpy as np

from dreamplace_b200 import bookshelf, synthetic


def test_round_trip(tmp_path):
    d = synthetic.cells_10k()
    aux = bookshelf.write_bookshelf(d, str(tmp_path))
    r = bookshelf.read_bookshelf(aux, num_bins=d.num_bins_x)
    assert (r.num_movable_nodes, r.num_terminals, r.num_nets, r.num_pins) == \
        (d.num_movable_nodes, d.num_terminals, d.num_nets, d.num_pins)
    assert (r.xl, r.yl, r.xh, r.yh) == (d.xl, d.yl, d.xh, d.yh)
    np.testing.assert_array_equal(r.node_size_x[:d.num_physical_nodes], d.node_size_x[:d.num_physical_nodes])
    np.testing.assert_array_equal(r.pin2node_map, d.pin2node_map)
    np.testing.assert_array_equal(r.flat_net2pin_start_map, d.flat_net2pin_start_map)
    np.testing.assert_allclose(r.pin_offset_x, d.pin_offset_x, atol=1e-5)
    np.testing.assert_allclose(r.pin_offset_y, d.pin_offset_y, atol=1e-5)
    np.testing.assert_allclose(r.node_x[d.num_movable_nodes:], d.node_x[d.num_movable_nodes:])
    assert r.num_filler_nodes == d.num_filler_nodes and r.target_density == d.target_density


def _write_case(g, directory):
    for ext in ("aux", "nodes", "nets", "pl", "scl"):
        (directory / ("simple." + ext)).write_text(str(g["text_" + ext]))
    return str(directory / "simple.aux")


def _nets_by_name(names, start, flat, pin2node, offx, offy):
    """net name -> sorted (node, offset x, offset y) of its pins"""
    out = {}
    for e, name in enumerate(names):
        pins = [flat[j] for j in range(int(start[e]), int(start[e + 1]))]
        out[str(name)] = sorted((int(pin2node[p]), float(offx[p]), float(offy[p])) for p in pins)
    return out


def test_reader_matches_reference_place_io(golden, tmp_path):
    """The reference's place_io unit-test design (10 nodes, 2 terminals, 8
    nets, 26 pins; unittest/ops/place_io_unittest) read by this package gives
    what the reference's parser gives (simple.golden): node order (movable in
    file order, then terminals), sizes, fixed positions, pin offsets relative
    to the lower-left corner, each net's pins, and the rows' bounding box."""
    g = golden("bookshelf_simple.npz")
    r = bookshelf.read_bookshelf(_write_case(g, tmp_path))
    n = int(g["num_nodes"])
    assert (r.num_physical_nodes, r.num_terminals) == (n, int(g["num_terminals"]))
    assert (r.num_nets, r.num_pins) == (len(g["net_names"]), len(g["pin2node_map"]))
    np.testing.assert_array_equal(r.node_size_x[:n], g["node_size_x"])
    np.testing.assert_array_equal(r.node_size_y[:n], g["node_size_y"])
    m = r.num_movable_nodes
    np.testing.assert_array_equal(r.node_x[m:n], g["node_x"][m:n])
    np.testing.assert_array_equal(r.node_y[m:n], g["node_y"][m:n])
    assert (r.xl, r.yl, r.xh, r.yh) == (g["xl"], g["yl"], g["xh"], g["yh"])
    assert r.row_height == g["row_height"]
    # nets keep the file's order here and the parser's map order there: compare by name
    file_names = [line.split()[-1] for line in str(g["text_nets"]).splitlines() if line.startswith("NetDegree")]
    ours = _nets_by_name(file_names, r.flat_net2pin_start_map, r.flat_net2pin_map, r.pin2node_map,
                         r.pin_offset_x, r.pin_offset_y)
    ref = _nets_by_name(g["net_names"], g["flat_net2pin_start_map"], g["flat_net2pin_map"].astype(int),
                        g["pin2node_map"], g["pin_offset_x"], g["pin_offset_y"])
    assert ours == ref
    assert int(np.sum(r.pin2node_map < m)) == int(g["num_movable_pins"])


# line shapes of the reference's Bookshelf files (its writer,
# dreamplace/ops/place_io/src/BookshelfWriter.cpp:53-232, and its unit-test
# design), after comments and blank lines are dropped
_NUM = r"[-+]?\d+(\.\d*)?([eE][-+]?\d+)?"
_GRAMMAR = {
    "nodes": [r"UCLA nodes 1\.0", r"NumNodes\s*:\s*\d+", r"NumTerminals\s*:\s*\d+",
              r"\S+\s+%s\s+%s(\s+terminal(_NI)?)?" % (_NUM, _NUM)],
    "nets": [r"UCLA nets 1\.0", r"NumNets\s*:\s*\d+", r"NumPins\s*:\s*\d+", r"NetDegree\s*:\s*\d+\s+\S+",
             r"\S+\s+[IOB]\s*:\s*%s\s+%s" % (_NUM, _NUM)],
    "pl": [r"UCLA pl 1\.0", r"\S+\s+%s\s+%s\s*:\s*N(\s+/(FIXED|Fixed)(_NI)?)?" % (_NUM, _NUM)],
    "scl": [r"UCLA scl 1\.0", r"NumRows\s*:\s*\d+", r"CoreRow Horizontal", r"Coordinate\s*:\s*\d+",
            r"Height\s*:\s*\d+", r"Sitewidth\s*:\s*\d+", r"Sitespacing\s*:\s*\d+", r"Siteorient\s*:\s*\d+",
            r"Sitesymmetry\s*:\s*\d+", r"SubrowOrigin\s*:\s*\d+\s+NumSites\s*:\s*\d+", r"End"],
}


def _grammar_violations(ext, text):
    pats = [re.compile(p + r"\s*$") for p in _GRAMMAR[ext]]
    bad = []
    for line in text.splitlines():
        line = line.split("#", 1)[0].strip()
        if line and not any(p.match(line) for p in pats):
            bad.append(line)
    return bad


def test_writer_follows_reference_line_grammar(golden, tmp_path):
    """Every line this package's writer emits has one of the shapes of the
    reference's Bookshelf files; the reference's own unit-test design passes
    the same check (so the grammar is the reference's, not this writer's)."""
    g = golden("bookshelf_simple.npz")
    for ext in _GRAMMAR:
        assert _grammar_violations(ext, str(g["text_" + ext])) == [], ext
    aux = bookshelf.write_bookshelf(synthetic.scaled(300, num_bins=16, seed=3, name="gram"), str(tmp_path))
    for ext in _GRAMMAR:
        with open(aux[:-4] + "." + ext) as f:
            assert _grammar_violations(ext, f.read()) == [], ext


def test_reference_design_write_read(golden, tmp_path):
    """The reference's unit-test design read, written and read again keeps its
    node sizes, fixed positions, pins and offsets, and rows."""
    g = golden("bookshelf_simple.npz")
    src = tmp_path / "in"
    src.mkdir()
    r = bookshelf.read_bookshelf(_write_case(g, src))
    aux = bookshelf.write_bookshelf(r, str(tmp_path / "out"), name="again")
    r2 = bookshelf.read_bookshelf(aux)
    n = r.num_physical_nodes
    assert (r2.num_physical_nodes, r2.num_terminals, r2.num_nets, r2.num_pins) == \
        (n, r.num_terminals, r.num_nets, r.num_pins)
    np.testing.assert_array_equal(r2.node_size_x[:n], r.node_size_x[:n])
    np.testing.assert_array_equal(r2.node_x[r.num_movable_nodes:n], r.node_x[r.num_movable_nodes:n])
    np.testing.assert_array_equal(r2.pin2node_map, r.pin2node_map)
    np.testing.assert_array_equal(r2.flat_net2pin_start_map, r.flat_net2pin_start_map)
    np.testing.assert_allclose(r2.pin_offset_x, r.pin_offset_x, atol=1e-5)
    np.testing.assert_allclose(r2.pin_offset_y, r.pin_offset_y, atol=1e-5)
    assert (r2.xl, r2.yl, r2.xh, r2.yh, r2.row_height) == (r.xl, r.yl, r.xh, r.yh, r.row_height)
