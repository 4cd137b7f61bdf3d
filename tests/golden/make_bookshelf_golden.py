"""Builds tests/golden/bookshelf_simple.npz from the reference's place_io unit
test (unittest/ops/place_io_unittest): the five files of its 10-node Bookshelf
design (simple/simple.{aux,nodes,nets,pl,scl}, stored as text) and what the
reference's own parser reads from them (simple.golden, the output of
place_io_unittest.py: node sizes and positions, pin offsets relative to the
node's lower-left corner, the net -> pin maps, the rows' bounding box).

    DREAMPLACE_REFERENCE=<checkout> python tests/golden/make_bookshelf_golden.py

Test infrastructure: only tests/test_bookshelf.py reads the fixture.
"""
import ast
import os
import re

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.environ.get("DREAMPLACE_REFERENCE", "/root/reference")
CASE = os.path.join(REF, "unittest", "ops", "place_io_unittest")

# keys of simple.golden kept in the fixture, and how their values parse
NUMERIC_LISTS = ("node_x", "node_y", "node_size_x", "node_size_y", "pin_offset_x", "pin_offset_y", "flat_net2pin_map",
                 "flat_net2pin_start_map", "pin2node_map", "pin2net_map", "flat_node2pin_start_map")
NAME_LISTS = ("node_names", "net_names")
SCALARS = ("num_nodes", "num_terminals", "xl", "yl", "xh", "yh", "row_height", "site_width", "num_movable_pins")


def parse_golden(text):
    """key = value lines of simple.golden -> dict of numpy arrays / scalars."""
    out = {}
    for line in text.splitlines():
        if " = " not in line:
            continue
        key, value = line.split(" = ", 1)
        key = key.strip()
        if key in NUMERIC_LISTS:
            out[key] = np.array(ast.literal_eval(value), np.float64)
        elif key in NAME_LISTS:
            out[key] = np.array([s.strip() for s in value.strip()[1:-1].split(",")])
        elif key in SCALARS:
            out[key] = np.float64(ast.literal_eval(value))
    missing = [k for k in NUMERIC_LISTS + NAME_LISTS + SCALARS if k not in out]
    assert not missing, missing
    return out


def main():
    files = {}
    for ext in ("aux", "nodes", "nets", "pl", "scl"):
        with open(os.path.join(CASE, "simple", "simple." + ext)) as f:
            files["text_" + ext] = np.array(f.read())
    with open(os.path.join(CASE, "simple.golden")) as f:
        golden = parse_golden(f.read())
    # the aux line must name exactly the stored files
    assert re.findall(r"simple\.(\w+)", str(files["text_aux"])) == ["nodes", "nets", "pl", "scl"]
    np.savez_compressed(os.path.join(HERE, "bookshelf_simple.npz"), **files, **golden)
    print("wrote bookshelf_simple.npz: %d nodes, %d nets, %d pins"
          % (int(golden["num_nodes"]), len(golden["net_names"]), len(golden["pin2node_map"])))


if __name__ == "__main__":
    main()
