"""The library's input.data reader (n2p2_structures_*, Structure::readFromLines
on every block) against an independent Python restatement and, for
positions, against the reference library itself: bit-identical numbers,
the same symbols, boxes, comments, and the reference's error messages."""
import os

import numpy as np
import pytest

from n2p2_b200 import Structure, read_structures, water
from n2p2_b200._lib import N2P2Error, OutOfRangeError
from oracle import ref as oref
from tests import helpers as H


def _same(native, checker):
    assert len(native) == len(checker)
    for s, c in zip(native, checker):
        assert s.elements == c["elements"]
        assert np.array_equal(s.positions.view(np.int64), c["positions"].view(np.int64))
        assert np.array_equal(s.forcesRef.view(np.int64), c["forces"].view(np.int64))
        assert np.array_equal(s.chargesRef.view(np.int64), c["charges"].view(np.int64))
        assert s.energyRef == c["energy"] and s.chargeRef == c["charge"]
        assert s.comment == c["comment"]
        assert (s.box is None) == (c["box"] is None)
        if s.box is not None:
            assert np.array_equal(s.box.view(np.int64), c["box"].view(np.int64))


@pytest.mark.parametrize("name", ["H2O_RPBE-D3", "Cu2S_PBE"])
def test_reference_example_files(name):
    path = os.path.join(H.GOLDEN, "examples", name, "input.data")
    _same(read_structures(path), H.python_read_structures(open(path).read()))


def test_generated_file_with_every_keyword(tmp_path):
    rng = np.random.default_rng(2)
    structs = water.water_batch(5, seed=21, n_min=32, n_max=64)
    structs.append(Structure(structs[0].positions[:9], structs[0].elements[:9], None, comment="a cluster"))
    lines = []
    for k, s in enumerate(structs):
        s.comment = s.comment or "box %d  with  spaces" % k
        s.energyRef = float(rng.normal())
        s.chargeRef = float(rng.normal())
        s.forcesRef = rng.normal(size=(s.numAtoms, 3))
        s.chargesRef = rng.normal(size=s.numAtoms)
        text = s.to_text().replace("begin", "begin set=train" if k % 2 else "begin", 1)
        lines.append(text + ("\n\n" if k == 2 else ""))
    text = "".join(lines).replace("\n", "\r\n", 40)   # some CRLF line ends
    p = tmp_path / "input.data"
    p.write_bytes(text.encode())
    checker = H.python_read_structures(text)
    _same(read_structures(str(p)), checker)
    _same(read_structures(text, is_text=True), checker)
    assert len(read_structures(str(p), limit=2)) == 2


@pytest.mark.skipif(not oref.available(), reason="reference library not built")
def test_positions_bit_identical_to_the_reference_reader():
    s = water.water_box(32, seed=9)
    cluster = Structure(s.positions * (1.0 + 1e-7), s.elements, None)   # non-periodic: no remap
    text = cluster.to_text()
    got = read_structures(text, is_text=True)[0]
    snap = H.reference_snapshot(H.WATER40, got)
    assert np.array_equal(got.positions.view(np.int64), snap["positions"].view(np.int64))


@pytest.mark.parametrize("text,cls,msg", [
    ("atom 0 0 0 H 0 0 0 0 0\nend\n", N2P2Error, 'expected "begin" keyword'),
    ("begin\nbogus 1\nend\n", N2P2Error, 'unknown keyword "bogus"'),
    ("begin set=valid\nend\n", N2P2Error, "check \\\"begin\\\" arguments|check \"begin\" arguments"),
    ("begin\nlattice 1 0 0\nlattice 0 1 0\nend\n", N2P2Error, "Strange number of box vectors"),
    ("begin\n" + "lattice 1 0 0\n" * 4 + "end\n", N2P2Error, "Too many box vectors"),
    ("begin\natom 0 0 0 H 0 0\nend\n", OutOfRangeError, "too short"),
])
def test_reference_error_messages(text, cls, msg):
    with pytest.raises(cls, match=msg):
        read_structures(text, is_text=True)


def test_trailing_block_without_end_is_not_read():
    s = water.water_box(32, seed=1)
    text = s.to_text() + s.to_text().rsplit("end", 1)[0]
    assert len(read_structures(text, is_text=True)) == 1
