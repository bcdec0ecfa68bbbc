"""The .unv -> .fly converter (the reference's tofly.py command): nodes, volume elements
with group names as tags, optional face elements, contact groups, and the command line."""

import io
import sys

import numpy as np
import pytest

from mammos_mumag import fly, tofly

UNV = """    -1
   164
         1  SI: Meter (newton)
    -1
    -1
  2411
         1         1         1        11
   0.0000000000000000D+00   0.0000000000000000D+00   0.0000000000000000D+00
         2         1         1        11
   1.0000000000000000D+00   0.0000000000000000D+00   0.0000000000000000D+00
         3         1         1        11
   0.0000000000000000D+00   1.0000000000000000D+00   0.0000000000000000D+00
         4         1         1        11
   0.0000000000000000D+00   0.0000000000000000D+00   1.0000000000000000D+00
         5         1         1        11
   1.0000000000000000D+00   1.0000000000000000D+00   1.0000000000000000D+00
    -1
    -1
  2412
         7        91         2         1         7         3
         1         2         3
        10       111         2         1         7         4
         1         2         3         4
        11       111         2         1         7         4
         2         3         4         5
    -1
    -1
  2467
         1         0         0         0         0         0         0         2
1
         8        10         0         0         8         7         0         0
         2         0         0         0         0         0         0         1
2
         8        11         0         0
    -1
"""


def test_convert_volume_elements(tmp_path):
    (tmp_path / "m.unv").write_text(UNV)
    tofly.convert(tmp_path / "m.unv", tmp_path / "out" / "m.fly")
    X, T, tag = fly.read_mesh(tmp_path / "out" / "m.fly")
    np.testing.assert_array_equal(X, [[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [1, 1, 1]])
    np.testing.assert_array_equal(T, [[0, 1, 2, 3], [1, 2, 3, 4]])
    np.testing.assert_array_equal(tag, [1, 2])
    text = (tmp_path / "out" / "m.fly").read_text().splitlines()
    assert text[0] == "Mesh" and text[1] == "3D-nodes 5" and text[2].split()[:3] == ["1", "1", "0"]
    assert text[-4:] == ["Tri3 0", "Tri3_Contact 0", "Point1 0", "Tags"]


def test_faces_kept_and_contact_group():
    nodes, elems, tag, contact = tofly.read_unv(UNV, exclude_dims=(1,))
    assert [e[1] for e in elems] == ["91", "111", "111"] and contact == set()
    text = tofly.fly_text(nodes, elems, tag, contact, exclude_dims=(1,)).splitlines()
    i = text.index("Tri3 1")
    assert text[i + 1] == "1 1 1 2 3"  # the face carries group "1"
    j = text.index("Tet4 2")
    assert text[j + 1] == "1 1 1 2 3 4" and text[j + 2] == "2 2 2 3 4 5"
    assert text[-3:] == ["Tri3_Contact 0", "Point1 0", "Tags"]
    # a group named "contact" turns its elements into contact elements; a tetrahedron has
    # no contact counterpart in finley
    unv = UNV.replace("\n2\n         8        11", "\ncontact\n         8        11")
    nodes, elems, tag, contact = tofly.read_unv(unv)
    assert contact == {"11"}
    with pytest.raises(tofly.UnvError):
        tofly.fly_text(nodes, elems, tag, contact)


def test_command_line_stdin_stdout(monkeypatch, capsys):
    monkeypatch.setattr(sys, "stdin", io.StringIO(UNV))
    assert tofly.main(["-", "-"]) == 0
    out = capsys.readouterr().out.splitlines()
    assert out[1] == "3D-nodes 5" and "Tet4 2" in out
