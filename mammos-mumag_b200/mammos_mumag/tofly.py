"""Convert I-DEAS universal (``.unv``) meshes, as Salome exports them, to finley ``.fly``.

    python -m mammos_mumag.tofly [-e DIMENSIONS] [UNV] [FLY]

The reference's converter (``src/mammos_mumag/tofly.py:1-386``, same command line and
``convert(unv_path, fly_path, exclude_list)``) feeds the hysteresis loop its mesh; this is
the same conversion, written from the universal-file layout:

* dataset 2411 (nodes): per node a line ``label coord_sys disp_sys colour`` and a line
  ``x y z`` (Fortran ``D`` exponents allowed);
* dataset 2412 (elements): per element a line ``label fe_type phys mat colour n_nodes``;
  beam types (11, 21, 22, 23, 24) add a line of 3 orientation fields; then the n node
  labels over one or more lines;
* dataset 2467 (groups): per group a line of 8 integers whose last is the entity count, a
  line with the group name, then the entities, 4 integers each ``type tag 0 0``, two per
  line.  An element's tag in the ``.fly`` file is the name of the group that holds it
  (``-1`` if none); elements of a group named ``contact`` become contact elements.

Output: ``Mesh``; ``3D-nodes N`` with lines ``label label 0 x y z``; one section per
element type (``Tet4``, ``Tri3``, ...) with lines ``i tag n1 n2 ...`` numbered from 1 per
type, contact sections numbered on after the last normal type; then the empty sections
and ``Tags``.  Elements of excluded dimensions (default 1 and 2: only volume elements)
are dropped.  Coordinates are copied as written, with ``D`` exponents turned into ``E``.
"""

from __future__ import annotations

import argparse
import contextlib
import pathlib
import sys

DELIM = "-1"
BEAM_TYPES = {"11", "21", "22", "23", "24"}
TYPES_BY_DIM = {1: {"11", "21", "22", "24"}, 2: {"41", "81", "91", "42", "82", "92", "44"},
                3: {"115", "116", "111", "118"}}
FLY_NAME = {"11": "Line2", "21": "Line2", "22": "Line3", "24": "Line3", "41": "Tri3", "81": "Tri3",
            "91": "Tri3", "42": "Tri6", "82": "Tri6", "92": "Tri6", "44": "Rec4", "115": "Hex8",
            "116": "Hex20", "111": "Tet4", "118": "Tet10"}
FLY_CONTACT_NAME = {"115": "Rec4_Contact", "116": "Rec8_Contact", "112": "Tri3_Contact"}
CONTACT_GROUP = "contact"


class UnvError(ValueError):
    pass


def _datasets(lines):
    """Yield (dataset number, its lines) of a universal file."""
    i, n = 0, len(lines)
    while i < n:
        if lines[i].strip() == DELIM and i + 1 < n:
            kind = lines[i + 1].strip()
            j = i + 2
            while j < n and lines[j].strip() != DELIM:
                j += 1
            if j >= n:
                raise UnvError(f"dataset {kind} is not terminated")
            yield kind, lines[i + 2:j]
            i = j + 1
        else:
            i += 1


def _nodes(body):
    if len(body) % 2:
        raise UnvError("node dataset 2411 has an odd number of lines")
    out = []
    for k in range(0, len(body), 2):
        label = body[k].split()[0]
        xyz = body[k + 1].replace("D", "E").replace("d", "e").split()
        if len(xyz) != 3:
            raise UnvError(f"node {label}: expected 3 coordinates")
        out.append((label, xyz))
    return out


def _elements(body):
    words = iter(w for line in body for w in line.split())
    out = []
    for label in words:
        try:
            fe_type = next(words)
            next(words), next(words), next(words)  # physical, material, colour
            count = int(next(words))
            if fe_type in BEAM_TYPES:
                next(words), next(words), next(words)  # orientation fields
            nodes = [next(words) for _ in range(count)]
        except StopIteration:
            raise UnvError(f"element {label}: record ends early") from None
        out.append((label, fe_type, nodes))
    return out


def _groups(body):
    tag, contact = {}, set()
    i = 0
    while i < len(body):
        head = body[i].split()
        if not head:
            i += 1
            continue
        if len(head) < 8 or i + 1 >= len(body):
            raise UnvError("group record ends early")
        count, name = int(head[7]), body[i + 1].strip()
        ints = []
        i += 2
        while len(ints) < 4 * count:
            if i >= len(body):
                raise UnvError(f"group {name}: entity list ends early")
            ints.extend(body[i].split())
            i += 1
        members = ints[1::4][:count]
        if name == CONTACT_GROUP:
            contact.update(members)
        else:
            for e in members:
                tag[e] = name
    return tag, contact


def read_unv(text: str, exclude_dims=(1, 2)):
    """Nodes [(label, [x, y, z])], elements [(label, fe_type, [node labels])] of the kept
    dimensions, element tags {label: group name} and the contact element labels."""
    excluded = set().union(*(TYPES_BY_DIM[d] for d in exclude_dims)) if exclude_dims else set()
    nodes, elements, tag, contact = [], [], {}, set()
    for kind, body in _datasets(text.splitlines()):
        if kind == "2411":
            nodes.extend(_nodes(body))
        elif kind == "2412":
            elements.extend(e for e in _elements(body) if e[1] not in excluded)
        elif kind == "2467":
            t, c = _groups(body)
            tag.update(t)
            contact |= c
    return nodes, elements, tag, contact


def fly_text(nodes, elements, tag, contact, exclude_dims=(1, 2)) -> str:
    out = ["Mesh", f"3D-nodes {len(nodes)}"]
    out += [f"{label} {label} 0 {x} {y} {z}" for label, (x, y, z) in nodes]
    normal, contacts = {}, {}
    for label, fe_type, ns in elements:
        line = f"{tag.get(label, '-1')} {' '.join(ns)}"
        if label in contact:
            if fe_type not in FLY_CONTACT_NAME:
                raise UnvError(f"element {label}: type {fe_type} has no contact counterpart")
            contacts.setdefault(FLY_CONTACT_NAME[fe_type], []).append(line)
        else:
            if fe_type not in FLY_NAME:
                raise UnvError(f"element {label}: unsupported element type {fe_type}")
            normal.setdefault(fe_type, []).append(line)
    nxt = 1
    for fe_type, lines in normal.items():
        out.append(f"{FLY_NAME[fe_type]} {len(lines)}")
        out += [f"{i} {ln}" for i, ln in enumerate(lines, start=1)]
        nxt = len(lines) + 1
    for name, lines in contacts.items():
        out.append(f"{name} {len(lines)}")
        out += [f"{i} {ln}" for i, ln in enumerate(lines, start=nxt)]
    if 2 in set(exclude_dims or ()):
        out += ["Tri3 0", "Tri3_Contact 0", "Point1 0", "Tags"]
    else:
        out += ["Tri3_Contact 0", "Point1 0", "Tags"]
    return "\n".join(out) + "\n"


def convert(unv_path, fly_path, exclude_list=(1, 2)) -> None:
    """Convert ``unv_path`` to ``fly_path`` (parent folders are created)."""
    text = pathlib.Path(unv_path).read_text()
    fly = fly_text(*read_unv(text, exclude_list), exclude_dims=exclude_list)
    fly_path = pathlib.Path(fly_path)
    fly_path.parent.mkdir(parents=True, exist_ok=True)
    fly_path.write_text(fly)


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description="Convert unv files to the fly format.")
    ap.add_argument("unv", nargs="?", default="-", help="input .unv path, '-' for stdin")
    ap.add_argument("fly", nargs="?", default="-", help="output .fly path, '-' for stdout")
    ap.add_argument("-e", "--exclude", default="1,2", metavar="DIMENSIONS",
                    help="comma-separated dimensions to drop (default 1,2: volume elements only)")
    args = ap.parse_args(argv)
    dims = tuple(int(d) for d in args.exclude.split(",") if d.strip())
    text = sys.stdin.read() if args.unv == "-" else pathlib.Path(args.unv).read_text()
    fly = fly_text(*read_unv(text, dims), exclude_dims=dims)
    if args.fly == "-":
        sys.stdout.write(fly)
    else:
        with contextlib.suppress(FileExistsError):
            pathlib.Path(args.fly).parent.mkdir(parents=True, exist_ok=True)
        pathlib.Path(args.fly).write_text(fly)
    return 0


if __name__ == "__main__":
    sys.exit(main())
