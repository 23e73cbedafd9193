"""CPU restatement of OFELI's XML mesh-file reading and writing, for small
files (plain Python loops).

TEST INFRASTRUCTURE ONLY: the parity tests use it as the checker of the
library's ofg_mesh_file_read / ofg_mesh_file_write; the product never
imports it.  It follows (paths within the OFELI project):

  Mesh::get                  src/mesh/Mesh.cpp:2639-2668
  XMLParser::on_tag_open     src/io/XMLParser.cpp:646-760 (every open resets
                             the element node count; a Material open leaves
                             mesh mode)
  XMLParser::read_mesh       src/io/XMLParser.cpp:1174-1217 (Mesh: shape
                             defaults from the dimension known before each
                             attribute, attributes in name order)
  XMLParser::on_cdata        src/io/XMLParser.cpp:1316-1375 (whitespace
                             tokens; Material pairs while in a mesh)
  XMLParser::read_mesh_data  src/io/XMLParser.cpp:2211-2295 (coordinates
                             through std::stof, codes through DOFCode)
  DOFCode                    src/mesh/MeshUtil.cpp:101-116
  Material::set / check / getName   src/mesh/Material.cpp:90-134
  Mesh::put                  src/mesh/Mesh.cpp:2731-2806
"""
import ctypes
import re

import numpy as np

_libc = ctypes.CDLL(None, use_errno=True)
_libc.strtof.restype = ctypes.c_float
_libc.strtof.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_char_p)]

ELEMENT_SHAPES = {"point": 1, "line": 2, "triangle": 3, "tria": 3, "quadrilateral": 4, "quad": 4,
                  "tetrahedron": 5, "tetra": 5, "hexahedron": 6, "hexa": 6, "pentahedron": 7,
                  "penta": 7, "prism": 8, "pyramid": 9}
SIDE_SHAPES = {"line": 2, "tria": 3, "triangle": 3, "quad": 4, "quadrilateral": 4}
PUT_NAMES = ["none", "point", "line", "triangle", "quadrilateral", "tetrahedron", "hexahedron",
             "pentahedron"]


class MeshFileError(ValueError):
    pass


def stof(tok):
    """std::stof: strtof on the token; no conversion or ERANGE is an error."""
    raw = tok.encode()
    end = ctypes.c_char_p()
    buf = ctypes.create_string_buffer(raw)
    ctypes.set_errno(0)
    v = _libc.strtof(buf, ctypes.byref(end))
    if ctypes.cast(end, ctypes.c_void_p).value == ctypes.cast(buf, ctypes.c_void_p).value:
        raise MeshFileError("invalid coordinate %r" % tok)
    if ctypes.get_errno() == 34:  # ERANGE
        raise MeshFileError("coordinate out of float range %r" % tok)
    return float(np.float32(v))


def stoi(tok):
    """std::stoi: leading blanks, sign, digits, stop at the first other char."""
    m = re.match(r"\s*([+-]?)(\d+)", tok)
    if not m:
        raise MeshFileError("invalid integer %r" % tok)
    v = int(m.group(2))
    v = -v if m.group(1) == "-" else v
    if not -2 ** 31 <= v < 2 ** 31:
        raise MeshFileError("integer out of range %r" % tok)
    return v


def dof_code(mark, nb_dof):
    """DOFCode: the remainder keeps the mark's sign, each quotient (C
    truncation) is multiplied by it."""
    sign = -1 if mark < 0 else 1
    j = mark
    out = []
    for k in range(nb_dof):
        kk = 10 ** (nb_dof - k - 1)
        m = j // kk if j >= 0 else -((-j) // kk)
        out.append(m * sign)
        j -= m * kk
    return out


_LABEL = re.compile(r"[A-Za-z0-9_.:\-]*")
_TAGSPACE = " \n\t\r"


def _blank(seg):
    return all(c in _TAGSPACE for c in seg)


def read(path):
    text = open(path, "r", encoding="latin-1", newline="").read()
    st = dict(dim=2, nb_dof=1, el_shape=0, el_nodes=0, sd_shape=0, sd_nodes=0, coords=[],
              node_code=[], elem=[], elem_code=[], sides=[], side_code=[], materials=[])
    set_mesh, mesh_type, tag = True, True, ""
    el_shape_s, sd_shape_s, el_nodes, sd_nodes = "triangle", "line", 0, 2
    pos, stack = 0, []
    seen = set()

    def on_text(seg):
        toks = [t for t in re.split(r"[ \t\n\v\f\r]+", seg) if t]
        if not toks:
            return
        if tag == "Material" and set_mesh:
            if len(toks) % 2:
                raise MeshFileError("Material block ends inside a pair")
            for i in range(0, len(toks), 2):
                st["materials"].append((stoi(toks[i]), toks[i + 1]))
            return
        if not (set_mesh and mesh_type):
            return
        dim, nd = st["dim"], st["nb_dof"]
        kind = tag.lower()
        if kind in ("nodes", "elements", "sides"):
            # Node's coordinates hold 3 values, its codes MAX_NBDOF_NODE = 6
            if not (1 <= dim <= 3 and 1 <= nd <= 6):
                raise MeshFileError("dim must be 1..3 and nb_dof 1..6")
            # OFELI restarts its labels on a second text of a block
            if kind in seen:
                raise MeshFileError("more than one %s text" % tag)
            seen.add(kind)
        if tag in ("Nodes", "nodes"):
            rec = dim + 1
            if len(toks) % rec:
                raise MeshFileError("Nodes block ends inside a record")
            for r in range(0, len(toks), rec):
                st["coords"].append([stof(t) for t in toks[r:r + dim]])
                st["node_code"].append(dof_code(stoi(toks[r + dim]), nd))
        elif tag in ("Elements", "elements"):
            if not 1 <= el_nodes <= 20:
                raise MeshFileError("Elements without a nodes attribute")
            st["el_shape"], st["el_nodes"] = ELEMENT_SHAPES.get(el_shape_s, 0), el_nodes
            rec = el_nodes + 1
            if len(toks) % rec:
                raise MeshFileError("Elements block ends inside a record")
            nn = len(st["coords"])
            for r in range(0, len(toks), rec):
                labels = [stoi(t) for t in toks[r:r + el_nodes]]
                if any(v < 1 or v > nn for v in labels):
                    raise MeshFileError("element names a missing node")
                st["elem"].append([v - 1 for v in labels])
                st["elem_code"].append(stoi(toks[r + el_nodes]))
        elif tag in ("Sides", "sides"):
            if sd_shape_s not in SIDE_SHAPES:
                raise MeshFileError("unknown side shape")
            st["sd_shape"], st["sd_nodes"] = SIDE_SHAPES[sd_shape_s], sd_nodes
            rec = sd_nodes + 1
            if len(toks) % rec:
                raise MeshFileError("Sides block ends inside a record")
            nn = len(st["coords"])
            for r in range(0, len(toks), rec):
                labels = [stoi(t) for t in toks[r:r + sd_nodes]]
                if any(v < 1 or v > nn for v in labels):
                    raise MeshFileError("side names a missing node")
                st["sides"].append([v - 1 for v in labels])
                st["side_code"].append(dof_code(stoi(toks[r + sd_nodes]), nd))

    had_root = False
    n = len(text)

    def fail(msg):
        raise MeshFileError("XML: " + msg)

    def label(q):
        return _LABEL.match(text, q).end()

    def on_open(name, attrs):
        nonlocal el_nodes, tag, mesh_type, el_shape_s, sd_shape_s, sd_nodes
        el_nodes = 0
        tag = name
        if name == "Material":
            mesh_type = False
        if not (set_mesh and mesh_type):
            return
        for k in sorted(attrs):
            v = attrs[k]
            if name == "Mesh":
                if st["dim"] == 1:
                    el_shape_s = "line"
                elif st["dim"] == 2:
                    el_shape_s, sd_shape_s, sd_nodes = "triangle", "line", 2
                elif st["dim"] == 3:
                    el_shape_s, sd_shape_s, sd_nodes = "tetrahedron", "triangle", 3
                if k == "file":
                    raise MeshFileError("included mesh files are not supported")
                if k == "dim":
                    st["dim"] = stoi(v)
                elif k == "nb_dof":
                    st["nb_dof"] = stoi(v)
            elif name in ("Elements", "elements"):
                if k == "shape":
                    el_shape_s = v
                if k == "nodes":
                    el_nodes = stoi(v)
            elif name in ("Sides", "sides"):
                if k == "shape":
                    sd_shape_s = v
                if k == "nodes":
                    sd_nodes = stoi(v)

    while pos < n:
        if not stack:
            while pos < n and text[pos] in _TAGSPACE:
                pos += 1
            if pos >= n:
                break
            if text[pos] != "<":
                fail("unexpected character outside tag")
        else:
            lt = text.find("<", pos)
            seg = text[pos:lt if lt >= 0 else n]
            if ">" in seg:
                fail("'>' in text")
            if not _blank(seg):
                if "&" in seg and tag.lower() in ("nodes", "elements", "sides"):
                    fail("entity in data")
                on_text(seg)
            if lt < 0:
                fail("open tag missing close tag")
            pos = lt
        pos += 1
        if pos >= n:
            fail("tag not finished")
        c = text[pos]
        if c == "?":
            if stack:
                fail("processing instruction inside an element")
            q = text.find("?>", pos)
            if q < 0:
                fail("processing instruction not closed")
            pos = q + 2
        elif c == "!":
            pos += 1
            if text.startswith("-", pos):
                if not text.startswith("--", pos):
                    fail("expecting '-' for comment")
                q = text.find("-->", pos)
                if q < 0:
                    fail("comment not closed")
                pos = q + 3
            elif text.startswith("[", pos):
                if not text.startswith("[CDATA[", pos):
                    fail("unknown element")
                q = text.find("]]>", pos + 7)
                if q < 0 or not stack:
                    fail("bad CDATA")
                if not _blank(text[pos + 7:q]):
                    on_text(text[pos + 7:q])
                pos = q + 3
            else:
                if stack or had_root or not text.startswith("DOCTYPE", pos):
                    fail("unexpected '<!'")
                q = text.find(">", pos)
                if q < 0 or q - pos < 8:
                    fail("bad DOCTYPE")
                pos = q + 1
        elif c == "/":
            q = label(pos + 1)
            name = text[pos + 1:q]
            if q >= n or text[q] != ">" or not stack or stack[-1] != name:
                fail("closing tag mismatch")
            stack.pop()
            if name == "Mesh":
                set_mesh = False
            pos = q + 1
        else:
            q = label(pos)
            if q == pos:
                fail("unexpected character at the beginning of a tag")
            if not stack and had_root:
                fail("second root")
            name = text[pos:q]
            pos = q
            attrs, single, after_name = {}, False, True
            while True:
                if pos >= n:
                    fail("tag not finished")
                c = text[pos]
                if c in _TAGSPACE:
                    pos += 1
                    after_name = False
                elif c == ">":
                    pos += 1
                    break
                elif c == "/":
                    if not text.startswith("/>", pos):
                        fail("unexpected character after slash")
                    pos += 2
                    single = True
                    break
                elif not after_name and _LABEL.match(text, pos).end() > pos:
                    q = label(pos)
                    key = text[pos:q]
                    if not text.startswith('="', q):
                        fail("attribute without a double-quoted value")
                    v1 = text.find('"', q + 2)
                    if v1 < 0:
                        fail("tag not finished")
                    val = text[q + 2:v1]
                    if "&" in val:
                        fail("entity in attribute")
                    attrs[key] = val
                    pos = v1 + 1
                else:
                    fail("unexpected character in tag")
            on_open(name, attrs)
            if single:
                if name == "Mesh":
                    set_mesh = False
                if not stack:
                    had_root = True
            else:
                stack.append(name)
    if stack:
        raise MeshFileError("open tag missing close tag")
    dim, nd = st["dim"], st["nb_dof"]
    out = dict(dim=dim, nb_dof=nd, el_shape=st["el_shape"], el_nodes=st["el_nodes"],
               sd_shape=st["sd_shape"], sd_nodes=st["sd_nodes"], materials=st["materials"])
    out["coords"] = np.array(st["coords"], dtype=np.float64).reshape(-1, dim)
    out["node_code"] = np.array(st["node_code"], dtype=np.int32).reshape(-1, nd)
    out["elem"] = np.array(st["elem"], dtype=np.int32).reshape(-1, max(st["el_nodes"], 1))
    out["elem_code"] = np.array(st["elem_code"], dtype=np.int32)
    out["sides"] = np.array(st["sides"], dtype=np.int32).reshape(-1, max(st["sd_nodes"], 1))
    out["side_code"] = np.array(st["side_code"], dtype=np.int32).reshape(-1, nd)
    return out


def material_name_1(m):
    """Material::getName(1) after Mesh::get (pairs first, then element codes
    registered as Generic by Material::check)."""
    for code, name in m.get("materials", []):
        if code == 1:
            return name
    if np.any(np.asarray(m["elem_code"]) == 1):
        return "Generic"
    return " "


def put(m, path=None):
    """Mesh::put, returned as bytes (and written to path when given)."""
    dim, n = m["dim"], m["nb_dof"]
    coords = np.asarray(m["coords"], dtype=np.float64).reshape(-1, dim)
    ncode = np.asarray(m["node_code"], dtype=np.int64).reshape(-1, n)
    lines = ['<?xml version="1.0"?>', "<OFELI_File>", "<info>", "   <title></title>",
             "   <date></date>", "   <author></author>", "</info>",
             '<Mesh dim="%d" nb_dof="%d">' % (dim, n)]
    if coords.shape[0]:
        lines.append("   <Nodes>")
        for x, c in zip(coords, ncode):
            mm = sum(abs(int(c[j])) * 10 ** (n - 1 - j) for j in range(n))
            if c[0] < 0:
                mm = (2 ** 64 - mm) % 2 ** 64
            lines.append("".join("  %18.8e" % v for v in x) + "%10d" % mm)
        lines.append("   </Nodes>")
    elem = np.asarray(m["elem"]).reshape(len(m["elem_code"]), -1) if len(m["elem_code"]) else []
    if len(m["elem_code"]):
        lines.append('   <Elements shape="%s" nodes="%d">' % (PUT_NAMES[m["el_shape"]], m["el_nodes"]))
        for e, c in zip(elem, m["elem_code"]):
            lines.append("".join("%8d" % (v + 1) for v in e) + "%8d" % c)
        lines.append("   </Elements>")
    scode = np.asarray(m["side_code"], dtype=np.int64).reshape(-1, n)
    if scode.shape[0]:
        sides = np.asarray(m["sides"]).reshape(scode.shape[0], -1)
        lines.append('   <Sides shape="%s" nodes="%d">' % (PUT_NAMES[m["sd_shape"]], m["sd_nodes"]))
        for s, c in zip(sides, scode):
            mm = sum(int(c[j]) * 10 ** (n - 1 - j) for j in range(n)) % 2 ** 64
            lines.append("".join("%8d" % (v + 1) for v in s) + "%6d" % mm)
        lines.append("   </Sides>")
    if material_name_1(m) != "Generic":
        lines += ["   <Material>", "   </Material>"]
    lines += ["</Mesh>", "</OFELI_File>"]
    data = ("\n".join(lines) + "\n").encode()
    if path is not None:
        with open(path, "wb") as fh:
            fh.write(data)
    return data
