"""Input files for the reader parity tests: hand-written edge cases of every
format the reference viewer's reader handles (viewer/mesh_io.cpp) and seeded
random files built from the same token grammar.  Each case is (file name,
bytes); the extension picks the reader."""
import struct

import numpy as np

# ---- hand-written cases ------------------------------------------------------------

NUMBERS = ["1", "-2.5", "+.5", "3.", "1e5", "1E-3", "-0", "0.1e+2", "00012", "4.9e-324",
           "2.5e-324", "1e-400", "1.7976931348623157e308"]
BAD_NUMBERS = ["nan", "inf", "-inf", "1e", "1e+", ".", "+", "-.e1", "e5", "5e", "1e400", "-1e400",
               "0x1A", "1,5", "1.5.3", "1-2", "+-1", "x"]


def hand_cases():
    c = {}
    # "x y z" lines (viewer/mesh_io.cpp:402-413)
    c["plain.xyz"] = b"0 0 0\n1 0 0\n0 1 0\n0 0 1\n"
    c["comments.xyz"] = b"# header\n\n1 2 3\n  # indented is not a comment\n4 5 6 # trailing\n#7 8 9\n"
    c["crlf.txt"] = b"1 2 3\r\n4 5 6\r\n\r\n7 8 9"
    c["spaces.pts"] = b"\t1\v2\f3\r\n  -1   -2   -3  \n"
    c["noext"] = b"1 2 3\n"
    c["upper.XYZ"] = b"1 2 3\n"
    c["empty.xyz"] = b""
    c["only_comments.xyz"] = b"# a\n# b\n"
    c["numbers.xyz"] = "".join(f"{a} {b} {n}\n" for a, b in zip(NUMBERS, NUMBERS[1:] + NUMBERS[:1])
                               for n in NUMBERS[:3]).encode()
    c["bad_numbers.xyz"] = "".join(f"1 2 {b}\n{b} 1 2\n" for b in BAD_NUMBERS).encode() + b"9 9 9\n"
    c["short_lines.xyz"] = b"1 2\n3\n4 5 6 7\n8 9 10\n"
    c["unknown.abc"] = b"1 2 3\n"
    c["dir.with.dots/points"] = b"5 6 7\n"
    # OBJ (viewer/mesh_io.cpp:42-71)
    c["quad.obj"] = b"# quad\nv 0 0 0\nv 1 0 0\nv 1 1 0\nv 0 1 0\nvt 0 0\nvn 0 0 1\nf 1/1/1 2/2/1 3/3/1 4/4/1\n"
    c["negative.obj"] = b"v 0 0 0\nv 1 0 0\nv 0 1 0\nf -3 -2 -1\nv 0 0 1\nf -1 -2 -3 -4\n"
    c["bad_faces.obj"] = (b"v 0 0 0\nv 1 0 0\nv 0 1 0\nv 0 0 1\n"
                          b"f 1 2\nf 0 1 2 3\nf 1 2 99\nf //1 2// 3/4 4\nf a b c\n"
                          b"f 99999999999999999999 1 2 3\nf -99999999999999999999 1 2 3\n"
                          b"f +1 +2 +3\nf 1.9 2.9 3.9\nf 4 3 2 1\n")
    c["faces_first.obj"] = b"f 1 2 3\nv 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 3\n"
    c["tags.obj"] = b"v1 0 0 0\n  v 1 1 1\nv 2 2\nv 3 3 3 1.0\nV 4 4 4\n\tf 1 2 3\nv nan 0 0\nv 5 5 5\r\n"
    c["empty.obj"] = b"# nothing\nvt 0 0\n"
    # OFF (viewer/mesh_io.cpp:76-134)
    c["cube.off"] = (b"OFF\n# comment\n8 6 12\n0 0 0\n1 0 0\n1 1 0\n0 1 0\n0 0 1\n1 0 1\n1 1 1\n0 1 1\n"
                     b"4 0 1 2 3\n4 4 5 6 7\n4 0 1 5 4\n4 2 3 7 6\n4 0 3 7 4\n4 1 2 6 5\n")
    c["counts_on_magic.off"] = b"OFF 4 1 0\n0 0 0\n1 0 0\n0 1 0\n0 0 1\n3 0 1 2\n"
    c["coff.off"] = b"COFF\n3 1 0\n0 0 0 255 0 0 255\n1 0 0 0 255 0 255\n0 1 0 0 0 255 255\n3 0 1 2 10 20 30\n"
    c["noff.off"] = b"noff\n\n  # c\n3 1 0 # counts\n0 0 0 0 0 1\n1 0 0 0 0 1\n0 1 0 0 0 1\n3 2 1 0\n"
    c["split_counts.off"] = b"OFF 3\n1 0\n0 0 0\n1 0 0\n0 1 0\n3 0 1 2\n"
    c["truncated.off"] = b"OFF\n4 1 0\n0 0 0\n1 0 0\n0 1\n"
    c["malformed.off"] = b"OFF\nfour one zero\n"
    c["not_off.off"] = b"PLY\n3 1 0\n"
    c["empty.off"] = b"\n  \n# only a comment\n"
    c["bad_faces.off"] = (b"OFF\n4 5 0\n0 0 0\n1 0 0\n0 1 0\n0 0 1\n3 0 1 9\n4 0 1 2 3\n-1 0 1 2\n"
                          b"3 0 1\n2\n")
    c["no_newline.off"] = b"OFF\n3 1 0\n0 0 0\n1 0 0\n0 1 0\n3 0 1 2"
    c["comment_in_body.off"] = b"OFF\n3 0 0\n0 0 0\n# no\n1 0 0\n0 1 0\n"
    c["bad_vertex_number.off"] = b"OFF\n2 0 0\n0 0 nan\n1 1 1\n"
    # PLY (viewer/mesh_io.cpp:139-315)
    c["ascii.ply"] = (b"ply\nformat ascii 1.0\ncomment made by hand\nobj_info x\nelement vertex 4\n"
                      b"property float x\nproperty float y\nproperty float z\nproperty uchar red\n"
                      b"element face 2\nproperty list uchar int vertex_indices\nend_header\n"
                      b"0 0 0 255\n1 0 0 0\n0 1 0 1\n0 0 1 2\n3 0 1 2\n4 0 1 2 3\n")
    c["crlf.ply"] = (b"ply\r\nformat ascii 1.0\r\nelement vertex 3\r\nproperty double x\r\nproperty double y\r\n"
                     b"property double z\r\nelement face 1\r\nproperty list uchar int vertex_index\r\n"
                     b"end_header\r\n0 0 0\r\n1 0 0\r\n0 1 0\r\n3 0 1 2\r\n")
    c["order.ply"] = (b"ply\nformat ascii 1.0\nelement vertex 2\nproperty float z\nproperty float nx\n"
                      b"property float y\nproperty float x\nproperty float x\nend_header\n1 2 3 4 5\n6 7 8 9 10\n")
    c["edges.ply"] = (b"ply\nformat ascii 1.0\nelement vertex 3\nproperty float x\nproperty float y\n"
                      b"property float z\nelement edge 2\nproperty int vertex1\nproperty int vertex2\n"
                      b"element face 2\nproperty list uchar int vertex_indices\nend_header\n"
                      b"0 0 0\n1 0 0\n0 1 0\n0 1\n1 2\n3 0 1 2\n3 2 1 -1\n")
    c["short_rows.ply"] = (b"ply\nformat ascii 1.0\nelement vertex 3\nproperty float x\nproperty float y\n"
                           b"property float z\nelement face 1\nproperty list uchar int vertex_indices\n"
                           b"end_header\n1 2\n3 x 5\n6 7 8 9\n5 0 1 2\n")
    c["early_end.ply"] = (b"ply\nformat ascii 1.0\nelement vertex 3\nproperty float x\nproperty float y\n"
                          b"property float z\nend_header\n0 0 0\n1 1 1\n")
    c["no_xyz.ply"] = b"ply\nformat ascii 1.0\nelement vertex 1\nproperty float x\nproperty float y\nend_header\n1 2\n"
    c["big_endian.ply"] = b"ply\nformat binary_big_endian 1.0\nelement vertex 0\nend_header\n"
    c["not_ply.ply"] = b"plx\nformat ascii 1.0\n"
    c["no_vertices.ply"] = b"ply\nformat ascii 1.0\nelement vertex 0\nproperty float x\nproperty float y\nproperty float z\nend_header\n"
    c["header_only.ply"] = b"ply\nformat ascii 1.0\nelement vertex\nproperty\nproperty list\nelement face abc\nend_header\n"
    c["binary.ply"] = binary_ply(np.random.default_rng(1), 40, 20)
    c["binary_empty_element.ply"] = (b"ply\nformat binary_little_endian 1.0\nelement marker 5\n"
                                     b"element vertex 1\nproperty double x\nproperty double y\n"
                                     b"property double z\nend_header\n" + struct.pack("<3d", 1, 2, 3))
    c["binary_truncated.ply"] = binary_ply(np.random.default_rng(2), 10, 5)[:-7]
    c["binary_unknown_type.ply"] = (b"ply\nformat binary_little_endian 1.0\nelement vertex 1\n"
                                    b"property float x\nproperty float y\nproperty float z\nproperty half w\n"
                                    b"end_header\n" + struct.pack("<fff", 1, 2, 3) + b"\0\0")
    # STL (viewer/mesh_io.cpp:320-397)
    c["binary.stl"] = binary_stl(np.random.default_rng(3), 30, header=b"made by hand")
    c["binary_solid_header.stl"] = binary_stl(np.random.default_rng(4), 12, header=b"solid but binary")
    c["binary_truncated.stl"] = binary_stl(np.random.default_rng(5), 10, header=b"x")[:-30]
    c["binary_short.stl"] = b"tiny"
    c["binary_zero.stl"] = binary_stl(np.random.default_rng(8), 0, header=b"no triangles")
    c["ascii.stl"] = ascii_stl(np.random.default_rng(6), 8, shared=True)
    c["ascii_upper.stl"] = ascii_stl(np.random.default_rng(7), 3, shared=False).replace(b"vertex", b"VERTEX")
    c["ascii_no_facet.stl"] = b"solid x\n" + b" " * 600 + b"\nfacet normal 0 0 1\nvertex 0 0 0\nvertex 1 0 0\nvertex 0 1 0\n"
    c["ascii_degenerate.stl"] = (b"solid t\nfacet normal 0 0 0\nouter loop\nvertex 0 0 0\nvertex 0 0 0\n"
                                 b"vertex 1 0 0\nendloop\nendfacet\nfacet\nvertex -0 0 0\nvertex 1 0 0\n"
                                 b"vertex 0 1 0\nvertex 5 5 5\nendsolid\n")
    c["ascii_empty.stl"] = b"solid nothing\nfacet\nendsolid\n"
    return c


def binary_ply(rng, nv, nf):
    """A binary little-endian PLY with every scalar type and several list types."""
    types = [("char", "b"), ("uchar", "B"), ("short", "h"), ("ushort", "H"), ("int", "i"), ("uint", "I"),
             ("float", "f"), ("double", "d"), ("int8", "b"), ("uint8", "B"), ("int16", "h"),
             ("uint16", "H"), ("int32", "i"), ("uint32", "I"), ("float32", "f"), ("float64", "d")]
    extra = [types[int(k)] for k in rng.integers(0, len(types), 3)]
    xyz_t = [types[int(k)] for k in rng.choice([6, 7, 14, 15, 2, 4], 3)]
    hdr = ["ply", "format binary_little_endian 1.0", "comment binary", f"element vertex {nv}"]
    props = [(f"e{i}", t) for i, t in enumerate(extra[:1])] + [("x", xyz_t[0]), ("y", xyz_t[1])] + \
            [(f"e{i}", t) for i, t in enumerate(extra[1:], 1)] + [("z", xyz_t[2])]
    hdr += [f"property {t[0]} {n}" for n, t in props]
    hdr += [f"element face {nf}", "property list uchar int vertex_indices", "property float quality",
            "element misc 2", "property list ushort double values", "end_header"]
    body = b""
    for _ in range(nv):
        for n, (tn, code) in props:
            body += struct.pack("<" + code, _value(rng, code))
    for _ in range(nf):
        k = int(rng.integers(0, 6))
        body += struct.pack("<B", k) + struct.pack(f"<{k}i", *rng.integers(-2, nv + 3, k).tolist())
        body += struct.pack("<f", float(rng.normal()))
    for _ in range(2):
        k = int(rng.integers(0, 4))
        body += struct.pack("<H", k) + struct.pack(f"<{k}d", *rng.normal(size=k).tolist())
    return ("\n".join(hdr) + "\n").encode() + body


def _value(rng, code):
    lim = {"b": 127, "B": 255, "h": 32767, "H": 65535, "i": 2**31 - 1, "I": 2**32 - 1}
    if code in "fd":
        x = float(rng.normal() * 10 ** int(rng.integers(-3, 4)))
        return x if rng.random() > 0.05 else float(["nan", "inf", "-inf"][int(rng.integers(0, 3))])
    lo = 0 if code.isupper() else -lim[code] - 1
    return int(rng.integers(lo, lim[code], endpoint=True))


def binary_stl(rng, n, header=b""):
    hdr = header.ljust(80, b"\0")[:80]
    body = b""
    corners = rng.normal(size=(max(n, 1) * 3 // 2 + 1, 3)).astype(np.float32)
    for _ in range(n):
        tri = corners[rng.integers(0, corners.shape[0], 3)]
        body += struct.pack("<3f", *rng.normal(size=3).astype(np.float32).tolist())
        body += struct.pack("<9f", *tri.reshape(-1).tolist()) + struct.pack("<H", 0)
    return hdr + struct.pack("<I", n) + body


def ascii_stl(rng, n, shared):
    pts = rng.integers(-3, 4, size=(n + 2, 3)) if shared else rng.normal(size=(3 * n, 3))
    out = ["solid test"]
    for t in range(n):
        out += ["  facet normal 0 0 1", "    outer loop"]
        idx = rng.integers(0, pts.shape[0], 3) if shared else range(3 * t, 3 * t + 3)
        out += ["      vertex " + " ".join(repr(float(x)) for x in pts[i]) for i in idx]
        out += ["    endloop", "  endfacet"]
    out.append("endsolid test")
    return ("\n".join(out) + "\n").encode()


# ---- random cases ------------------------------------------------------------------


def _num(rng):
    r = rng.random()
    if r < 0.08:
        return BAD_NUMBERS[int(rng.integers(0, len(BAD_NUMBERS)))]
    if r < 0.2:
        return NUMBERS[int(rng.integers(0, len(NUMBERS)))]
    if r < 0.35:
        return str(int(rng.integers(-5, 50)))
    return repr(float(rng.normal() * 10 ** int(rng.integers(-4, 5))))


def _ws(rng):
    return [" ", " ", " ", "\t", "  ", " \v", "\f "][int(rng.integers(0, 7))]


def _eol(rng):
    return ["\n", "\n", "\n", "\r\n", " \n", "\t\n"][int(rng.integers(0, 6))]


def random_xyz(rng):
    lines = []
    for _ in range(int(rng.integers(0, 40))):
        r = rng.random()
        if r < 0.05:
            lines.append("# " + _num(rng))
        elif r < 0.1:
            lines.append("")
        else:
            k = int(rng.choice([2, 3, 3, 3, 4]))
            lines.append(_ws(rng).join(_num(rng) for _ in range(k)))
    return "".join(l + _eol(rng) for l in lines).encode()


def random_obj(rng):
    lines, nv = [], 0
    for _ in range(int(rng.integers(0, 60))):
        r = rng.random()
        if r < 0.5:
            lines.append("v " + _ws(rng).join(_num(rng) for _ in range(int(rng.choice([3, 3, 3, 2, 4])))))
            nv += 1
        elif r < 0.85:
            toks = []
            for _ in range(int(rng.integers(1, 7))):
                i = int(rng.integers(-nv - 2, nv + 3))
                form = int(rng.integers(0, 5))
                toks.append([f"{i}", f"{i}/1", f"{i}//2", f"{i}/3/4", f"/{i}"][form])
            lines.append("f " + " ".join(toks))
        elif r < 0.92:
            lines.append(["vt 0 1", "vn 0 0 1", "o name", "g grp", "s off", "usemtl m"][int(rng.integers(0, 6))])
        else:
            lines.append("# " + _num(rng))
    return "".join(l + _eol(rng) for l in lines).encode()


def random_off(rng):
    nv, nf = int(rng.integers(0, 12)), int(rng.integers(0, 8))
    magic = ["OFF", "COFF", "NOFF", "off"][int(rng.integers(0, 4))]
    out = [f"{magic} {nv} {nf} 0" if rng.random() < 0.3 else magic]
    if not out[0].endswith(" 0"):
        if rng.random() < 0.3:
            out.append("# counts next")
        out.append(f"{nv} {nf} {int(rng.integers(0, 3))}")
    for _ in range(nv - (1 if rng.random() < 0.1 else 0)):
        extra = " 0.5 0.5 0.5" if magic == "COFF" else ""
        out.append(" ".join(_num(rng) if rng.random() < 0.1 else repr(float(rng.normal())) for _ in range(3)) + extra)
    for _ in range(nf):
        k = int(rng.integers(0, 6))
        out.append(" ".join([str(k)] + [str(int(rng.integers(-1, nv + 2))) for _ in range(k)]))
    text = "\n".join(out)
    return (text + ("\n" if rng.random() < 0.8 else "")).encode()


def random_ply_ascii(rng):
    nv, nf = int(rng.integers(0, 10)), int(rng.integers(0, 6))
    props = ["x", "y", "z"]
    rng.shuffle(props)
    if rng.random() < 0.5:
        props.insert(int(rng.integers(0, 4)), "nx")
    hdr = ["ply", "format ascii 1.0", f"element vertex {nv}"] + [f"property float {p}" for p in props]
    hdr += [f"element face {nf}", "property list uchar int vertex_indices", "end_header"]
    rows = []
    for _ in range(nv):
        k = len(props) - (1 if rng.random() < 0.1 else 0)
        rows.append(" ".join(_num(rng) for _ in range(k)))
    for _ in range(nf):
        k = int(rng.integers(0, 6))
        rows.append(" ".join([str(k)] + [str(int(rng.integers(-1, nv + 2))) for _ in range(k)]))
    if rng.random() < 0.1 and rows:
        rows.pop()
    return ("\n".join(hdr + rows) + "\n").encode()


def random_cases(n_each=40, seed=7):
    rng = np.random.default_rng(seed)
    c = {}
    for i in range(n_each):
        c[f"r{i}.xyz"] = random_xyz(rng)
        c[f"r{i}.obj"] = random_obj(rng)
        c[f"r{i}.off"] = random_off(rng)
        c[f"r{i}.ply"] = random_ply_ascii(rng)
        c[f"rb{i}.ply"] = binary_ply(rng, int(rng.integers(0, 30)), int(rng.integers(0, 10)))
        c[f"rb{i}.stl"] = binary_stl(rng, int(rng.integers(0, 20)), header=b"rand")
        c[f"ra{i}.stl"] = ascii_stl(rng, int(rng.integers(0, 6)), shared=bool(rng.random() < 0.5))
    return c


def write_cases(root, cases):
    """Writes the cases under `root`; returns their paths in order."""
    import os

    paths = []
    for name, data in cases.items():
        p = os.path.join(root, name)
        os.makedirs(os.path.dirname(p), exist_ok=True)
        with open(p, "wb") as f:
            f.write(data)
        paths.append(p)
    return paths


def mutated_cases(n, seed):
    """Byte-level mutations of the cases above (flips to separators and number
    characters, cuts, inserted text and tokens): malformed files of every kind."""
    rng = np.random.default_rng(seed)
    items = list({**hand_cases(), **random_cases(8, 3)}.items())
    toks = [b"12", b"-1", b"1e3", b" \n", b"nan", b"0.5", b"\r\n", b"#"]
    out = {}
    for it in range(n):
        name, data = items[int(rng.integers(0, len(items)))]
        b = bytearray(data)
        for _ in range(int(rng.integers(1, 4))):
            op = int(rng.integers(0, 4))
            if op == 0 and b:
                b[int(rng.integers(0, len(b)))] = int(rng.choice([32, 10, 13, 9, 46, 45, 43, 101, 48, 49, 35, 47, 0,
                                                                  255, int(rng.integers(0, 256))]))
            elif op == 1 and b:
                i = int(rng.integers(0, len(b)))
                del b[i:i + int(rng.integers(1, 10))]
            elif op == 2:
                i = int(rng.integers(0, len(b) + 1))
                b[i:i] = bytes(rng.integers(32, 127, int(rng.integers(1, 6))).astype(np.uint8))
            else:
                i = int(rng.integers(0, len(b) + 1))
                b[i:i] = toks[int(rng.integers(0, len(toks)))]
        out[f"m{it}_{name.replace('/', '_')}"] = bytes(b)
    return out
