"""Re-encode CULS's 4-input rewriting library into ``rwlib.bin``.

The rewriting pass must reproduce CULS's NPN classes and replacement
subgraphs bit for bit, so it needs exactly the same library table that CULS
ships as ``src/algorithms/rewrite_library.inc`` (a flat C ``int`` array of
218,008 entries, decoded by ``rw::CPUSolver::ReadLibrary`` in
``src/algorithms/rewrite.cu:1281-1307``).  That table is data, licensed
BSD-3-Clause by CUHK (see ``LICENSE.rwlib`` beside this script); this script
stores the same values in a compact byte layout of this project's own:

    magic   8 bytes  b"CULSRWL1"
    sha256 32 bytes  digest of the decoded int sequence (little-endian int32)
    phase  u8[65536] NPN input/output negation mask per truth table (0..31)
    perm   u8[65536] index into perm4 per truth table (0..23)
    perm4  u8[24*4]  the 24 permutations of 4 inputs
    cls    u8[65536] NPN class per truth table (0..221)
    nNodes u8[222]   internal nodes per class forest (<= 50)
    nRoots u8[222]   subgraph roots per class (<= 15)
    then per class: nNodes * (fanin0, fanin1, compl0, compl1) as u8,
                    followed by nRoots root indices as u8

Every value fits in a byte (checked below).  Usage::

    python make_rwlib.py <path/to/rewrite_library.inc> [out.bin]
"""
import hashlib
import re
import struct
import sys
from pathlib import Path

N_TT = 1 << 16
N_CLASS = 222
MAGIC = b"CULSRWL1"
# SHA-256 of the decoded library (int32 little-endian), pinned so that a
# different library version cannot be encoded silently.
EXPECTED_SHA = "5b552d1fcc10dd1b4d651301a0aee032017ecfc764b615d1cc99a80fce5863af"


def decode_inc(text: str):
    m = re.search(r"LIBRARY\s*\[\s*\]\s*=\s*\{([^}]*)\}", text)
    if not m:
        raise ValueError("no LIBRARY[] array found")
    vals = [int(v) for v in m.group(1).split(",") if v.strip()]
    return vals


def encode(vals):
    cur = 0

    def take(k):
        nonlocal cur
        out = vals[cur:cur + k]
        if len(out) != k:
            raise ValueError("library truncated")
        cur += k
        return out

    phase = take(N_TT)
    perm = take(N_TT)
    perm4 = take(24 * 4)
    cls = take(N_TT)
    n_nodes = take(N_CLASS)
    n_roots = take(N_CLASS)
    body = []
    for c in range(N_CLASS):
        for i in range(n_nodes[c]):
            f0, f1, c0, c1 = take(4)
            # forests are topological: a node only reads inputs 0..3 or
            # earlier nodes (index i+4 is this node)
            if not (0 <= f0 < i + 4 and 0 <= f1 < i + 4 and c0 in (0, 1) and c1 in (0, 1)):
                raise ValueError(f"bad node class {c} index {i}")
            body += [f0, f1, c0, c1]
        roots = take(n_roots[c])
        if any(not (0 <= r < n_nodes[c] + 4) for r in roots):
            raise ValueError(f"bad root in class {c}")
        body += roots
    if cur != len(vals):
        raise ValueError("trailing data in library")
    allv = phase + perm + perm4 + cls + n_nodes + n_roots + body
    if any(not (0 <= v < 256) for v in allv):
        raise ValueError("value out of byte range")
    digest = hashlib.sha256(struct.pack(f"<{len(vals)}i", *vals)).digest()
    if digest.hex() != EXPECTED_SHA:
        raise ValueError(f"library digest {digest.hex()} != pinned {EXPECTED_SHA}")
    return MAGIC + digest + bytes(allv)


def main(argv):
    src = Path(argv[1])
    out = Path(argv[2]) if len(argv) > 2 else Path(__file__).with_name("rwlib.bin")
    vals = decode_inc(src.read_text())
    blob = encode(vals)
    out.write_bytes(blob)
    print(f"wrote {out} ({len(blob)} bytes), sha256(lib)={blob[8:40].hex()}")


if __name__ == "__main__":
    main(sys.argv)
