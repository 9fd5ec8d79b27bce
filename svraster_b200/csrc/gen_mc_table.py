"""Generate mc_table.inc: the marching-cubes case table packed one 64-bit word per case.

Topology parity with the reference extraction requires the identical triangulation, so the
table is derived from the reference's own case table (cuda/svraster_cuda/marching_cubes.py:11-268,
edge numbering of its pair list :336-349).  Packing: entry k of case c (an edge id 0..11, or
15 for "none") sits in bits [4k, 4k+4) of kMcCases[c].

Usage:  python svraster_b200/csrc/gen_mc_table.py <reference root>
"""
import ast
import os
import sys


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("SVR_REFERENCE_DIR")
    if not ref:
        sys.exit("usage: give the reference checkout as the first argument or in SVR_REFERENCE_DIR")
    src = open(os.path.join(ref, "cuda", "svraster_cuda", "marching_cubes.py")).read()
    start = src.index("tri_table = torch.tensor(")
    end = src.index("], dtype=torch.long", start)
    rows = ast.literal_eval(src[start + len("tri_table = torch.tensor("):end + 1])
    assert len(rows) == 256 and all(len(r) == 15 for r in rows)
    words = []
    for r in rows:
        w = 0
        for k, e in enumerate(r):
            w |= (15 if e < 0 else e) << (4 * k)
        words.append(w)
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "mc_table.inc")
    with open(out, "w") as f:
        f.write("// Generated by gen_mc_table.py: marching-cubes cases, 15 x 4-bit edge ids per case\n")
        f.write("// (15 = no edge).  Identical triangulation to the reference extraction.\n")
        for i in range(0, 256, 4):
            f.write("    " + ", ".join(f"0x{w:016x}ull" for w in words[i:i + 4]) + ",\n")
    print("wrote", out)


if __name__ == "__main__":
    main()
