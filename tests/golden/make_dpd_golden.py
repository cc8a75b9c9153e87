"""Extracts the DPD layout golden vectors from the reference's MArray test
(src/external/marray/test/dpd_varray.cxx: the `layouts`, `irreps`, `lengths`,
`strides` and `offsets` tables, and the tensor they describe: irrep 1,
2 irreps, lengths {{3,1},{2,2},{1,2},{3,4}}) into dpd_layout_golden.json.

    python tests/golden/make_dpd_golden.py <tblis source tree>   (default: $TBLIS_REFERENCE)
"""
import json
import os
import re
import sys

LAYOUT_CODE = {"BALANCED_COLUMN_MAJOR": 0, "BALANCED_ROW_MAJOR": 1, "BLOCKED_COLUMN_MAJOR": 2,
               "BLOCKED_ROW_MAJOR": 3, "PREFIX_COLUMN_MAJOR": 4, "PREFIX_ROW_MAJOR": 5}


def block_of(src, name):
    m = re.search(name + r"\s*(\[[^\]]*\])+\s*=\s*\{", src)
    i = m.end() - 1
    depth = 0
    for j in range(i, len(src)):
        if src[j] == "{":
            depth += 1
        elif src[j] == "}":
            depth -= 1
            if depth == 0:
                return src[i:j + 1]
    raise ValueError(name)


def ints(text):
    # evaluates simple sums like "80+66+3"
    out = []
    for tok in re.findall(r"[0-9][0-9+\s]*", text):
        tok = tok.strip()
        if tok:
            out.append(sum(int(x) for x in tok.split("+") if x.strip()))
    return out


def main(ref):
    path = os.path.join(ref, "src/external/marray/test/dpd_varray.cxx")
    src = open(path).read()
    layouts = [LAYOUT_CODE[x] for x in re.findall(r"(\w+_(?:ROW|COLUMN)_MAJOR)", block_of(src, "layouts"))]
    irreps = ints(block_of(src, "irreps"))
    lengths = ints(block_of(src, "lengths"))
    strides = ints(block_of(src, "strides"))
    offsets = ints(block_of(src, "offsets"))
    assert len(layouts) == 6 and len(irreps) == 32 and len(lengths) == 32
    assert len(strides) == 6 * 32 and len(offsets) == 48
    out = {
        "source": "src/external/marray/test/dpd_varray.cxx:7-51",
        "irrep": 1, "nirrep": 2, "lens": [[3, 1], [2, 2], [1, 2], [3, 4]],
        "layouts": layouts,
        "blocks": [irreps[4 * i:4 * i + 4] for i in range(8)],
        "block_lengths": [lengths[4 * i:4 * i + 4] for i in range(8)],
        "block_strides": [[strides[32 * j + 4 * i:32 * j + 4 * i + 4] for i in range(8)] for j in range(6)],
        "block_offsets": [offsets[8 * j:8 * j + 8] for j in range(6)],
    }
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "dpd_layout_golden.json")
    with open(dst, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", dst)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("TBLIS_REFERENCE", "/root/reference"))
