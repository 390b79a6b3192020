"""Build step of the reference-kernel checker (test infrastructure only).

Copies, unchanged, the named kernels and device helpers of the reference's
gkway/coarsen.hpp and gkway/uncoarsen.hpp out of the reference tree into
oracle/_ref/refkern_src.cuh (git-ignored), so that oracle/refkern.cu can run the
reference's own kernels on small cases and compare them with the oracle.  The
reference headers cannot be compiled whole: they include ModernGPU, which is
not vendored (the host functions call it); the kernels listed here call
nothing from it.  Each function is found by name and taken from its
qualifier line to the brace that closes its body.

Usage: python refkern_extract.py <reference root> <output file>
"""
from __future__ import annotations

import re
import sys

# (header, function names) in the order they appear
FUNCS = [
    ("gkway/coarsen.hpp", [
        "get_value_combo", "get_first_val_from_value_combo", "get_second_val_from_val_combo",
        "matching_with_score", "HEC_union_find", "count_num_coarsen_vertex", "construct_cmap",
        "cal_coarsen_vwgt", "construct_tmp_adjp", "copied_adjncy", "construct_coarsen_graph",
        "HEC_remove_duplicate_edge", "init_group_id", "count_coarsen_group", "init_group_ptr",
        "breakdown_large_group",
    ]),
    ("gkway/uncoarsen.hpp", [
        "is_valid_move", "calculate_gain", "update_vertex_info", "find_mv_wgt_sequence",
        "find_balance_sequence", "apply_sequence_move", "expand_partition", "calculate_cutsize",
    ]),
]


def extract(text: str, name: str) -> str:
    m = re.search(r"(__global__|__device__)\s+(?:[\w\*]+\s+)*\**" + re.escape(name) + r"\s*\(", text)
    if not m:
        raise SystemExit(f"refkern_extract: {name} not found")
    start = text.rfind("\n", 0, m.start()) + 1
    brace = text.index("{", m.end())
    depth = 0
    for i in range(brace, len(text)):
        if text[i] == "{":
            depth += 1
        elif text[i] == "}":
            depth -= 1
            if depth == 0:
                return text[start:i + 1]
    raise SystemExit(f"refkern_extract: unbalanced braces in {name}")


def main(argv) -> int:
    ref, out = argv[1], argv[2]
    parts = ["// generated by oracle/refkern_extract.py from the reference tree; not part of the repository",
             "namespace gk {"]
    for header, names in FUNCS:
        with open(f"{ref}/{header}") as f:
            text = f.read()
        for name in names:
            parts.append(f"// {header}: {name}")
            parts.append(extract(text, name))
    parts.append("}  // namespace gk")
    with open(out, "w") as f:
        f.write("\n".join(parts) + "\n")
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv))
