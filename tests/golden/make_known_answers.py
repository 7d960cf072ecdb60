"""Extract the known-answer arrays of cuCIM's own tests and docstrings into
tests/golden/known_answers.json.

cuCIM cannot be imported here (it needs CuPy), so its files are read as
text: each entry below names the file and line range that holds a literal
array, which is parsed with ast.literal_eval. Run from the repository root
with the root of a cuCIM source checkout as the only argument:

    python tests/golden/make_known_answers.py <cucim source root>
"""

import ast
import json
import os
import re
import sys

if len(sys.argv) != 2:
    sys.exit("usage: python tests/golden/make_known_answers.py <cucim source root>")
REF = sys.argv[1]
SK = "python/cucim/src/cucim/skimage"

# (key, file, first line, last line): the literal arrays inside that range,
# in order of appearance
SOURCES = [
    ("gaussian_delta_docstring", f"{SK}/_shared/filters.py", 100, 117),
    ("hessian_5x5_fd", f"{SK}/feature/tests/test_corner.py", 136, 170),
    ("hessian_3d_fd_slice", f"{SK}/feature/tests/test_corner.py", 195, 213),
    ("hessian_eigvals_5x5_fd", f"{SK}/feature/tests/test_corner.py", 284, 307),
]


def _arrays_in(text):
    """Every balanced [[...]] literal in `text` (comments removed)."""
    text = re.sub(r"#[^\n]*", "", text)
    out, depth, start = [], 0, None
    for i, ch in enumerate(text):
        if ch == "[":
            if depth == 0:
                start = i
            depth += 1
        elif ch == "]":
            depth -= 1
            if depth == 0 and start is not None:
                lit = text[start:i + 1]
                if lit.startswith("[["):
                    out.append(ast.literal_eval(lit))
                start = None
    return out


def main():
    result = {}
    for key, rel, lo, hi in SOURCES:
        with open(os.path.join(REF, rel)) as f:
            lines = f.readlines()[lo - 1:hi]
        arrays = _arrays_in("".join(lines))
        result[key] = {"source": f"{rel}:{lo}-{hi}", "arrays": arrays}
    here = os.path.dirname(os.path.abspath(__file__))
    with open(os.path.join(here, "known_answers.json"), "w") as f:
        json.dump(result, f, indent=1)
    for k, v in result.items():
        print(k, [len(a) for a in v["arrays"]])


if __name__ == "__main__":
    main()
