"""Generate tests/golden/reference_stapi.json: the C API the reference's coretrace/stapi.h
declares (every st_* function with its return and parameter types), which the drop-in
library's include/stapi.h must declare the same way (tests/test_abi.py).

    python tests/golden/make_api_fixture.py <SolTrace checkout>   (or $SOLTRACE_REFERENCE)
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from helpers import c_declarations  # noqa: E402


def main():
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("SOLTRACE_REFERENCE")
    if not root:
        raise SystemExit("usage: make_api_fixture.py <SolTrace checkout> (or set SOLTRACE_REFERENCE)")
    decl = c_declarations(open(os.path.join(root, "coretrace", "stapi.h")).read())
    out = {"source": "coretrace/stapi.h", "functions": {k: {"returns": r, "params": p} for k, (r, p) in sorted(decl.items())}}
    with open(os.path.join(HERE, "reference_stapi.json"), "w") as f:
        json.dump(out, f, indent=1)
    print(len(decl), "functions")


if __name__ == "__main__":
    main()
