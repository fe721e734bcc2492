"""Generate tests/golden/airfoil_kernels.json: the five user kernels of the
reference's airfoil demo (demo/airfoil_kernels.py: save_soln_code,
adt_calc_code, res_calc_code, bres_calc_code, update_code), exactly as the
reference's users pass them to op2.Kernel.

The demo module is read as text and parsed with ``ast`` (it is never imported
or executed: it imports the reference's op2).  Run in a container that has
the reference sources (found where oracle/build.py looks for them); the
output is committed so tests never read the reference at run time.
"""

import ast
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from oracle.build import REFERENCE  # noqa: E402

NAMES = ("save_soln", "adt_calc", "res_calc", "bres_calc", "update")


def main():
    path = os.path.join(REFERENCE, "demo", "airfoil_kernels.py")
    tree = ast.parse(open(path).read())
    code = {}
    for node in tree.body:
        if (isinstance(node, ast.Assign) and len(node.targets) == 1
                and isinstance(node.targets[0], ast.Name)
                and node.targets[0].id.endswith("_code")
                and isinstance(node.value, ast.Constant) and isinstance(node.value.value, str)):
            code[node.targets[0].id[:-len("_code")]] = node.value.value
    assert set(code) == set(NAMES), sorted(code)
    out = {"source": "demo/airfoil_kernels.py", "kernels": {n: code[n] for n in NAMES}}
    with open(os.path.join(HERE, "airfoil_kernels.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
        f.write("\n")


if __name__ == "__main__":
    main()
