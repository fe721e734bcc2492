"""Generate the golden fixtures of tests/golden/ from the reference's own tests.

Run in a container that has the reference sources (found where
oracle/build.py looks for them: ``OP2B_REFERENCE``, else the build recipe's
own location); the output files are committed so tests never read the
reference at run time.  Sources read (as text, never imported or executed):

* test/unit/test_matrices.py: the Sparsity CSR golden (:54-62), the 2-element
  mesh (:76, :111-114, :122), the user kernels of the Mat/RHS tests
  (:150-576) and their expected values (:578-608);
* test/unit/test_indirect_loop.py / test_plan.py: the shuffled-map seed
  (``random.shuffle(u_map, _seed)``, :40-41 / :43-44) -- reproduced by the
  tests with Python 2's shuffle algorithm, not stored;
* test/regression/tests/mass2d_triangle/mass2d_triangle.expected: the
  regression golden (f, x, b, mat.array) of the 100x100 mass problem.  Its
  mesh numbering comes from gmsh and is not available, so only
  numbering-invariant summaries are stored: the distinct Mat values with their
  counts, the sorted RHS and f, and the sums.
"""

import ast
import json
import os
import pickle
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from oracle.build import REFERENCE as REF  # noqa: E402


def _fixture_body(src, name):
    """Source text of the body of ``def <name>(cls...)`` in a test class."""
    m = re.search(r"\n    def %s\(.*?\n(.*?)(?=\n    @|\n    def |\Z)" % re.escape(name), src, re.S)
    return m.group(1)


def _balanced(text, start):
    """The bracketed literal beginning at text[start] == '['."""
    depth = 0
    for k in range(start, len(text)):
        if text[k] in "[(":
            depth += 1
        elif text[k] in "])":
            depth -= 1
            if depth == 0:
                return text[start:k + 1]
    raise ValueError("unbalanced literal")


def _asarray_literal(body):
    k = body.index("asarray(") + len("asarray(")
    return ast.literal_eval(_balanced(body, k))


def _kernel_code(src, fixture):
    body = _fixture_body(src, fixture)
    m = re.search(r'kernel_code\s*=\s*"""(.*?)"""', body, re.S)
    code = m.group(1)
    n = re.search(r'op2\.Kernel\(kernel_code,\s*"(\w+)"\)', body).group(1)
    return code, n


def _literal_after(src, fixture, var):
    body = _fixture_body(src, fixture)
    k = body.index(var)
    return ast.literal_eval(_balanced(body, body.index("[", k)))


def matrices():
    path = os.path.join(REF, "test", "unit", "test_matrices.py")
    src = open(path).read()
    out = {"source": "test/unit/test_matrices.py"}
    m = re.search(r"elements = op2\.Set\((\d+)\).*?nodes = op2\.Set\((\d+)\).*?"
                  r"elem_node = op2\.Map\(elements, nodes, 3, (\[.*?\])\).*?"
                  r"_rowptr == (\[.*?\]).*?_colidx == (\[.*?\])\)", src, re.S)
    out["sparsity"] = {"nelem": int(m.group(1)), "nnodes": int(m.group(2)),
                       "map": ast.literal_eval(m.group(3).replace("\\", "")),
                       "rowptr": ast.literal_eval(m.group(4)),
                       "colidx": ast.literal_eval(m.group(5).replace("\\", ""))}
    out["elem_node_map"] = ast.literal_eval(
        re.search(r"elem_node_map = numpy\.asarray\((\[.*?\])", src).group(1))
    coords_body = _fixture_body(src, "coords")
    out["coords"] = _asarray_literal(coords_body)
    out["f"] = _asarray_literal(_fixture_body(src, "f"))
    m = re.search(r"asarray\((\[.*?\])\*(\d+)", _fixture_body(src, "f_vec"), re.S)
    out["f_vec"] = [list(t) for t in ast.literal_eval(m.group(1))] * int(m.group(2))
    kernels = {}
    for fx in ("mass", "rhs", "mass_ffc", "rhs_ffc", "rhs_ffc_itspace", "mass_vector_ffc",
               "rhs_ffc_vector", "rhs_ffc_vector_itspace", "zero_dat", "zero_vec_dat",
               "kernel_inc", "kernel_set", "kernel_inc_vec", "kernel_set_vec"):
        code, name = _kernel_code(src, fx)
        kernels[fx] = {"name": name, "code": code}
    out["kernels"] = kernels
    out["expected_matrix"] = _literal_after(src, "expected_matrix", "expected_vals")
    out["expected_vector_matrix"] = _literal_after(src, "expected_vector_matrix", "expected_vals")
    out["expected_rhs"] = _asarray_literal(_fixture_body(src, "expected_rhs"))
    out["expected_vec_rhs"] = _asarray_literal(_fixture_body(src, "expected_vec_rhs"))
    with open(os.path.join(HERE, "matrices.json"), "w") as f:
        json.dump(out, f, indent=1)


def regression():
    path = os.path.join(REF, "test", "regression", "tests", "mass2d_triangle",
                        "mass2d_triangle.expected")
    with open(path, "rb") as f:
        fv, xv, bv, mat = pickle.load(f, encoding="latin1")
    mat = np.asarray(mat, dtype=np.float64)
    vals, counts = np.unique(mat, return_counts=True)
    np.savez_compressed(os.path.join(HERE, "mass2d_triangle_summary.npz"),
                        mat_values=vals, mat_counts=counts,
                        b_sorted=np.sort(np.asarray(bv, np.float64).ravel()),
                        f_sorted=np.sort(np.asarray(fv, np.float64).ravel()),
                        mat_sum=mat.sum(), b_sum=np.asarray(bv, np.float64).sum(),
                        nnz=mat.size, nnodes=np.asarray(fv).size)


if __name__ == "__main__":
    matrices()
    regression()
    print("fixtures written to", HERE)
