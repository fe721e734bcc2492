"""Build the oracle's native parts.  TEST INFRASTRUCTURE ONLY.

* ``oracle/_build/liboracle.so`` from ``oracle/csrc/oracle_core.c`` (gcc).
* ``oracle/_ref/libref_sparsity.so``: the reference's own
  ``pyop2/sparsity_utils.cxx`` compiled unmodified with g++ against the shim
  header ``oracle/ref_shim/op_lib_core.h``, when the reference sources are
  present (``OP2B_REFERENCE``, else the read-only checkout this recipe was
  written against).  The reference's build
  system is not used: its other native parts need OP2-Common and PETSc, which
  are not available, so only this one translation unit is compiled.
* ``oracle/_ref/plan<ext>``: the reference's own ``pyop2/plan.pyx``
  translated unmodified by Cython (``-2``: the Python 2 language level it was
  written for; the generated C lives in a temporary directory removed after
  the build) and compiled with gcc as a CPython extension.  ``oracle/reference.py`` imports it with
  stand-ins for the two modules it imports (``base``, ``utils``).
"""

import os
import subprocess
import sys
import sysconfig

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
REF_OUT = os.path.join(HERE, "_ref")
# Where the reference sources are read from.  This recipe (and the fixture
# generators under tests/golden/, which import this name) is the only code
# that reads them; nothing at test or bench time does.  When the directory is
# absent the reference builds are skipped and the prebuilt files are used.
REFERENCE = os.environ.get("OP2B_REFERENCE", "/root/reference")


def _stale(target, deps):
    return not os.path.exists(target) or any(os.path.getmtime(d) > os.path.getmtime(target)
                                             for d in deps)


def build_oracle(force=False):
    os.makedirs(BUILD, exist_ok=True)
    src = os.path.join(HERE, "csrc", "oracle_core.c")
    out = os.path.join(BUILD, "liboracle.so")
    if force or _stale(out, [src]):
        subprocess.check_call(["gcc", "-O2", "-std=gnu99", "-shared", "-fPIC", src, "-o", out])
    return out


def build_ref(force=False):
    """Compile the reference's sparsity_utils.cxx; None if it is absent."""
    src = os.path.join(REFERENCE, "pyop2", "sparsity_utils.cxx")
    if not os.path.exists(src):
        return None
    os.makedirs(REF_OUT, exist_ok=True)
    out = os.path.join(REF_OUT, "libref_sparsity.so")
    if force or _stale(out, [src]):
        subprocess.check_call(["g++", "-O2", "-shared", "-fPIC",
                               "-I" + os.path.join(HERE, "ref_shim"),
                               "-I" + os.path.join(REFERENCE, "pyop2"), src, "-o", out])
    return out


def build_ref_plan(force=False):
    """Translate and compile the reference's plan.pyx; None if it is absent."""
    src = os.path.join(REFERENCE, "pyop2", "plan.pyx")
    if not os.path.exists(src):
        return None
    import shutil
    import tempfile

    import numpy
    os.makedirs(REF_OUT, exist_ok=True)
    out = os.path.join(REF_OUT, "plan" + sysconfig.get_config_var("EXT_SUFFIX"))
    if force or _stale(out, [src]):
        tmp = tempfile.mkdtemp(prefix="op2b_refplan_")
        try:
            csrc = os.path.join(tmp, "plan.c")
            subprocess.check_call([sys.executable, "-m", "cython", "-2", src, "-o", csrc])
            subprocess.check_call(["gcc", "-O2", "-shared", "-fPIC", "-w",
                                   "-I" + sysconfig.get_paths()["include"], "-I" + numpy.get_include(),
                                   csrc, "-o", out])
        finally:
            shutil.rmtree(tmp, ignore_errors=True)
    return out


def ref_plan_path():
    p = os.path.join(REF_OUT, "plan" + sysconfig.get_config_var("EXT_SUFFIX"))
    return p if os.path.exists(p) else None


def ref_lib_path():
    p = os.path.join(REF_OUT, "libref_sparsity.so")
    return p if os.path.exists(p) else None


if __name__ == "__main__":
    print(build_oracle(force="--force" in sys.argv))
    print(build_ref(force="--force" in sys.argv))
    print(build_ref_plan(force="--force" in sys.argv))
