"""Build recipe for the CPU oracle (test infrastructure only).

* ``oracle/_build/liboracle.so``   from ``oracle/restated.c`` (this project's restatement).
* ``oracle/_ref/libctools_ref.so`` from the reference's own ``fem_c/ctools.c``, compiled where
  it lies in the reference checkout, with the reference's flags (``build.py:14-20``: ``-O3``)
  minus ``-fopenmp`` (libgomp's spec file is missing in this image; every OpenMP pragma on
  the hot path is commented out in the reference, so the result is behaviour-identical).

Run ``python oracle/build_oracle.py [--reference DIR]`` (or call ``build()``).  The reference
checkout is found from ``--reference``, else the environment variable ``SNOOPY_REFERENCE``, else
its location in the build container; it is only needed for ``_ref``, and where it is absent the
prebuilt ``_ref`` library is used as is.
"""

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def reference_root(argv=None):
    """The reference checkout: ``--reference DIR`` in argv, else $SNOOPY_REFERENCE, else the
    build container's checkout."""
    argv = sys.argv if argv is None else argv
    if "--reference" in argv:
        return argv[argv.index("--reference") + 1]
    return os.environ.get("SNOOPY_REFERENCE", "/root/reference")


LIB_ORACLE = os.path.join(HERE, "_build", "liboracle.so")
LIB_REF = os.path.join(HERE, "_ref", "libctools_ref.so")


def _newer(target, *sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources if os.path.exists(s))


def build(force=False, verbose=False, reference=None):
    fem_c = os.path.join(reference or reference_root([]), "fem_c")
    os.makedirs(os.path.dirname(LIB_ORACLE), exist_ok=True)
    src = os.path.join(HERE, "restated.c")
    if force or _newer(LIB_ORACLE, src):
        cmd = ["gcc", "-O2", "-fPIC", "-shared", "-o", LIB_ORACLE, src, "-lm"]
        if verbose:
            print(" ".join(cmd))
        subprocess.check_call(cmd)
    ref_src = os.path.join(fem_c, "ctools.c")
    if os.path.exists(ref_src):
        os.makedirs(os.path.dirname(LIB_REF), exist_ok=True)
        if force or _newer(LIB_REF, ref_src):
            cmd = ["gcc", "-O3", "-fPIC", "-shared", "-w", "-I", fem_c, "-o", LIB_REF, ref_src, "-lm"]
            if verbose:
                print(" ".join(cmd))
            subprocess.check_call(cmd)
    return LIB_ORACLE, (LIB_REF if os.path.exists(LIB_REF) else None)


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True, reference=reference_root()))
