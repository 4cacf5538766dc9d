"""Test infrastructure: where the reference source tree (Yahiahu/Lagbound) is, for the scripts that run the
reference itself (tests/golden/make_golden.py, oracle/reference_chain.py).

The tree is taken from $LAGBOUND_REF, else from an importable `lagbound` package laid out as in the reference
project (<root>/src/lagbound/__init__.py with <root>/src/lagbound/_core beside it).  There is no default path: a
script that needs the reference stops with a message when neither is available.
"""
import importlib.util
import os


def reference_root():
    env = os.environ.get("LAGBOUND_REF")
    if env:
        if not os.path.isdir(os.path.join(env, "src", "lagbound", "_core")):
            raise SystemExit(f"LAGBOUND_REF={env} does not hold src/lagbound/_core of the reference project")
        return env
    spec = importlib.util.find_spec("lagbound")
    if spec is not None and spec.origin:
        pkg = os.path.dirname(spec.origin)
        root = os.path.dirname(os.path.dirname(pkg))
        if os.path.isdir(os.path.join(pkg, "_core")) and os.path.basename(os.path.dirname(pkg)) == "src":
            return root
    raise SystemExit("the reference source tree was not found: set LAGBOUND_REF to its root (the directory holding "
                     "src/lagbound/_core) or put its src/ on PYTHONPATH")
