"""Where the reference's sources are, for the recipes that compile or read them.

The reference location comes from the environment variable
FUNDEM_REFERENCE_ROOT; when it is unset, the checkout location the build
recipes use by convention is tried.  None when neither holds the reference
(for example on a machine that only runs the prebuilt checkers): callers
skip what needs the sources.

Test infrastructure: only the oracle recipes, tests and the build step use it.
"""
import os

ENV = "FUNDEM_REFERENCE_ROOT"
_CONVENTIONAL = "/root/reference"


def reference_root():
    for cand in (os.environ.get(ENV), _CONVENTIONAL):
        if cand and os.path.isfile(os.path.join(cand, "kernel", "LSSolver.h")):
            return cand
    return None


def reference_path(*parts):
    """A path inside the reference, or None when the reference is absent."""
    root = reference_root()
    return os.path.join(root, *parts) if root else None
