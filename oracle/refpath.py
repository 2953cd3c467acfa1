"""Where the ProFit source tree lies, for the recipes that read it in place.

The oracle's build (oracle/Makefile, driven by ``__graft_entry__.build``) and
the tests that read the tree's example data take the tree from the
PROFIT_REFERENCE environment variable, else from the location it has in the
container the oracle is built in.  Machines without the tree (where only the
prebuilt oracle libraries and the committed fixtures travel) see no tree and
skip what needs it.

Test infrastructure only.
"""
from __future__ import annotations

import os

_BUILD_CONTAINER_TREE = "/root/reference"


def reference_root() -> str:
    """The ProFit tree: $PROFIT_REFERENCE, else the build container's copy."""
    return os.environ.get("PROFIT_REFERENCE") or _BUILD_CONTAINER_TREE


def libprofit_sources() -> str:
    """libprofit's C++ sources inside the tree (src/libprofit/src/profit)."""
    return os.path.join(reference_root(), "src", "libprofit", "src", "profit")


def has_libprofit_sources() -> bool:
    return os.path.exists(os.path.join(libprofit_sources(), "model.cpp"))
