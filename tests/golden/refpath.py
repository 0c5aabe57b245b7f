"""Location of the reference checkout (PacesaLab/XPG) that the fixture generators import: the XPG_REFERENCE_ROOT
environment variable (the directory holding the `xpg` package). Only the generators use it; the tests read the
committed fixtures."""
from __future__ import annotations

import os
import sys


def reference_root():
    root = os.environ.get("XPG_REFERENCE_ROOT")
    if not root or not os.path.isdir(os.path.join(root, "xpg")):
        raise SystemExit("set XPG_REFERENCE_ROOT to the reference checkout (the directory that holds the xpg package)")
    return root


def import_reference():
    """Puts the reference checkout first on sys.path (its `xpg` package then imports) and returns its root."""
    root = reference_root()
    if root not in sys.path:
        sys.path.insert(0, root)
    return root
