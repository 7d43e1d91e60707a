"""Where the golden-vector scripts find the reference checkout.

The path is the script's first argument or the CHIMERA_REFERENCE environment
variable; there is no default, so a script never reads a checkout it was not
pointed at."""
import os
import sys


def reference_path():
    path = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("CHIMERA_REFERENCE")
    if not path:
        sys.exit(f"usage: python {os.path.basename(sys.argv[0])} /path/to/reference "
                 "(or set CHIMERA_REFERENCE)")
    if not os.path.isdir(path):
        sys.exit(f"reference checkout not found: {path}")
    return path
