"""Where the reference tree lies, for the recipes that compile the checkers
from it (oracle/Makefile, tests/cpp/Makefile) and the tests that read its
headers.  SELDON_REF overrides the default location; where neither exists
(a GPU host) the prebuilt checkers are used as they are."""
import os

DEFAULT = "/root/reference"


def reference_tree():
    return os.environ.get("SELDON_REF") or DEFAULT


def have_reference():
    return os.path.isfile(os.path.join(reference_tree(), "Seldon.hxx"))
