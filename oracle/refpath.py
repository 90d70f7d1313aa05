"""Where the reference source tree lives (TEST INFRASTRUCTURE ONLY).

The oracle build (oracle/Makefile), the fixture generators under
tests/golden/ and the CPU tests that read the reference's own example
goldens all take the reference tree from the environment variable
JURASSIC_REFERENCE; this module holds its one default.  On a machine
without the reference tree (a GPU box) nothing here is read: the prebuilt
oracle libraries under oracle/_ref and the committed fixtures are used.
"""
import os

DEFAULT = "/root/reference"


def reference_dir():
    """The reference tree: $JURASSIC_REFERENCE, else the default."""
    return os.environ.get("JURASSIC_REFERENCE", DEFAULT)


def reference_path(*parts):
    return os.path.join(reference_dir(), *parts)


def available():
    """True where the reference's sources are present."""
    return os.path.isdir(reference_path("src"))
