"""Where the reference's source tree is read from when it is present: the
TNBP_REFERENCE environment variable, else the default mount point.  Test
infrastructure only (fixture generation, host-parity tests and the oracle
build); nothing on the product path reads the reference."""
import os

DEFAULT = "/root/reference"


def reference_root():
    return os.environ.get("TNBP_REFERENCE", DEFAULT)


def reference_file(*parts):
    """Path of a file inside the reference tree (it may not exist)."""
    return os.path.join(reference_root(), *parts)
