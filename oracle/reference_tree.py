"""Location of the reference's sources in the build container, for the checks
that read them there (the compile check of the hpGEM-side adapter).  Test
infrastructure: nothing on the product path imports it.  The environment
variable HPGEM_SOURCE_DIR overrides the default location."""
import os

DEFAULT = "/root/reference"


def kernel_include_dir():
    """hpGEM's kernel/ header tree, or None where the sources are absent."""
    root = os.environ.get("HPGEM_SOURCE_DIR", DEFAULT)
    d = os.path.join(root, "kernel")
    return d if os.path.isfile(os.path.join(d, "Base", "HpgemAPISimplified.h")) else None
