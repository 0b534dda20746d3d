"""pamtra_b200 -- B200-native passive microwave forward path of PAMTRA.

User surface mirrors the reference's ``pyPamtra`` package: ``pyPamtra``
(session), ``importer`` (profile builders), ``descriptorFile``.
"""

__version__ = "0.1.0"

from . import importer  # noqa: F401
from .core import pyPamtra  # noqa: F401
from .descriptorFile import pamDescriptorFile  # noqa: F401
