"""``curig`` drop-in: the reference package name (python/curagridder, installed
as ``curig`` by its setup.py) served by cugridder_b200.  ``from curig import
ms2dirty, dirty2ms`` and ``vis2dirty``/``dirty2vis`` keep working unchanged
(reference python/curagridder/__init__.py)."""
from cugridder_b200.curagridder import *  # noqa: F401,F403
from cugridder_b200.curagridder import vis2dirty, dirty2vis  # noqa: F401
from cugridder_b200.cursl import ms2dirty, dirty2ms  # noqa: F401
