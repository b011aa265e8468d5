"""Import name for the package in ``gkmsvm-lite_b200/``.

A directory name with a hyphen is not importable, so this module loads the
package from that directory under the name ``gkmsvm_lite_b200`` and puts it
in ``sys.modules``; ``import gkmsvm_lite_b200`` and its submodules then
resolve to the package itself.
"""

import importlib.util
import os
import sys

_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "gkmsvm-lite_b200")
_spec = importlib.util.spec_from_file_location(
    __name__, os.path.join(_DIR, "__init__.py"), submodule_search_locations=[_DIR]
)
_pkg = importlib.util.module_from_spec(_spec)
sys.modules[__name__] = _pkg
_spec.loader.exec_module(_pkg)
