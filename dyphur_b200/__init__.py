"""B200-native dyphur frame step."""
import os as _os
import sys as _sys

LIB_DIR = _os.path.join(_os.path.dirname(_os.path.abspath(__file__)), "lib")


def import_dyphur_py():
    """Import the dyphur_py extension module (built into dyphur_b200/lib)."""
    if LIB_DIR not in _sys.path:
        _sys.path.insert(0, LIB_DIR)
    import dyphur_py
    return dyphur_py
