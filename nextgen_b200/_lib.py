"""Locating and loading the package's in-tree shared libraries."""
import ctypes
import os

LIB_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib")

_cache = {}


def path(name):
    return os.path.join(LIB_DIR, name)


def load(name):
    """Load nextgen_b200/lib/<name>; raise a clear error if it was not built."""
    if name in _cache:
        return _cache[name]
    p = path(name)
    if not os.path.exists(p):
        raise OSError("%s not found: build the package first (python -c 'import "
                      "__graft_entry__ as g; g.build()')" % p)
    lib = ctypes.CDLL(p, mode=ctypes.RTLD_GLOBAL)
    _cache[name] = lib
    return lib
