"""Locate and load the in-tree native libraries.

libjq_frontend.so  host-side script front end (C++), include/jacquard_frontend.h
libjacquard_b200.so  sm_100a interpreter kernels + C ABI, include/jacquard_b200.h

Both are built in-tree by jacquard_b200.build (``__graft_entry__.build()``).
Loading never falls back to anything else: a missing library raises.
"""
import ctypes
import os

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
REPO_DIR = os.path.dirname(PKG_DIR)

_cache = {}


def lib_path(name):
    return os.path.join(PKG_DIR, name)


def load(name):
    if name in _cache:
        return _cache[name]
    path = lib_path(name)
    if not os.path.exists(path):
        raise RuntimeError(
            f"{name} is not built ({path}); run `python -c 'import __graft_entry__ as g; g.build()'`")
    lib = ctypes.CDLL(path)
    _cache[name] = lib
    return lib
