"""protocell-genesis_b200: the soup MD step of nefayran/protocell-genesis on B200.

The compute path is hand-written sm_100a CUDA in csrc/, exported through the C ABI declared in
include/soup_b200.h (libsoup_b200.so, built in-tree by csrc/build.py).  This package is the Python
host: it resolves the reference's configuration (config.py) and mirrors the reference's SoupSystem
API (soup.py).  There is no CPU implementation behind it: without the library every call raises.
"""
from . import _abi, checkpoint, config, observables  # noqa: F401
from .config import SoupOptions, resolve  # noqa: F401
from .soup import SoupBatch, SoupSystem, create_soup, createSoup  # noqa: F401
