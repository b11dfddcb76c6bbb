"""B200-native graph-index builder, a drop-in for ZJU-DAILY/Tagore's Python API.

`tagore_b200.Tagore` (compiled module) mirrors `import Tagore`; the C ABI is
bound in `tagore_b200.capi`. Build with `python -m tagore_b200.build`.
"""
import os as _os
import sys as _sys

_HERE = _os.path.dirname(_os.path.abspath(__file__))


def load_tagore():
    """Imports the compiled `Tagore` module from this package (fails loudly
    when it has not been built)."""
    if _HERE not in _sys.path:
        _sys.path.insert(0, _HERE)
    import Tagore  # noqa: F401
    return Tagore
