"""Backend registry (backend.py:18-41 of the reference) with the B200 backend.

``resolve_backend('b200')`` returns (torch, float64) after checking that a
CUDA device is present and the sm_100a library loads; there is no fallback to
NumPy or to PyTorch arithmetic.  'cpu' is not served here -- the reference
package itself is the CPU path.
"""

import numpy as np

_BACKENDS = {"b200": "torch+libspt_b200"}


def resolve_backend(name):
    if name not in _BACKENDS:
        raise ValueError(f"Unknown backend {name!r}; choose from {sorted(_BACKENDS)}")
    import torch

    if not torch.cuda.is_available():
        raise RuntimeError("backend='b200' needs a CUDA device (B200, sm_100a)")
    from . import _lib
    _lib.lib()
    return torch, np.dtype("float64")


def to_numpy(array):
    """Bring an array back to NumPy, whatever produced it (backend.py:44-46)."""
    if hasattr(array, "detach"):
        return array.detach().cpu().numpy()
    return np.asarray(array)
