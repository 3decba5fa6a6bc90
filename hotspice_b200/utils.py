"""Host-side helpers mirroring hotspice/utils.py (the parts the hot path needs)."""
from __future__ import annotations

import math

import numpy as np
import torch


def as_2D_array(value, shape) -> np.ndarray:
    """Scalar -> constant array; array with prod(shape) values -> reshaped
    (hotspice/utils.py:208-228). Always a float64 numpy array on the host."""
    if isinstance(value, torch.Tensor):
        value = value.detach().cpu().numpy()
    if isinstance(value, list):
        try:
            value = np.asarray(value, dtype=float)
        except ValueError:
            raise ValueError("List of lists could not be converted to rectangular float64 array.")
    if isinstance(value, np.ndarray) and value.size != 1:
        if value.size != math.prod(shape):
            raise ValueError(f"Incorrect shape: passed array of shape {value.shape} is not of desired shape {shape}.")
        return np.asarray(value, dtype=float).reshape(shape)
    return np.ones(shape, dtype=float) * float(np.asarray(value).reshape(-1)[0] if isinstance(value, np.ndarray) else value)


def lower_than(x, y, rtol=1e-10):
    """False if x is within rtol of y or larger (hotspice/utils.py:90-92)."""
    if math.isinf(y):  # numpy.isclose: an infinite y is close only to itself
        return x < y
    return x < y and not (abs(x - y) <= rtol * abs(y))


def check_repetition(arr, nx: int, ny: int) -> bool:
    """True if ``arr`` is periodic with period nx along axis 1 and ny along axis 0: every
    element close (numpy.allclose) to the element of the leading ny x nx block at the same
    phase (hotspice/utils.py:42-66). The block is checked against regions that double in
    alternating directions, y first, as there, so a wrong period is usually rejected on a
    small region; each region takes an exact comparison before the tolerance one."""
    arr = np.asarray(arr)
    H, W = arr.shape[:2]
    base = arr[:ny, :nx, ...]
    h, w = base.shape[:2]
    i = 0
    while h < H or w < W:
        if i % 2:   # columns [w, 2w) of rows [0, h)
            y0, y1, x0, x1 = 0, min(h, H), w, min(2 * w, W)
            w *= 2
        else:       # rows [h, 2h) of columns [0, w)
            y0, y1, x0, x1 = h, min(2 * h, H), 0, min(w, W)
            h *= 2
        i += 1
        if y1 <= y0 or x1 <= x0:
            continue
        a = arr[y0:y1, x0:x1, ...]
        b = base[np.ix_(np.arange(y0, y1) % ny, np.arange(x0, x1) % nx)]
        if not (np.array_equal(b, a) or np.allclose(b, a)):
            return False
    return True


_NP_OF = {torch.int8: np.int8, torch.int32: np.int32, torch.int64: np.int64, torch.float32: np.float32,
          torch.float64: np.float64, torch.uint8: np.uint8}


def to_device(arr, device, dtype: torch.dtype | None = None) -> torch.Tensor:
    """A new contiguous device tensor holding ``arr`` (cast to ``dtype`` on the host), copied
    from a pinned staging buffer asynchronously on the current stream: the host does not wait
    for the stream, as it does for a copy from pageable memory. Same values as
    torch.as_tensor(arr, device=device, dtype=dtype)."""
    a = np.asarray(arr)
    if dtype is not None:
        a = a.astype(_NP_OF[dtype], copy=False)
    t = torch.from_numpy(np.ascontiguousarray(a))
    return t.pin_memory().to(device, non_blocking=True)


def copy_to_device(dst: torch.Tensor, arr) -> torch.Tensor:
    """dst.copy_(arr) from a pinned staging buffer, asynchronously on the current stream."""
    a = np.ascontiguousarray(np.asarray(arr).astype(_NP_OF[dst.dtype], copy=False))
    dst.copy_(torch.from_numpy(a).pin_memory().reshape(dst.shape), non_blocking=True)
    return dst


def full_obj_name(obj) -> str:
    cls = type(obj)
    return f'{cls.__module__}.{cls.__qualname__}'


def asnumpy(array) -> np.ndarray:
    if isinstance(array, torch.Tensor):
        return array.detach().cpu().numpy()
    return np.asarray(array)
