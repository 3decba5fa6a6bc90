"""Run-time configuration, mirroring hotspice/config.py.

The engine is CUDA-only (sm_100a): ``USE_GPU`` is always True and there is no NumPy path.
``DEVICE_ID`` (``HOTSPICE_DEVICE_ID``) selects the CUDA device, as in the reference.
"""
import os

__all__ = ['USE_GPU', 'DEVICE_ID', 'get_dict']

USE_GPU = True
DEVICE_ID = os.environ.get('HOTSPICE_DEVICE_ID', None)
DEVICE_ID = int(DEVICE_ID.split(',')[0]) if isinstance(DEVICE_ID, str) else None


def get_dict():
    return {'USE_GPU': USE_GPU, 'DEVICE_ID': DEVICE_ID}
