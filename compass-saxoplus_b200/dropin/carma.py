"""Drop-in `carma` module for COMPASS's shesha: the parts of the reference's
pybind11 `carma` module (python_module/carma/src/carma.cpp; context in
python_module/carma/src/context.cpp) that the hot path touches, over
libaob200.

* ``context``: the device context handed to every sutra constructor
  (get_instance, get_instance_1gpu, get_instance_ngpu, activate_device).
* device arrays: the sutra objects here expose ``aob200.core.DeviceArray``
  views; ``np.array(view)`` copies to the host as ``np.array(carma_obj)`` does.

Put this directory first on ``sys.path`` (or ``PYTHONPATH``) so that
``import carma`` / ``import sutra`` resolve here.
"""

from __future__ import annotations

import os
import sys

_PKG = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if _PKG not in sys.path:
    sys.path.insert(0, _PKG)

from aob200 import _lib  # noqa: E402
from aob200.core import DeviceArray  # noqa: E402,F401  (the carma_obj stand-in)


class context:
    """CarmaContext: the GPUs this process drives and the active one."""

    _instance = None

    def __init__(self, devices=None):
        n = _lib.device_count()
        self.devices = list(devices) if devices is not None else list(range(max(n, 1)))
        self.active_device = self.devices[0]

    @classmethod
    def get_instance(cls):
        if cls._instance is None:
            cls._instance = cls()
        return cls._instance

    @classmethod
    def get_instance_1gpu(cls, dev):
        cls._instance = cls([int(dev)])
        return cls._instance

    @classmethod
    def get_instance_ngpu(cls, ngpu, devices):
        cls._instance = cls([int(d) for d in list(devices)[: int(ngpu)]])
        return cls._instance

    @property
    def ndevice(self):
        return len(self.devices)

    def activate_device(self, dev, silent=True):
        if int(dev) not in self.devices:
            raise ValueError(f"device {dev} is not in this context")
        self.active_device = int(dev)

    def get_device(self, dev):
        return int(dev)

    @property
    def active_device_id(self):
        return self.active_device
