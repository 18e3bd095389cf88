"""B200 (sm_100a) implementation of the GATT_DNS per-RK4-stage hot path.

The compute path is the CUDA library ``libgatt_dns_b200.so`` behind the C-ABI declared in
``include/gatt_dns.h``; this package holds its ctypes binding (:mod:`._lib`), the host
mirror of the reference solver operations (:class:`GattDNS`), the coefficient emitter
restating the MATLAB preprocessing (:mod:`.matrices`) and the case builders
(:mod:`.case`).
"""
from .case import Case  # noqa: F401
from . import matrices  # noqa: F401


def GattDNS(*args, **kwargs):  # noqa: N802 - keeps the import of the CUDA binding lazy
    from .solver import GattDNS as _G
    return _G(*args, **kwargs)
