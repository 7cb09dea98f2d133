"""nexd_b200: B200-native time stepping for NEXD-3D's nodal-DG elastic solver.

Host side (libnexd_host.so): single-partition mesher / solver set-up that
builds the ``nexd_desc`` of include/nexd.h.  Device side (libnexd.so): the
sm_100a kernels behind nexd_create / nexd_run / nexd_get_traces.
"""
from ._abi import NEXD_NCOMP  # noqa: F401
from .host import Mesh, NexdError  # noqa: F401
