"""B200 (sm_100a) backend for three-avbd's 3D Augmented Vertex Block Descent step.

`CudaSolver3D` mirrors the reference's `GpuSolver3D` over the C ABI in include/avbd.h
(libavbd_cuda.so, built in-tree by three-avbd_b200/build.py); `scenes` builds the reference's
demo scenes and the synthetic workloads; `BatchSolver3D` steps many small worlds together.
"""

from . import pose_cache, scenes  # noqa: F401
from ._abi import AvbdError, DeviceError, DeviceTimeout, StorageCapacityError, BODY_DTYPE, CONTACT_DTYPE, INFO_DTYPE, JOINT_DTYPE, MANIFOLD_DTYPE, LIB_PATH, load  # noqa: F401
from .solver import CudaSolver3D, PoseCapture, device_info, find_pairs_noalloc, pack_bodies, pack_force, scene_records  # noqa: F401
from .batch import BatchSolver3D  # noqa: F401
from .adjoint import Adjoint  # noqa: F401
