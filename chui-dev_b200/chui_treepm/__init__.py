"""B200-native TreePM gravity solver (CUDA kernels behind a C-ABI).

Host-side mirror of the reference's TreePmCoordinator interface; see
chui_treepm.solver. The CUDA library is chui-dev_b200/_build/libchui_treepm.so.
"""
from . import _abi, softening
from .config import config_from_param_file, config_from_param_text
from .sharded import ShardedTreePm
from .solver import (AllocationError, DeviceError, InvalidArgument, NotSupported, OutOfRange, StateError,
                     TreePmConfig, TreePmCoordinator, TreePmError, kdk_factors_lcdm, kdk_factors_static,
                     probe_fp32_peak_tflops)

__all__ = [
    "TreePmConfig", "TreePmCoordinator", "TreePmError", "InvalidArgument", "OutOfRange", "StateError",
    "DeviceError", "AllocationError", "NotSupported", "config_from_param_file", "config_from_param_text",
    "kdk_factors_static", "kdk_factors_lcdm", "probe_fp32_peak_tflops", "ShardedTreePm", "_abi", "softening",
]
