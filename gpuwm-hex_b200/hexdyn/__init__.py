"""hexdyn: B200-native MPAS-A v8.4.2 dry-plus-tracer dycore step.

Python host code over a C ABI (include/hexdyn.h) to hand-written sm_100a
CUDA kernels; PyTorch is used only for device tensors and streams.
"""

from .config import ConfigurationRefusal, DycoreConfig
from .driver import DeviceStepResult, HexDycoreDriver, HostSidecar, HostState, HostStepResult
from .ensemble import HexEnsemble, assign_members, step_batched

__all__ = [
    "ConfigurationRefusal",
    "DycoreConfig",
    "DeviceStepResult",
    "HexDycoreDriver",
    "HexEnsemble",
    "HostSidecar",
    "HostState",
    "HostStepResult",
    "assign_members",
    "from_case",
    "step_batched",
]


def from_case(case, config: DycoreConfig, **kwargs) -> HexDycoreDriver:
    """Driver for a synthetic ``hexdyn.case.DycoreCase`` (which carries the
    state, reference, terrain, advection and wind inputs under the
    reference's attribute names)."""
    return HexDycoreDriver.from_host(case.mesh, case, case.vertical, case, config,
                                     terrain_metrics=case, advection_coefficients=case,
                                     reference_wind_profiles=case, **kwargs)
