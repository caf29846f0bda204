"""Drop-in for ``detnqs.operator`` on the Hamiltonian path
(reference ``detnqs/operator/__init__.py:118-153``): builders and H.psi
operators on device-resident blocks.  ``make_energy_step`` (the JAX
energy functional) consumes these operators unchanged and is not part of
this package."""

from .hamiltonian import (
    DeviceBlock,
    DiagonalInfo,
    ProxyHamiltonian,
    VVHamiltonian,
    build_effective_hamiltonian,
    build_proxy_hamiltonian,
    build_vv_hamiltonian,
)
from .kernel import (
    ProxyContraction,
    VVContraction,
    build_proxy_operator,
    build_vv_operator,
    local_energy,
)

__all__ = [
    "DiagonalInfo",
    "DeviceBlock",
    "VVHamiltonian",
    "ProxyHamiltonian",
    "build_vv_hamiltonian",
    "build_proxy_hamiltonian",
    "build_effective_hamiltonian",
    "VVContraction",
    "ProxyContraction",
    "build_vv_operator",
    "build_proxy_operator",
    "local_energy",
]
