"""tenax_b200: B200-native block-sparse symmetric contraction for tenax.

Drop-in GPU path for tenax's ``SymmetricTensor`` contraction and the
two-site DMRG H_eff matvec built on it, the dense CTMRG step with a
hand-written adjoint and the block-sparse CTMRG: the same names and
argument meanings as ``tenax.contract``, ``SymmetricTensor``/``TensorIndex``,
``dmrg()``, ``ctm()``/``compute_energy_ctm()`` and
``ctm_tensor()``/``compute_energy_ctm_tensor()``; arithmetic runs in this
package's sm_100a kernels through the C ABI in ``include/tenax_b200.h``.
"""

from tenax_b200 import _capi  # noqa: F401  (loads libtenax_b200.so or raises)
from tenax_b200.core import (  # noqa: F401
    BaseSymmetry,
    FermionicU1,
    FermionParity,
    FlowDirection,
    Label,
    TensorIndex,
    U1Symmetry,
    ZnSymmetry,
)
from tenax_b200.tensor import SymmetricTensor, compute_valid_blocks, inner  # noqa: F401
from tenax_b200.contraction import (  # noqa: F401
    blockwise_contract,
    contract,
    contract_ad,
    contract_with_subscripts,
)
from tenax_b200.heff import HeffBatch, HeffOperator  # noqa: F401
from tenax_b200.netfile import NetworkBlueprint, from_netfile, parse_netfile  # noqa: F401
from tenax_b200.ipeps import (  # noqa: F401
    CTMConfig,
    CTMEnvironment,
    compute_energy_ctm,
    compute_energy_ctm_2site,
    ctm,
)
from tenax_b200.tensor_ctm import (  # noqa: F401
    CTMTensorEnv,
    compute_energy_ctm_tensor,
    compute_energy_ctm_tensor_2site,
    ctm_tensor,
    ctm_tensor_2site,
    initialize_ctm_tensor_env,
)

EPS = 1e-15
LOG_EPS = 1e-250
