"""tenrso_b200 — a B200-native (sm_100a) CP-ALS hot path for tenrso.

The product is the CUDA library libtenrso_b200.so behind the C ABI in
include/tenrso_b200.h. This package is its Python host mirror (the tests and
bench.py drive the library through it) plus the seeded input generators.
"""
from ._lib import TenrsoError, load  # noqa: F401
from .dense import (  # noqa: F401
    Context,
    ConvergenceInfo,
    CpDecomp,
    cp_als,
    cp_als_dev,
    cp_als_f64,
    mttkrp_f64,
    cp_als_accelerated,
    cp_als_accelerated_dev,
    default_context,
    gram_inverse,
    initialize_factors,
    khatri_rao,
    mttkrp,
    mttkrp_all_modes,
    mttkrp_blocked,
    mttkrp_blocked_parallel,
    mttkrp_dev,
    mttkrp_fused,
    mttkrp_fused_parallel,
    profile_mttkrp_dev,
)

from .sparse import (  # noqa: F401
    CooError,
    CooTensor,
    CsfError,
    CsfTensor,
    HiCooTensor,
    SparseTensor,
    coo_deduplicate_dev,
    synth_zipf_coo_dev,
)

from .constrained import (  # noqa: F401
    CpConstraints,
    RegularizationType,
    cp_als_constrained,
    cp_als_constrained_dev,
)

from .sparse_io import (  # noqa: F401
    MatrixMarketHeader,
    SparseIoError,
    read_matrix_market,
    read_tns,
    write_matrix_market,
    write_tns,
)

from .adjoint import (  # noqa: F401
    CpReconstructionGrad,
    CpReconstructionOp,
    DenseTensor,
    cp_loss_grad,
    cp_reconstruct,
    cp_reconstruct_dev,
    cp_residual_dev,
    reconstruction_grad_dev,
)

from .batched import BatchedCpAls  # noqa: F401

__version__ = "0.1.0"

from .tucker import (  # noqa: F401
    nmode_product,
    nmode_products_seq,
    tucker_operator,
    tucker_operator_ordered,
    tucker_reconstruct,
)
