"""LigeSIS / Basefold prover for NVIDIA B200 (sm_100a).

The compute path is liblgs.so (hand-written CUDA, C ABI in include/lgs.h); this package is the
Python host mirror of the reference's API for the path (paulguoyanpei/ligesis:
pcs/src/ligesis.rs, pcs/src/subset_sum.rs, utils/src/poly.rs, utils/src/oracle.rs).
"""
from ._lib import Context, DeviceTimeout, LgsError, OracleExhausted, ShapeError, load
from .ligesis import (
    CODE_RATE,
    C_ROWS,
    ETA,
    NUM_COLS_OPENED,
    CommitData,
    Ligesis,
    LigesisCommit,
    LigesisProof,
    MlPoly,
    ProvingKey,
    RandomOracle,
    SubsetSumHash,
    VerifyingKey,
    dft,
    merkle_root,
    oracle_need,
    shape_ok,
    sumcheck_prove,
)
from .basefold import Basefold, BasefoldCommit, BasefoldProof, BasefoldProverState
from .logup import (FracSum, FracSumProof, Lookup, LookupProof, OpeningClaim, Poly,
                    multiplicity_vector)
from . import proofsys
from .pcs import BasefoldPcs, LigesisPcs, NoopCommit, NoopPcs
from .rng import SeededRng

__all__ = [
    "Basefold", "BasefoldCommit", "BasefoldPcs", "BasefoldProof", "BasefoldProverState",
    "CODE_RATE", "FracSum", "FracSumProof", "Lookup", "LookupProof", "OpeningClaim", "Poly",
    "multiplicity_vector", "LigesisPcs", "NoopCommit", "NoopPcs", "C_ROWS", "ETA", "NUM_COLS_OPENED", "CommitData", "Context", "DeviceTimeout", "LgsError",
    "Ligesis", "LigesisCommit", "LigesisProof", "MlPoly", "OracleExhausted", "ProvingKey",
    "RandomOracle", "SeededRng", "ShapeError", "SubsetSumHash", "VerifyingKey", "dft", "load",
    "merkle_root", "oracle_need", "shape_ok", "sumcheck_prove",
]
