"""ziros_b200 — B200 (sm_100a) polynomial-commitment path for ZirOS-style STARK proving.

Coset NTT / low-degree extension, Poseidon2 Merkle commitment and FRI folding over
BabyBear and Goldilocks, as CUDA kernels behind the C ABI of include/zkb200.h.
This package is the host-side mirror of the reference's accelerator types.
"""
from ._native import ZkbDeclined, ZkbError, device_count, load  # noqa: F401
from .accel import (  # noqa: F401
    BABYBEAR,
    BatchCommit,
    Challenger,
    CommitEngine,
    GOLDILOCKS,
    CudaDft,
    CudaFri,
    CudaFriProver,
    FriProof,
    combine_columns_dev,
    CudaMerkleTreeMmcs,
    CudaNttAccelerator,
    CudaPolyOps,
    CudaPoseidon2,
    CudaTwoAdicPcs,
    ProverRuntime,
    Tree,
    round_constants,
)
