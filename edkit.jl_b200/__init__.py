"""edkit_b200 — B200 (sm_100a) implementation of EDKit.jl's matrix-free
operator application and the Lanczos / Krylov loops built on it.

The compute path is libedk.so (hand-written CUDA behind the C ABI in
include/edk.h); this package is the Python mirror of the reference's Julia API.
"""
from ._lib import EDKError, load as _load
from .algorithms import (KrylovEvolutionCache, KrylovEvolutionDiagnostics, batch_lanczos_e0,
                         block_lanczos, gapratio, ground_state, lanczos_e0, meangapratio,
                         productstate, timeevolve, tridiag_eigen)
from .basis import (AbelianBasis, AbstractBasis, FlipBasis, ParityBasis, ParityFlipBasis,
                    ProjectedBasis, TensorBasis, TranslationalBasis, TranslationFlipBasis,
                    TranslationParityBasis, basis)
from .entanglement import DoubleBasis, ent_S, ent_spec, entropy, schmidt, symmetrizer
from .operator import Operator, mul, mul_, operator, spin, trans_inv_operator, σ

__all__ = [
    "EDKError", "TensorBasis", "ProjectedBasis", "TranslationalBasis", "TranslationParityBasis",
    "AbelianBasis", "AbstractBasis", "ParityBasis", "FlipBasis", "ParityFlipBasis",
    "TranslationFlipBasis", "basis", "spin", "σ", "operator", "trans_inv_operator",
    "Operator", "mul", "mul_", "lanczos_e0", "ground_state", "batch_lanczos_e0", "block_lanczos",
    "timeevolve", "KrylovEvolutionCache",
    "tridiag_eigen", "gapratio", "meangapratio", "productstate", "KrylovEvolutionDiagnostics", "version",
    "schmidt", "ent_spec", "entropy", "ent_S", "DoubleBasis", "symmetrizer",
]


def version():
    return _load().edk_version().decode()
