"""kira_ls_aligner_b200 -- B200-native (sm_100a) candidate verification for
kira-ls-aligner: 2-bit multi-shift Hamming sieve, Myers bounded edit distance and
banded affine Smith-Waterman with CIGAR traceback, as CUDA kernels behind the C
ABI of include/kira_gpu.h (libkira_gpu.so). The Python modules are the host side
of that boundary; there is no CPU compute path in this package.
"""
from . import _abi
from .runtime import (AlignmentConfig, CapacityError, CudaError, GpuContext, InvalidArgument,
                      PairBatch, PrefilterConfig, Server, SwPublicResult, Ticket, Timeout, VerifyParams,
                      WfaParams, cigar_string, decode_cigar, is_available, results_to_list)

__all__ = ["AlignmentConfig", "CapacityError", "CudaError", "GpuContext", "InvalidArgument",
           "PairBatch", "PrefilterConfig", "Server", "SwPublicResult", "Ticket", "Timeout", "VerifyParams",
           "WfaParams", "cigar_string", "decode_cigar", "is_available", "results_to_list", "_abi"]
