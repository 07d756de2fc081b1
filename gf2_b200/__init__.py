"""gf2_b200: B200-native (sm_100a) batched LDPC encoder / decoder.

A drop-in for the belief-propagation path of erankavija/gf2's gf2-coding crate.
The compute runs in libgf2cuda.so (hand-written CUDA for sm_100a) behind the C
ABI of include/gf2cuda.h; this package is the host-side mirror of the
reference's Rust API over that ABI.
"""
from . import _capi
from .bch import BchCode, BchDecoder, BchEncoder
from . import gf2io
from .gf2io import DenseEncoder, EncodingCache
from .ldpc import (AwgnChannel, BpskModulator, CirculantMatrix, CodeRate, DecoderResult, FrameSize, Llr,
                   LdpcCode, LdpcDecoder, LdpcEncoder, QuasiCyclicLdpc, awgn_frames, judge_spa64, pack_bits,
                   sigma2_from_ebn0, unpack_bits, words)

ALGO_MINSUM = _capi.ALGO_MINSUM
ALGO_SPA = _capi.ALGO_SPA
ALGO_NMS = _capi.ALGO_NMS
ALGO_SPA_FAST = _capi.ALGO_SPA_FAST
SCHED_FLOODING = _capi.SCHED_FLOODING
SCHED_LAYERED = _capi.SCHED_LAYERED
MSG_F32 = _capi.MSG_F32
MSG_F16 = _capi.MSG_F16
Gf2cError = _capi.Gf2cError

__all__ = ["BchCode", "BchDecoder", "BchEncoder", "DenseEncoder", "EncodingCache", "gf2io", "AwgnChannel", "BpskModulator", "CirculantMatrix", "CodeRate", "DecoderResult", "FrameSize", "Llr",
           "LdpcCode", "LdpcDecoder", "LdpcEncoder", "QuasiCyclicLdpc", "awgn_frames", "judge_spa64", "pack_bits",
           "sigma2_from_ebn0", "unpack_bits", "words", "ALGO_MINSUM", "ALGO_SPA", "ALGO_NMS", "ALGO_SPA_FAST", "SCHED_FLOODING",
           "SCHED_LAYERED", "MSG_F32", "MSG_F16", "Gf2cError"]
