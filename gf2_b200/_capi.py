"""ctypes binding of libgf2cuda.so (the C ABI declared in include/gf2cuda.h).

There is no fallback: if the shared library is missing or fails to load,
importing the binding raises.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgf2cuda.so")

OK = 0
ERR_INVALID_ARG = 1
ERR_CUDA = 2
ERR_UNSUPPORTED = 3
ERR_NOMEM = 4
ERR_RANK = 5
ERR_KERNEL = 6
MEM_HOST = 0
MEM_DEVICE = 1
ALGO_MINSUM = 0
ALGO_SPA = 1
ALGO_NMS = 2
ALGO_SPA_FAST = 3
SCHED_FLOODING = 0
SCHED_LAYERED = 1
MSG_F32 = 0
MSG_F16 = 1

# Every symbol the header declares, for the load / export check.
EXPORTS = [
    "gf2c_decoder_opts_default", "gf2c_last_error", "gf2c_version",
    "gf2c_code_create_dvbt2", "gf2c_code_create_qc", "gf2c_code_create_edges",
    "gf2c_code_destroy", "gf2c_code_dims", "gf2c_code_csr", "gf2c_syndrome_batch",
    "gf2c_encode_batch", "gf2c_channel_awgn", "gf2c_sigma2_from_ebn0",
    "gf2c_decoder_create", "gf2c_decoder_create_multi", "gf2c_decoder_destroy",
    "gf2c_decode_batch", "gf2c_decode_batch_fallback", "gf2c_decode_mixed", "gf2c_decoder_last_launches", "gf2c_decode_batch_noalloc",
    "gf2c_judge_spa64",
    "gf2c_nms_trainer_create", "gf2c_nms_trainer_destroy", "gf2c_nms_trainer_layers", "gf2c_nms_trainer_set_schedule", "gf2c_nms_loss_grad",
    "gf2c_adam_step", "gf2c_count_errors",
    "gf2c_bch_create_dvbt2", "gf2c_bch_destroy", "gf2c_bch_dims", "gf2c_bch_generator",
    "gf2c_bch_encode_batch", "gf2c_bch_decode_batch",
    "gf2c_io_probe", "gf2c_io_write_bitvec", "gf2c_io_read_bitvec", "gf2c_io_write_bitmatrix",
    "gf2c_io_read_bitmatrix", "gf2c_io_write_sparse", "gf2c_io_read_sparse", "gf2c_code_create_file",
    "gf2c_io_write_code", "gf2c_siphash13", "gf2c_code_cache_hash", "gf2c_code_parity_part",
    "gf2c_dense_encoder_create", "gf2c_dense_encoder_destroy", "gf2c_dense_encode_batch",
]


class DecoderOpts(ctypes.Structure):
    _fields_ = [
        ("algorithm", ctypes.c_int32),
        ("schedule", ctypes.c_int32),
        ("msg_dtype", ctypes.c_int32),
        ("early_stop", ctypes.c_int32),
        ("nms_alpha", ctypes.POINTER(ctypes.c_float)),
        ("nms_beta", ctypes.POINTER(ctypes.c_float)),
        ("nms_iters", ctypes.c_int32),
        ("threads_per_block", ctypes.c_int32),
        ("blocks_per_sm", ctypes.c_int32),
    ]


class Gf2cError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"gf2cuda error {code}: {msg}")
        self.code = code


_vp = ctypes.c_void_p
_i32 = ctypes.c_int32
_i64 = ctypes.c_int64
_u64 = ctypes.c_uint64


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python gf2_b200/build.py`")
    L = ctypes.CDLL(LIB_PATH)
    L.gf2c_last_error.restype = ctypes.c_char_p
    L.gf2c_version.restype = ctypes.c_char_p
    L.gf2c_decoder_opts_default.argtypes = [ctypes.POINTER(DecoderOpts)]
    L.gf2c_decoder_opts_default.restype = None
    L.gf2c_code_create_dvbt2.argtypes = [_i32, _i32, ctypes.POINTER(_vp)]
    L.gf2c_code_create_qc.argtypes = [_vp, _i32, _i32, _i32, ctypes.POINTER(_vp)]
    L.gf2c_code_create_edges.argtypes = [_i64, _i64, _vp, _i64, ctypes.POINTER(_vp)]
    L.gf2c_code_destroy.argtypes = [_vp]
    L.gf2c_code_dims.argtypes = [_vp, _vp, _vp, _vp, _vp, _vp]
    L.gf2c_code_csr.argtypes = [_vp, _vp, _vp]
    L.gf2c_syndrome_batch.argtypes = [_vp, _vp, _i64, _vp, _vp, _i32, _vp]
    L.gf2c_encode_batch.argtypes = [_vp, _vp, _i64, _vp, _i32, _vp]
    L.gf2c_channel_awgn.argtypes = [_vp, _u64, _u64, _i64, _vp, _vp, _vp, _vp, _i32, _vp]
    L.gf2c_sigma2_from_ebn0.argtypes = [ctypes.c_double, ctypes.c_double]
    L.gf2c_sigma2_from_ebn0.restype = ctypes.c_double
    L.gf2c_decoder_create.argtypes = [_vp, ctypes.POINTER(DecoderOpts), ctypes.POINTER(_vp)]
    L.gf2c_decoder_create_multi.argtypes = [_vp, _i32, ctypes.POINTER(DecoderOpts), ctypes.POINTER(_vp)]
    L.gf2c_decoder_destroy.argtypes = [_vp]
    L.gf2c_decode_batch.argtypes = [_vp, _vp, _i64, _i32, _vp, _vp, _vp, _vp, _vp, _i32, _vp]
    L.gf2c_decode_batch_fallback.argtypes = [_vp, _vp, _vp, _i64, _i32, _i32, _vp, _vp, _vp, _vp, _vp, _i32, _vp]
    L.gf2c_decode_mixed.argtypes = [_vp, _vp, _vp, _vp, _vp, _i64, _vp, _vp, _vp, _vp, _vp, _i32, _i32, _vp]
    L.gf2c_decoder_last_launches.argtypes = [_vp, ctypes.POINTER(_i32)]
    L.gf2c_decode_batch_noalloc.argtypes = [_vp, _vp, _i64, _i32, _vp, _vp, _vp, _vp, _vp]
    L.gf2c_judge_spa64.argtypes = [_vp, _i32, _vp, _i64, _i32, _vp, _vp, _vp, _vp, _vp, _vp]
    L.gf2c_nms_trainer_create.argtypes = [_vp, _i32, _i64, ctypes.POINTER(_vp)]
    L.gf2c_nms_trainer_destroy.argtypes = [_vp]
    L.gf2c_nms_trainer_layers.argtypes = [_vp, ctypes.POINTER(_i32)]
    L.gf2c_nms_trainer_set_schedule.argtypes = [_vp, _i32]
    L.gf2c_nms_loss_grad.argtypes = [_vp, _vp, _vp, _i64, _vp, _vp, _vp, _vp, _vp, _vp, _vp]
    L.gf2c_count_errors.argtypes = [_vp, _vp, _i64, _i32, _vp, _vp, _vp]
    L.gf2c_adam_step.argtypes = [_vp, _vp, _vp, _vp, _i64, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                                 ctypes.c_float, _i32, ctypes.c_float, ctypes.c_float, _vp]
    L.gf2c_bch_create_dvbt2.argtypes = [_i32, _i32, ctypes.POINTER(_vp)]
    L.gf2c_bch_destroy.argtypes = [_vp]
    L.gf2c_bch_dims.argtypes = [_vp, _vp, _vp, _vp, _vp]
    L.gf2c_bch_generator.argtypes = [_vp, _vp]
    L.gf2c_bch_encode_batch.argtypes = [_vp, _vp, _i64, _vp, _i32, _vp]
    L.gf2c_bch_decode_batch.argtypes = [_vp, _vp, _i64, _vp, _vp, _vp, _i32, _vp]
    _s = ctypes.c_char_p
    L.gf2c_io_probe.argtypes = [_s, _vp, _vp, _vp]
    L.gf2c_io_write_bitvec.argtypes = [_s, _vp, _i64, _i32]
    L.gf2c_io_read_bitvec.argtypes = [_s, _vp, _i64, _vp]
    L.gf2c_io_write_bitmatrix.argtypes = [_s, _vp, _i64, _i64, _i32]
    L.gf2c_io_read_bitmatrix.argtypes = [_s, _i32, _vp, _i64, _vp, _vp]
    L.gf2c_io_write_sparse.argtypes = [_s, _i32, _i64, _i64, _vp, _vp, _i32]
    L.gf2c_io_read_sparse.argtypes = [_s, _i32, _vp, _vp, _vp, _vp, _vp, _i64]
    L.gf2c_code_create_file.argtypes = [_s, ctypes.POINTER(_vp)]
    L.gf2c_io_write_code.argtypes = [_s, _vp, _i32, _i32]
    L.gf2c_siphash13.argtypes = [_vp, _i64, _u64, _u64, _vp]
    L.gf2c_code_cache_hash.argtypes = [_vp, _vp]
    L.gf2c_code_parity_part.argtypes = [_vp, _vp]
    L.gf2c_dense_encoder_create.argtypes = [_vp, _i64, _i64, ctypes.POINTER(_vp)]
    L.gf2c_dense_encoder_destroy.argtypes = [_vp]
    L.gf2c_dense_encode_batch.argtypes = [_vp, _vp, _i64, _vp, _i32, _vp]
    return L


lib = _load()


def check(rc):
    if rc != OK:
        raise Gf2cError(rc, lib.gf2c_last_error().decode())
    return rc
