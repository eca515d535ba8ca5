"""Python binding of libb200enc.so, the B200 compute-encoder hot path.

The product is the C-ABI library (include/gpu_compute.h, include/b200enc.h);
this module only loads it with ctypes and moves torch device tensors through
it, for tests, benchmarks and Python callers. Every compute call goes to the
CUDA library; there is no CPU or PyTorch fallback, and using the module
without the built library or without a GPU raises.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.normpath(os.path.join(HERE, "..", "lib", "libb200enc.so"))

# Every entry point include/*.h declares (checked by the CPU test suite).
EXPORTS = [
    # include/b200enc.h
    "b200enc_me_full_search", "b200enc_p_frame", "b200enc_wavefront_scratch_bytes", "b200enc_i_frame",
    "b200enc_deblock", "b200enc_deblock_tiles", "b200enc_wavefront_status", "b200enc_i_frame_launch", "b200enc_deblock_launch",
    "b200enc_deblock_noalloc", "b200enc_gemm_bf16", "b200enc_me_full_search_ex",
    "b200enc_proposal_num_params", "b200enc_proposal_create", "b200enc_proposal_destroy",
    "b200enc_proposal_set_params", "b200enc_proposal_get_params", "b200enc_proposal_prepare",
    "b200enc_proposal_forward", "b200enc_proposal_labels", "b200enc_proposal_backward", "b200enc_proposal_adam",
    "b200enc_proposal_train_step", "b200enc_proposal_me", "b200enc_proposal_tensor", "b200enc_proposal_load",
    "b200enc_ctx_set_me", "b200enc_ctx_me_stats",
    "b200enc_hevc_transform_quant_4x4", "b200enc_hevc_dequant_itransform_4x4", "b200enc_hevc_transform_quant_8x8",
    "b200enc_hevc_dequant_itransform_8x8", "b200enc_hevc_build_hpel", "b200enc_hevc_motion_search",
    "b200enc_hevc_choose_luma_mode", "b200enc_hevc_deblock", "b200enc_hevc_build_hpel_10",
    "b200enc_hevc_motion_search_10", "b200enc_hevc_choose_luma_mode_10", "b200enc_hevc_build_hpel_host",
    "b200enc_tune_set", "b200enc_tune_get", "b200enc_tune_name", "b200enc_tune_load", "b200enc_me_wait_errors",
    "b200enc_pin_host", "b200enc_unpin_host", "b200enc_deblock_noalloc_status",
    "b200enc_batch_create", "b200enc_batch_destroy", "b200enc_batch_stream", "b200enc_batch_set_graph",
    "b200enc_batch_encode", "b200enc_batch_sync", "b200enc_batch_outputs", "b200enc_batch_graph_stats",
    "b200enc_h264_t8_forward", "b200enc_h264_t8_recon", "b200enc_deblock_tiles_t8", "b200enc_p_frame_t8",
    "b200enc_cavlc_scratch_bytes", "b200enc_cavlc_slices", "b200enc_ctx_set_entropy", "b200enc_ctx_slice_nals",
    # include/gpu_compute.h
    "bc250_gpu_init", "bc250_gpu_destroy", "gpu_compute_init", "gpu_compute_terminate",
    "gpu_compute_create_image", "gpu_compute_destroy_image", "gpu_compute_get_nv12_layout",
    "gpu_compute_map_surface", "gpu_compute_unmap_surface", "gpu_compute_upload_nv12",
    "gpu_compute_download_nv12", "gpu_compute_copy_from_wc", "gpu_compute_wait_for_image_ready_host",
    "gpu_compute_cpu_read_safe", "bc250_debug_dump_open", "gpu_compute_begin_picture",
    "gpu_compute_dispatch_encode", "gpu_compute_dispatch_encode_ext", "gpu_compute_dispatch_me_only",
    "gpu_compute_get_last_latency_ms", "gpu_compute_end_picture", "gpu_compute_sync",
    "gpu_compute_submitted_slot", "gpu_compute_sync_slot", "gpu_compute_get_quant_staging_data_slot",
    "gpu_compute_get_dc_staging_data_slot", "gpu_compute_get_pred_mode_staging_data_slot",
    "gpu_compute_get_mv_staging_data_slot", "gpu_compute_get_nz_staging_data_slot",
    "gpu_compute_get_staging_data", "gpu_compute_release_staging_data", "gpu_compute_get_quant_staging_data",
    "gpu_compute_get_dc_staging_data", "gpu_compute_get_pred_mode_staging_data",
    "gpu_compute_get_mv_staging_data", "gpu_compute_get_nz_staging_data", "gpu_compute_debug_dump_recon",
    "b200enc_ctx_configure", "b200enc_ctx_stream", "b200enc_ctx_recon", "b200enc_ctx_device_outputs",
    "b200enc_ctx_encode_device", "b200enc_ctx_perf", "b200enc_ctx_perf_read", "b200enc_host_register",
    "b200enc_host_unregister",
]

_vp = ctypes.c_void_p
_i = ctypes.c_int
_lib = None


class GpuImage(ctypes.Structure):
    _fields_ = [("y_plane", _vp), ("y_view", _vp), ("uv_plane", _vp), ("uv_view", _vp), ("width", ctypes.c_uint32),
                ("height", ctypes.c_uint32), ("current_layout", _i), ("format", _i), ("pitch", ctypes.c_uint32)]


class GpuMemory(ctypes.Structure):
    _fields_ = [("memory", _vp), ("size", ctypes.c_size_t), ("mapped_ptr", _vp)]


class GpuContext(ctypes.Structure):
    _fields_ = [("recon_image", GpuImage), ("recon_memory", GpuMemory), ("has_recon_frame", ctypes.c_bool),
                ("any_surface_exported", ctypes.c_bool), ("frame_width", ctypes.c_uint32),
                ("frame_height", ctypes.c_uint32), ("frames_submitted", ctypes.c_uint32), ("current_buf", _i),
                ("impl", _vp)]


def load_library(path=LIB_PATH):
    """Loads the library without touching the GPU (works on CPU hosts)."""
    if not os.path.exists(path):
        raise RuntimeError(f"libb200enc.so is not built ({path}); run __graft_entry__.build()")
    lib = ctypes.CDLL(path)
    lib.b200enc_wavefront_scratch_bytes.restype = ctypes.c_size_t
    lib.b200enc_wavefront_scratch_bytes.argtypes = [_i]
    lib.gpu_compute_get_last_latency_ms.restype = ctypes.c_double
    lib.b200enc_ctx_stream.restype = _vp
    lib.b200enc_i_frame.argtypes = [_vp, _vp, _i, _i, _i, _i, _i, _i, _i, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _i,
                                    _vp, ctypes.c_size_t, _i, _i, _vp]
    lib.b200enc_deblock.argtypes = [_i, _i, _i, _i, _vp, _vp, _vp, _vp, _i, _vp, ctypes.c_size_t, _i, _vp]
    lib.b200enc_p_frame_t8.argtypes = [_vp, _vp, _i, _vp, _vp, _i, _i, _i, _i, _i, _i, _vp, _vp, _vp, _vp, _vp, _vp,
                                       _vp, _i, _i, _vp, _vp]
    lib.b200enc_h264_t8_forward.argtypes = [_vp, _vp, _vp, _i, _i, _i, _vp]
    lib.b200enc_h264_t8_recon.argtypes = [_vp, _vp, _vp, _i, _i, _i, _vp]
    lib.b200enc_deblock_tiles_t8.argtypes = [_i, _i, _i, _i, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _i, _vp, _vp]
    lib.b200enc_cavlc_scratch_bytes.argtypes = [_i, _i]
    lib.b200enc_cavlc_scratch_bytes.restype = ctypes.c_size_t
    lib.b200enc_cavlc_slices.argtypes = [_vp, _vp]
    lib.b200enc_ctx_set_entropy.argtypes = [_vp, _i, _i]
    lib.b200enc_ctx_slice_nals.argtypes = [_vp, _i, _vp, _vp, _i, _i, _vp, ctypes.c_size_t, _vp]
    lib.b200enc_deblock_tiles.argtypes = [_i, _i, _i, _i, _vp, _vp, _vp, _vp, _vp, _vp, _i, _vp, _vp]
    lib.b200enc_me_full_search.argtypes = [_vp, _i, _vp, _i, _i, _i, _i, _i, _i, _i, _i, _vp, _vp]
    lib.b200enc_me_full_search_ex.argtypes = [_vp, _i, _vp, _i, _i, _i, _i, _i, _i, _i, _i, _vp, _vp, _vp, _i, _i,
                                              _vp]
    lib.b200enc_p_frame.argtypes = [_vp, _vp, _i, _vp, _vp, _i, _i, _i, _i, _i, _i, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                                    _i, _vp]
    lib.b200enc_wavefront_status.argtypes = [_vp, _vp]
    lib.gpu_compute_dispatch_encode_ext.argtypes = [ctypes.POINTER(GpuContext), GpuImage, _i, _i, _i, _i, _i, _i, _vp]
    lib.gpu_compute_begin_picture.argtypes = [ctypes.POINTER(GpuContext), GpuImage]
    lib.b200enc_ctx_encode_device.argtypes = [ctypes.POINTER(GpuContext), _vp, _vp, _i, _i, _i, _i, _i, _i, _i]
    lib.b200enc_gemm_bf16.argtypes = [_i, _i, _i, _vp, ctypes.c_longlong, ctypes.c_longlong, _vp, ctypes.c_longlong,
                                      ctypes.c_longlong, _vp, ctypes.c_longlong, _vp, _i, _vp, _vp]
    lib.b200enc_proposal_create.restype = _vp
    lib.b200enc_proposal_create.argtypes = [_i]
    lib.b200enc_proposal_destroy.argtypes = [_vp]
    lib.b200enc_proposal_destroy.restype = None
    lib.b200enc_proposal_set_params.argtypes = [_vp, _vp, _i]
    lib.b200enc_proposal_get_params.argtypes = [_vp, _vp, _i]
    lib.b200enc_proposal_prepare.argtypes = [_vp, _vp, _i, _vp, _i, _i, _i, _i, _i, _vp, _i, _i, _vp]
    lib.b200enc_proposal_forward.argtypes = [_vp, _i, _vp]
    lib.b200enc_proposal_labels.argtypes = [_vp, _i, _vp, _vp, _vp]
    lib.b200enc_proposal_backward.argtypes = [_vp, _i, _vp]
    lib.b200enc_proposal_adam.argtypes = [_vp, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float, _i,
                                          _vp]
    lib.b200enc_proposal_train_step.argtypes = [_vp, _i, ctypes.c_float, _i, _vp]
    lib.b200enc_proposal_me.argtypes = [_vp, _vp, _i, _vp, _i, _i, _i, _i, _i, _vp, _i, _i, _i, _i, ctypes.c_float,
                                        _vp, _vp]
    lib.b200enc_proposal_tensor.argtypes = [_vp, _i, ctypes.POINTER(_vp), ctypes.POINTER(ctypes.c_size_t)]
    lib.b200enc_proposal_load.argtypes = [_vp, ctypes.c_char_p]
    lib.b200enc_hevc_transform_quant_4x4.argtypes = [_vp, _vp, _i, _i, _i, _i, _i, _vp]
    lib.b200enc_hevc_dequant_itransform_4x4.argtypes = [_vp, _vp, _i, _i, _i, _i, _vp]
    lib.b200enc_hevc_transform_quant_8x8.argtypes = [_vp, _vp, _i, _i, _i, _i, _vp]
    lib.b200enc_hevc_dequant_itransform_8x8.argtypes = [_vp, _vp, _i, _i, _i, _vp]
    lib.b200enc_hevc_build_hpel.argtypes = [_vp, _i, _i, _i, _i, _vp, _vp, _vp, _vp, _i, _vp]
    lib.b200enc_hevc_motion_search.argtypes = [_vp, _i, _i, _i, _vp, _vp, _vp, _vp, _i, _i, _i, _vp, _i, _vp, _vp]
    lib.b200enc_hevc_choose_luma_mode.argtypes = [_vp, _i, _vp, _i, _i, _i, _vp, _i, _vp, _vp, _vp]
    lib.b200enc_hevc_build_hpel_10.argtypes = [_vp, _i, _i, _i, _i, _vp, _vp, _vp, _vp, _i, _vp]
    lib.b200enc_hevc_motion_search_10.argtypes = [_vp, _i, _i, _i, _vp, _vp, _vp, _vp, _i, _i, _i, _vp, _i, _vp,
                                                  _vp]
    lib.b200enc_hevc_choose_luma_mode_10.argtypes = [_vp, _i, _vp, _i, _i, _i, _vp, _i, _vp, _vp, _vp]
    lib.b200enc_hevc_deblock.argtypes = [ctypes.POINTER(HevcDeblockParams), _vp]
    lib.b200enc_ctx_set_me.argtypes = [ctypes.POINTER(GpuContext), _i, ctypes.c_char_p, ctypes.c_float]
    lib.b200enc_host_register.argtypes = [ctypes.POINTER(GpuContext), _vp, ctypes.c_size_t]
    lib.b200enc_host_unregister.argtypes = [ctypes.POINTER(GpuContext), _vp]
    lib.b200enc_batch_create.restype = _vp
    lib.b200enc_batch_create.argtypes = [_i, _vp, _vp, _i, _i, ctypes.c_float, _i]
    lib.b200enc_batch_destroy.argtypes = [_vp]
    lib.b200enc_batch_destroy.restype = None
    lib.b200enc_batch_stream.restype = _vp
    lib.b200enc_batch_stream.argtypes = [_vp]
    lib.b200enc_batch_set_graph.argtypes = [_vp, _i]
    lib.b200enc_batch_encode.argtypes = [_vp, _vp]
    lib.b200enc_batch_sync.argtypes = [_vp]
    lib.b200enc_batch_outputs.argtypes = [_vp, _i] + [ctypes.POINTER(_vp)] * 7 + [ctypes.POINTER(_i)]
    lib.b200enc_batch_graph_stats.argtypes = [_vp, ctypes.POINTER(ctypes.c_long), ctypes.POINTER(ctypes.c_long)]
    lib.b200enc_tune_set.argtypes = [_i, _i]
    lib.b200enc_tune_get.argtypes = [_i]
    lib.b200enc_tune_name.argtypes = [_i]
    lib.b200enc_tune_name.restype = ctypes.c_char_p
    lib.b200enc_tune_load.argtypes = [ctypes.c_char_p]
    lib.b200enc_me_wait_errors.argtypes = [_i]
    lib.b200enc_pin_host.argtypes = [_vp, ctypes.c_size_t]
    lib.b200enc_unpin_host.argtypes = [_vp]
    lib.b200enc_deblock_noalloc_status.argtypes = [_vp, _vp]
    return lib


def lib():
    """The loaded library; raises when it is missing or no GPU is present."""
    global _lib
    if _lib is None:
        import torch
        if not torch.cuda.is_available():
            raise RuntimeError("b200enc needs a CUDA device (sm_100a); none is available")
        _lib = load_library()
    return _lib


def _check(rc, what):
    if rc != 0:
        raise RuntimeError(f"{what} failed (rc={rc})")


def _stream(stream):
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return _vp(s.cuda_stream)


def coded(W, H):
    return (W + 15) // 16 * 16, (H + 15) // 16 * 16


class NV12:
    """An NV12 frame in device memory at the coded size, 128-byte pitch."""

    def __init__(self, W, H, device="cuda", pitch=None):
        import torch
        self.W, self.H = W, H
        self.CW, self.CH = coded(W, H)
        self.pitch = pitch or (self.CW + 127) // 128 * 128
        self.buf = torch.zeros((self.CH + self.CH // 2, self.pitch), dtype=torch.uint8, device=device)
        self.y = self.buf[: self.CH]
        self.uv = self.buf[self.CH:]

    @classmethod
    def from_host(cls, y, uv, device="cuda", pitch=None):
        """y: [H, W] uint8, uv: [H/2, W] uint8 (numpy); pads by edge replication."""
        import numpy as np
        import torch
        H, W = y.shape
        f = cls(W, H, device, pitch)
        yp = np.pad(y, ((0, f.CH - H), (0, f.pitch - W)), mode="edge")
        uvp = np.pad(uv, ((0, f.CH // 2 - H // 2), (0, f.pitch - W)), mode="edge")
        f.y.copy_(torch.from_numpy(yp))
        f.uv.copy_(torch.from_numpy(uvp))
        return f

    def yp(self):
        return _vp(self.y.data_ptr())

    def uvp(self):
        return _vp(self.uv.data_ptr())


class Outputs:
    """Per-frame outputs in device memory (reference staging layouts)."""

    def __init__(self, W, H, device="cuda"):
        import torch
        mbs = ((W + 15) // 16) * ((H + 15) // 16)
        self.levels = torch.zeros((mbs, 24, 16), dtype=torch.int16, device=device)
        self.dc = torch.zeros((mbs, 24), dtype=torch.int32, device=device)
        self.nz = torch.zeros((mbs, 24), dtype=torch.int32, device=device)
        self.pred_mode = torch.zeros((mbs,), dtype=torch.int32, device=device)
        self.mv = torch.zeros((mbs, 4), dtype=torch.int32, device=device)

    def host(self):
        import numpy as np
        return {"levels": self.levels.cpu().numpy(), "dc": self.dc.cpu().numpy(),
                "nz": self.nz.cpu().numpy().view(np.uint32), "pred_mode": self.pred_mode.cpu().numpy().view(np.uint32),
                "mv": self.mv.cpu().numpy()}


def _p(t):
    return _vp(t.data_ptr())


def me_full_search(cur, ref, W, H, RW, RH, rng, lam, zero_thresh, mv, stream=None):
    _check(lib().b200enc_me_full_search(cur.yp(), cur.pitch, ref.yp(), ref.pitch, W, H, RW, RH, rng, lam,
                                        zero_thresh, _p(mv), _stream(stream)), "b200enc_me_full_search")


ME_LOG_INTEGER = 1


def me_full_search_ex(cur, ref, W, H, RW, RH, rng, lam, zero_thresh, mv, mb_list=None, mb_count=None,
                      capacity=0, flags=0, stream=None):
    _check(lib().b200enc_me_full_search_ex(cur.yp(), cur.pitch, ref.yp(), ref.pitch, W, H, RW, RH, rng, lam,
                                           zero_thresh, _p(mv), _p(mb_list) if mb_list is not None else None,
                                           _p(mb_count) if mb_count is not None else None, capacity, flags,
                                           _stream(stream)), "b200enc_me_full_search_ex")


def me_log_decode(pad):
    """(valid, early_out, dx, dy) arrays from ME_LOG_INTEGER words."""
    import numpy as np
    pad = np.asarray(pad).astype(np.uint32)
    return ((pad >> 31) & 1).astype(bool), ((pad >> 30) & 1).astype(bool), \
        (pad & 0xFF).astype(np.int32) - 128, ((pad >> 8) & 0xFF).astype(np.int32) - 128


def p_frame(cur, ref, W, H, RW, RH, qp, mv, out, rec, stream=None):
    _check(lib().b200enc_p_frame(cur.yp(), cur.uvp(), cur.pitch, ref.yp(), ref.uvp(), ref.pitch, W, H, RW, RH, qp,
                                 _p(mv), _p(out.levels), _p(out.dc), _p(out.nz), _p(out.pred_mode), rec.yp(),
                                 rec.uvp(), rec.pitch, _stream(stream)), "b200enc_p_frame")


def p_frame_t8(cur, ref, W, H, RW, RH, qp, mv, out, rec, t8, t8_flags=None, stream=None):
    """The P chain with the 8x8 luma transform: t8 1 for every macroblock, 2
    chosen per macroblock (t8_flags: a device uint8 tensor [mbs] or None)."""
    _check(lib().b200enc_p_frame_t8(cur.yp(), cur.uvp(), cur.pitch, ref.yp(), ref.uvp(), ref.pitch, W, H, RW, RH, qp,
                                    _p(mv), _p(out.levels), _p(out.dc), _p(out.nz), _p(out.pred_mode), rec.yp(),
                                    rec.uvp(), rec.pitch, int(t8), _p(t8_flags) if t8_flags is not None else None,
                                    _stream(stream)), "b200enc_p_frame_t8")


def scratch(mbh, device="cuda"):
    import torch
    n = lib().b200enc_wavefront_scratch_bytes(mbh)
    return torch.zeros((n + 3) // 4, dtype=torch.int32, device=device)


INTRA_CORNER_CHECK = 1


def i_frame(cur, W, H, RW, RH, qp, num_slices, out, rec, scr, ctas=0, stream=None, flags=INTRA_CORNER_CHECK):
    _check(lib().b200enc_i_frame(cur.yp(), cur.uvp(), cur.pitch, W, H, RW, RH, qp, num_slices, _p(out.levels),
                                 _p(out.dc), _p(out.nz), _p(out.pred_mode), _p(out.mv), rec.yp(), rec.uvp(),
                                 rec.pitch, _p(scr), scr.numel() * 4, ctas, flags, _stream(stream)),
           "b200enc_i_frame")


def deblock(mbw, mbh, qp, is_intra, nz, mv, rec, scr, ctas=0, stream=None):
    _check(lib().b200enc_deblock(mbw, mbh, qp, int(is_intra), _p(nz), _p(mv), rec.yp(), rec.uvp(), rec.pitch,
                                 _p(scr), scr.numel() * 4, ctas, _stream(stream)), "b200enc_deblock")


def deblock_tiles(mbw, mbh, qp, is_intra, nz, mv, src, dst, status, stream=None):
    """Tile deblocking from the unfiltered planes `src` into `dst` (same
    pitch, no overlap); `status` is a device int32 tensor of >= 4 words."""
    _check(lib().b200enc_deblock_tiles(mbw, mbh, qp, int(is_intra), _p(nz), _p(mv), src.yp(), src.uvp(), dst.yp(),
                                       dst.uvp(), src.pitch, _p(status), _stream(stream)), "b200enc_deblock_tiles")


GEMM_ACCUMULATE, GEMM_RELU, GEMM_OUT_BF16 = 1, 2, 4


def GEMM_SPLITK(n):
    return n << 16


def gemm_bf16(A, B, C, M, N, K, a_strides, b_strides, bias=None, flags=0, err=None, stream=None):
    """C[:M,:N] = epilogue(A(m,k) . B(n,k)) on the tensor cores; A, B bf16
    tensors addressed through (row, k) element strides, C float32."""
    _check(lib().b200enc_gemm_bf16(M, N, K, _p(A), a_strides[0], a_strides[1], _p(B), b_strides[0], b_strides[1],
                                   _p(C), C.stride(0), _p(bias) if bias is not None else None, flags,
                                   _p(err) if err is not None else None, _stream(stream)), "b200enc_gemm_bf16")


def hevc_transform_quant_4x4(residual, coeff, qp, use_dst, round_q12, bit_depth=8, stream=None):
    """residual, coeff: int16 device tensors [n][16]."""
    _check(lib().b200enc_hevc_transform_quant_4x4(_p(residual), _p(coeff), residual.shape[0], qp, int(use_dst),
                                                  round_q12, bit_depth, _stream(stream)), "hevc_transform_quant_4x4")


def hevc_dequant_itransform_4x4(coeff, residual, qp, use_dst, bit_depth=8, stream=None):
    _check(lib().b200enc_hevc_dequant_itransform_4x4(_p(coeff), _p(residual), coeff.shape[0], qp, int(use_dst),
                                                     bit_depth, _stream(stream)), "hevc_dequant_itransform_4x4")


def hevc_transform_quant_8x8(residual, coeff, qp, round_q12, bit_depth=8, stream=None):
    """residual, coeff: int16 device tensors [n][64]."""
    _check(lib().b200enc_hevc_transform_quant_8x8(_p(residual), _p(coeff), residual.shape[0], qp, bit_depth,
                                                  round_q12, _stream(stream)), "hevc_transform_quant_8x8")


def hevc_dequant_itransform_8x8(coeff, residual, qp, bit_depth=8, stream=None):
    _check(lib().b200enc_hevc_dequant_itransform_8x8(_p(coeff), _p(residual), coeff.shape[0], qp, bit_depth,
                                                     _stream(stream)), "hevc_dequant_itransform_8x8")


def _ten_bit(t):
    import torch
    if t.dtype == torch.uint8:
        return False
    if t.dtype in (torch.int16, torch.uint16):
        return True
    raise TypeError(f"samples must be uint8 (8-bit) or 16-bit words (10-bit), not {t.dtype}")


def hevc_build_hpel(recon, w, h, margin, planes, stream=None):
    """recon: device tensor [>=h][pitch], uint8 (8-bit) or int16/uint16
    words holding 10-bit samples; planes: device tensor of the same type
    [4][h + 2*margin][pitch >= w + 2*margin] (I, H, V, HV). Pitches are in
    samples."""
    fn = "b200enc_hevc_build_hpel_10" if _ten_bit(recon) else "b200enc_hevc_build_hpel"
    _check(getattr(lib(), fn)(_p(recon), recon.stride(0), w, h, margin, _p(planes[0]), _p(planes[1]),
                              _p(planes[2]), _p(planes[3]), planes.stride(1), _stream(stream)), fn)


# b200enc_hevc_me_job_t / b200enc_hevc_me_result_t as numpy structured dtypes
import numpy as _np  # noqa: E402
HEVC_ME_JOB = _np.dtype([("cu_x", "<i4"), ("cu_y", "<i4"), ("mvp", "<i2", (2, 2)), ("starts", "<i2", (16, 2)),
                         ("n_starts", "<i4"), ("lambda_q8", "<i4")])
HEVC_ME_RESULT = _np.dtype([("mv", "<i2", (2,)), ("mvp_idx", "<i4"), ("cost_q8", "<i8"), ("sad", "<u4"),
                            ("pad", "<u4")])


def hevc_motion_search(src, w, h, planes, margin, qpel, jobs, results, stream=None):
    """src: uint8 device tensor [>=h][pitch]; planes as hevc_build_hpel;
    jobs / results: uint8 device tensors holding HEVC_ME_JOB / HEVC_ME_RESULT
    records."""
    n = jobs.numel() // HEVC_ME_JOB.itemsize
    fn = "b200enc_hevc_motion_search_10" if _ten_bit(src) else "b200enc_hevc_motion_search"
    _check(getattr(lib(), fn)(_p(src), src.stride(0), w, h, _p(planes[0]), _p(planes[1]), _p(planes[2]),
                              _p(planes[3]), planes.stride(1), margin, int(qpel), _p(jobs), n, _p(results),
                              _stream(stream)), fn)


def hevc_choose_luma_mode(src, recon, width, height, jobs, modes, preds, stream=None):
    """src, recon: uint8 device tensors, or 16-bit words holding 10-bit
    samples (pitch = stride(0), in samples); jobs: int32 device tensor
    [n][3] (x0, y0, y_min); modes: int32 [n]; preds: [n][16] of the sample
    type."""
    fn = "b200enc_hevc_choose_luma_mode_10" if _ten_bit(src) else "b200enc_hevc_choose_luma_mode"
    _check(getattr(lib(), fn)(_p(src), src.stride(0), _p(recon), recon.stride(0), width, height, _p(jobs),
                              jobs.shape[0], _p(modes), _p(preds), _stream(stream)), fn)


# b200enc_hevc_mvf_t / b200enc_hevc_slice_filter_t records and the
# b200enc_hevc_deblock_t parameter block
HEVC_MVF = _np.dtype([("mv", "<i2", (2, 2)), ("ref_poc", "<i4", (2,)), ("pred_flag", "u1"), ("pad", "u1", (3,))])
HEVC_SLICE_FILTER = _np.dtype([("beta_offset", "<i2"), ("tc_offset", "<i2"), ("disabled", "u1"),
                               ("across_slices", "u1"), ("pad", "u1", (2,))])


class CavlcParams(ctypes.Structure):
    """b200enc_cavlc_t (include/b200enc.h)."""
    _fields_ = [("mbw", _i), ("mbh", _i), ("qp", _i), ("is_intra", _i), ("num_slices", _i), ("quality_level", _i),
                ("levels", _vp), ("dc", _vp), ("nz", _vp), ("pred_mode", _vp), ("mv", _vp),
                ("header", _vp), ("header_bits", _vp), ("out", _vp), ("slice_cap", ctypes.c_size_t),
                ("out_bytes", _vp), ("out_copy", _vp), ("scratch", _vp), ("scratch_bytes", ctypes.c_size_t),
                ("transform8x8", _i), ("t8_flags", _vp)]


def cavlc_slices(mbw, mbh, qp, is_intra, num_slices, levels, dc, nz, pred_mode, mv, headers=None,
                 quality_level=4, slice_cap=None, stream=None, transform8x8=0, t8_flags=None):
    """CAVLC slice data of one picture on the GPU from device pointers (ints)
    to its staged outputs; headers: None or a list of (bits, nbits) per
    slice, bits an int holding nbits (<= 128) header bits. Returns a list of
    each slice's RBSP bytes."""
    import numpy as np
    import torch
    L = lib()
    mbs = mbw * mbh
    cap = slice_cap or ((mbs * 2560 // num_slices + 4096 + 3) // 4 * 4)
    out = torch.zeros(num_slices * cap, dtype=torch.uint8, device="cuda")
    nbytes = torch.zeros(num_slices, dtype=torch.int32, device="cuda")
    sb = L.b200enc_cavlc_scratch_bytes(mbw, mbh)
    scratch = torch.empty(sb + 256, dtype=torch.uint8, device="cuda")
    sp = (scratch.data_ptr() + 255) // 256 * 256
    hdr = hb = None
    if headers is not None:
        hdr = np.zeros((num_slices, 16), np.uint8)
        hb = np.zeros(num_slices, np.int32)
        for k, (bits, n) in enumerate(headers):
            hb[k] = n
            hdr[k] = np.frombuffer(((bits << (128 - n)) if n else 0).to_bytes(16, "big"), np.uint8)
    prm = CavlcParams(mbw, mbh, qp, int(is_intra), num_slices, quality_level, _vp(levels), _vp(dc), _vp(nz),
                      _vp(pred_mode) if pred_mode else None, _vp(mv),
                      _vp(hdr.ctypes.data) if hdr is not None else None,
                      _vp(hb.ctypes.data) if hb is not None else None, _vp(out.data_ptr()), cap,
                      _vp(nbytes.data_ptr()), None, _vp(sp), sb, int(transform8x8),
                      _vp(t8_flags) if t8_flags else None)
    _check(L.b200enc_cavlc_slices(ctypes.byref(prm), _stream(stream)), "b200enc_cavlc_slices")
    torch.cuda.synchronize()
    n = nbytes.cpu().numpy().view(np.uint32)
    o = out.cpu().numpy()
    res = []
    for k in range(num_slices):
        if n[k] == 0xffffffff:
            raise RuntimeError(f"slice {k} outgrew its region")
        res.append(o[k * cap:k * cap + int(n[k])].tobytes())
    return res


class HevcDeblockParams(ctypes.Structure):
    _fields_ = [("plane", ctypes.c_void_p * 3), ("stride", ctypes.c_int * 3), ("width", ctypes.c_int),
                ("height", ctypes.c_int), ("bit_depth_luma", ctypes.c_int), ("bit_depth_chroma", ctypes.c_int),
                ("log2_ctb", ctypes.c_int), ("log2_min_cb", ctypes.c_int), ("edges", ctypes.c_void_p),
                ("edges_stride", ctypes.c_int), ("mvf", ctypes.c_void_p), ("cbf", ctypes.c_void_p),
                ("min_pu_width", ctypes.c_int), ("qp_y", ctypes.c_void_p), ("no_filter", ctypes.c_void_p),
                ("slice_of_ctb", ctypes.c_void_p), ("slice_filter", ctypes.c_void_p),
                ("n_slice_filter", ctypes.c_int), ("tile_of_ctb", ctypes.c_void_p),
                ("loop_filter_across_tiles", ctypes.c_int), ("cb_qp_offset", ctypes.c_int),
                ("cr_qp_offset", ctypes.c_int)]


def hevc_deblock_params(ptr, planes, strides, width, height, bit_depth_luma, bit_depth_chroma, log2_ctb,
                        log2_min_cb, edges, edges_stride, qp_y, mvf=None, cbf=None, min_pu_width=0,
                        no_filter=None, slice_of_ctb=None, slice_filter=None, n_slice_filter=0, tile_of_ctb=None,
                        loop_filter_across_tiles=True, cb_qp_offset=0, cr_qp_offset=0):
    """The parameter block of b200enc_hevc_deblock; `ptr(x)` turns each
    buffer (device tensor for the GPU, numpy array for the oracle) into an
    address, None into NULL."""
    a = lambda x: None if x is None else ptr(x)
    q = HevcDeblockParams()
    for c in range(3):
        q.plane[c] = a(planes[c])
        q.stride[c] = int(strides[c])
    q.width, q.height = width, height
    q.bit_depth_luma, q.bit_depth_chroma = bit_depth_luma, bit_depth_chroma
    q.log2_ctb, q.log2_min_cb = log2_ctb, log2_min_cb
    q.edges, q.edges_stride = a(edges), edges_stride
    q.mvf, q.cbf, q.min_pu_width = a(mvf), a(cbf), min_pu_width
    q.qp_y, q.no_filter = a(qp_y), a(no_filter)
    q.slice_of_ctb, q.slice_filter, q.n_slice_filter = a(slice_of_ctb), a(slice_filter), n_slice_filter
    q.tile_of_ctb, q.loop_filter_across_tiles = a(tile_of_ctb), int(loop_filter_across_tiles)
    q.cb_qp_offset, q.cr_qp_offset = cb_qp_offset, cr_qp_offset
    return q


def hevc_deblock(params, stream=None):
    """HEVC deblocking of one picture in place (device buffers in `params`)."""
    _check(lib().b200enc_hevc_deblock(ctypes.byref(params), _stream(stream)), "hevc_deblock")


def wavefront_status(scr, stream=None):
    return lib().b200enc_wavefront_status(_p(scr), _stream(stream))


class Context:
    """The reference's gpu_compute_* boundary (include/gpu_compute.h)."""

    def __init__(self):
        self.ctx = GpuContext()
        self.L = lib()
        _check(self.L.bc250_gpu_init(ctypes.byref(self.ctx)), "bc250_gpu_init")

    def close(self):
        if self.ctx.impl:
            self.L.bc250_gpu_destroy(ctypes.byref(self.ctx))

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def configure(self, search_range=16, lam=-1, zero_thresh=512, coded_clamp=True, deblock=-1):
        _check(self.L.b200enc_ctx_configure(ctypes.byref(self.ctx), search_range, lam, zero_thresh,
                                            int(coded_clamp), deblock), "b200enc_ctx_configure")

    def create_image(self, W, H):
        img, mem = GpuImage(), GpuMemory()
        _check(self.L.gpu_compute_create_image(ctypes.byref(self.ctx), W, H, 0, ctypes.byref(img),
                                               ctypes.byref(mem)), "gpu_compute_create_image")
        return img, mem

    def destroy_image(self, img, mem):
        self.L.gpu_compute_destroy_image(ctypes.byref(self.ctx), img, mem)

    def upload(self, img, mem, y, uv):
        H, W = y.shape
        _check(self.L.gpu_compute_upload_nv12(ctypes.byref(self.ctx), ctypes.byref(img), mem, _vp(y.ctypes.data),
                                              y.strides[0], _vp(uv.ctypes.data), uv.strides[0], W, H),
               "gpu_compute_upload_nv12")

    def encode(self, img, W, H, qp, is_intra, num_slices=1, me_mode=0, cpu_mvs=None):
        """begin_picture + dispatch_encode_ext + end_picture; returns the slot."""
        c = ctypes.byref(self.ctx)
        _check(self.L.gpu_compute_begin_picture(c, img), "gpu_compute_begin_picture")
        mv = _vp(cpu_mvs.ctypes.data) if cpu_mvs is not None else None
        _check(self.L.gpu_compute_dispatch_encode_ext(c, img, W, H, qp, int(is_intra), num_slices, me_mode, mv),
               "gpu_compute_dispatch_encode_ext")
        _check(self.L.gpu_compute_end_picture(c), "gpu_compute_end_picture")
        return self.L.gpu_compute_submitted_slot(c)

    def sync(self, slot):
        return self.L.gpu_compute_sync_slot(ctypes.byref(self.ctx), slot)

    def set_entropy(self, mode, quality_level=4):
        """GPU entropy coding (b200enc_ctx_set_entropy): 0 off, 1 beside the
        staging, 2 instead of the level staging."""
        _check(self.L.b200enc_ctx_set_entropy(ctypes.byref(self.ctx), mode, quality_level),
               "b200enc_ctx_set_entropy")

    def slice_nals(self, slot, headers, header_bits, nal_ref_idc, nal_unit_type, out):
        """Annex B slice NAL units of a slot into the uint8 numpy array `out`
        (headers: uint8 [slices][16], header_bits: int32 [slices]); returns
        the byte count."""
        n = ctypes.c_size_t()
        _check(self.L.b200enc_ctx_slice_nals(ctypes.byref(self.ctx), slot, _vp(headers.ctypes.data),
                                             _vp(header_bits.ctypes.data), nal_ref_idc, nal_unit_type,
                                             _vp(out.ctypes.data), out.nbytes, ctypes.byref(n)),
               "b200enc_ctx_slice_nals")
        return n.value

    def staging(self, slot):
        """numpy views of the slot's staging buffers (valid until resubmitted)."""
        import numpy as np
        c = ctypes.byref(self.ctx)
        res = {}
        for name, fn, dt, shape in (("levels", "gpu_compute_get_quant_staging_data_slot", np.int16, (-1, 24, 16)),
                                    ("dc", "gpu_compute_get_dc_staging_data_slot", np.int32, (-1, 24)),
                                    ("pred_mode", "gpu_compute_get_pred_mode_staging_data_slot", np.uint32, (-1,)),
                                    ("mv", "gpu_compute_get_mv_staging_data_slot", np.int32, (-1, 4)),
                                    ("nz", "gpu_compute_get_nz_staging_data_slot", np.uint32, (-1, 24))):
            data, size = _vp(), ctypes.c_size_t()
            _check(getattr(self.L, fn)(c, slot, ctypes.byref(data), ctypes.byref(size)), fn)
            buf = (ctypes.c_uint8 * size.value).from_address(data.value)
            res[name] = np.frombuffer(buf, dtype=dt).reshape(shape)
        return res

    def recon_host(self):
        """(y, uv) of the latest reconstruction at the coded size, as numpy."""
        import torch
        y, uv, pitch = _vp(), _vp(), _i()
        _check(self.L.b200enc_ctx_recon(ctypes.byref(self.ctx), ctypes.byref(y), ctypes.byref(uv),
                                        ctypes.byref(pitch)), "b200enc_ctx_recon")
        CW, CH = coded(self.ctx.frame_width, self.ctx.frame_height)
        torch.cuda.synchronize()
        hy = device_view(y.value, CH * pitch.value).cpu().numpy().reshape(CH, pitch.value)
        huv = device_view(uv.value, CH // 2 * pitch.value).cpu().numpy().reshape(CH // 2, pitch.value)
        return hy[:, :CW], huv[:, :CW]

    def perf(self, enable=True):
        _check(self.L.b200enc_ctx_perf(ctypes.byref(self.ctx), int(enable)), "b200enc_ctx_perf")

    def perf_read(self, intra=False):
        """Summed stage milliseconds: dict(me, chain, deblock, staging, frames)."""
        vals = [ctypes.c_double() for _ in range(4)]
        frames = ctypes.c_long()
        _check(self.L.b200enc_ctx_perf_read(ctypes.byref(self.ctx), int(intra), *[ctypes.byref(v) for v in vals],
                                            ctypes.byref(frames)), "b200enc_ctx_perf_read")
        return dict(me=vals[0].value, chain=vals[1].value, deblock=vals[2].value, staging=vals[3].value,
                    frames=frames.value)

    def encode_device(self, frame, W, H, qp, is_intra, num_slices=1, stage=False):
        _check(self.L.b200enc_ctx_encode_device(ctypes.byref(self.ctx), frame.yp(), frame.uvp(), frame.pitch, W, H,
                                                qp, int(is_intra), num_slices, int(stage)),
               "b200enc_ctx_encode_device")

    def stream(self):
        return self.L.b200enc_ctx_stream(ctypes.byref(self.ctx))

    ME_PLAIN, ME_LEARNED, ME_CANDIDATES, ME_LEARNED_FP8 = 0, 1, 2, 3

    def set_me(self, mode, weights=None, conf=0.9):
        """Motion estimation form of P frames (plain / learned / candidates)."""
        rc = self.L.b200enc_ctx_set_me(ctypes.byref(self.ctx), mode, weights.encode() if weights else None, conf)
        if rc != 0:
            raise RuntimeError(f"b200enc_ctx_set_me failed (rc={rc})")

    def mv_field(self):
        """The latest frame's MV field from device memory, [mbs, 4] int32
        (mvx, mvy in quarter pel, sad, pad), without staging."""
        import numpy as np
        import torch
        mv = _vp()
        _check(self.L.b200enc_ctx_device_outputs(ctypes.byref(self.ctx), None, None, None, None, ctypes.byref(mv)),
               "b200enc_ctx_device_outputs")
        mbs = ((self.ctx.frame_width + 15) // 16) * ((self.ctx.frame_height + 15) // 16)
        torch.cuda.synchronize()
        return device_view(mv.value, mbs * 16).cpu().numpy().view(np.int32).reshape(mbs, 4)

    def me_stats(self):
        """(learned, fallback, early-out) MB counts of the last P frame."""
        v = [ctypes.c_int() for _ in range(3)]
        _check(self.L.b200enc_ctx_me_stats(ctypes.byref(self.ctx), *[ctypes.byref(x) for x in v]),
               "b200enc_ctx_me_stats")
        return tuple(x.value for x in v)


class BatchFrame(ctypes.Structure):
    _fields_ = [("y", _vp), ("uv", _vp), ("pitch", _i), ("qp", _i), ("is_intra", _i), ("num_slices", _i)]


class Batch:
    """Many streams of their own frame sizes through one launch per stage
    (b200enc_batch_*): sizes = [(W, H), ...]; me_mode 0 full search, 1
    learned (BF16 network), 3 learned (FP8 network)."""

    def __init__(self, sizes, search_range=32, me_mode=0, conf=0.9, deblock=1, graph=False):
        self.L = lib()
        self.sizes = list(sizes)
        n = len(self.sizes)
        ws = (ctypes.c_int * n)(*[w for w, _ in self.sizes])
        hs = (ctypes.c_int * n)(*[h for _, h in self.sizes])
        self.h = self.L.b200enc_batch_create(n, ws, hs, search_range, me_mode, ctypes.c_float(conf), deblock)
        if not self.h:
            raise RuntimeError("b200enc_batch_create failed")
        self.frames = (BatchFrame * n)()
        _check(self.L.b200enc_batch_set_graph(self.h, int(graph)), "b200enc_batch_set_graph")

    def close(self):
        if self.h:
            self.L.b200enc_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def stream(self):
        return self.L.b200enc_batch_stream(self.h)

    def encode(self, frames, qps, intra, num_slices=1):
        """frames: NV12 objects, one per stream; qps, intra: per stream."""
        for s, f in enumerate(frames):
            self.frames[s] = BatchFrame(f.y.data_ptr(), f.uv.data_ptr(), f.pitch, int(qps[s]), int(bool(intra[s])),
                                        num_slices)
        _check(self.L.b200enc_batch_encode(self.h, self.frames), "b200enc_batch_encode")

    def sync(self):
        return self.L.b200enc_batch_sync(self.h)

    def graph_stats(self):
        a, b = ctypes.c_long(), ctypes.c_long()
        _check(self.L.b200enc_batch_graph_stats(self.h, ctypes.byref(a), ctypes.byref(b)), "b200enc_batch_graph_stats")
        return a.value, b.value

    def outputs_host(self, s):
        """Host copies of stream s's latest outputs and reconstruction."""
        import numpy as np
        import torch
        p = [_vp() for _ in range(7)]
        pitch = _i()
        _check(self.L.b200enc_batch_outputs(self.h, s, *[ctypes.byref(x) for x in p], ctypes.byref(pitch)),
               "b200enc_batch_outputs")
        W, H = self.sizes[s]
        CW, CH = coded(W, H)
        mbs = (CW // 16) * (CH // 16)
        torch.cuda.synchronize()
        rd = lambda ptr, n: device_view(ptr.value, n).cpu().numpy()
        out = {"levels": rd(p[0], mbs * 768).view(np.int16).reshape(mbs, 24, 16),
               "dc": rd(p[1], mbs * 96).view(np.int32).reshape(mbs, 24),
               "nz": rd(p[2], mbs * 96).view(np.uint32).reshape(mbs, 24),
               "pred_mode": rd(p[3], mbs * 4).view(np.uint32),
               "mv": rd(p[4], mbs * 16).view(np.int32).reshape(mbs, 4)}
        out["rec_y"] = rd(p[5], CH * pitch.value).reshape(CH, pitch.value)[:, :CW]
        out["rec_uv"] = rd(p[6], CH // 2 * pitch.value).reshape(CH // 2, pitch.value)[:, :CW]
        return out


class _DeviceSpan:
    def __init__(self, ptr, nbytes):
        self.__cuda_array_interface__ = {"shape": (nbytes,), "typestr": "|u1", "data": (ptr, False),
                                         "version": 3, "strides": None}


def device_view(ptr, nbytes):
    """A uint8 torch tensor aliasing library-owned device memory (no copy)."""
    import torch
    return torch.as_tensor(_DeviceSpan(ptr, nbytes), device="cuda")
