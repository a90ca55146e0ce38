"""zap_b200 - B200 (sm_100a) texture block encoders behind zap_tex.h's API (zap 1.3.0).

Host functions mirror zap_tex.h one for one and take / return numpy arrays (HxWx4, row-major):
    bc_encode(rgba, fmt, rdo=0)   -> zap_bc_encode   (zap_tex.h:1474)
    bc6h_encode(rgba_f32)         -> zap_bc6h_encode (zap_tex.h:946)
    astc_encode(rgba)             -> zap_astc_encode (zap_tex.h:1291)
    mip_next(rgba, srgb)          -> zap_mip_next    (zap_tex.h:1442)
    mip_next_f(rgba_f32)          -> zap_mip_next_f  (zap_tex.h:1460)
    bc_size / mip_levels / block_bytes
`*_dev` variants take torch CUDA tensors and return CUDA tensors (asynchronous on the current torch stream).
All work runs in the CUDA library (zap_b200/lib/libzap_tex_cuda.so); there is no CPU fallback.
"""
import ctypes as C

import numpy as np

from ._lib import ZapTexError, build, check, load

BC1, BC3, BC4, BC5, BC7, BC6H, ASTC4X4 = range(7)
FORMAT_NAMES = {BC1: "bc1", BC3: "bc3", BC4: "bc4", BC5: "bc5", BC7: "bc7", BC6H: "bc6h", ASTC4X4: "astc4x4"}

__all__ = ["BC1", "BC3", "BC4", "BC5", "BC7", "BC6H", "ASTC4X4", "ZapTexError", "build", "load", "bc_size", "block_bytes",
           "mip_levels", "bc_encode", "bc6h_encode", "astc_encode", "mip_next", "mip_next_f", "bc_encode_dev",
           "bc6h_encode_dev", "astc_encode_dev", "mip_next_dev", "mip_next_f_dev", "mip_chain_dev", "dds_header",
           "astc_header", "tex_file"]


def trace(enable=True):
    """Start (or stop) recording CUDA events around every kernel launch of the library."""
    check(load().zap_tex_cuda_trace_enable(int(enable)), "trace")


def trace_report():
    """{kernel name: (launches, total ms, units processed)} since trace() was enabled; clears the record.
    Units are 4x4 blocks for encoders (for the second BC7 / ASTC kernels: the blocks on their work list) and output
    texels for mips."""
    buf = C.create_string_buffer(1 << 16)
    load().zap_tex_cuda_trace_report(buf, len(buf))
    out = {}
    for line in buf.value.decode().splitlines():
        name, n, ms, units = line.split()
        out[name] = (int(n), float(ms), int(units))
    return out


def block_bytes(fmt):
    return int(load().zap_tex_cuda_block_bytes(fmt))


def bc_size(w, h, fmt):
    return int(load().zap_tex_cuda_bc_size(w, h, fmt))


def mip_levels(w, h):
    return int(load().zap_tex_cuda_mip_levels(w, h))


def _img(a, dtype):
    a = np.asarray(a)
    if a.dtype != dtype or a.ndim != 3 or a.shape[2] != 4:
        raise ValueError(f"expected an HxWx4 {np.dtype(dtype).name} image, got {a.shape} {a.dtype}")
    if not a.flags.c_contiguous and a.strides[1:] != (4 * a.itemsize, a.itemsize):
        a = np.ascontiguousarray(a)
    return a, a.shape[1], a.shape[0], a.strides[0]


# ---------------------------------------------------------------- host memory (synchronous drop-ins)
def _out(out, n):
    if out is None:
        return np.empty(n, np.uint8)
    if out.dtype != np.uint8 or out.size < n or not out.flags.c_contiguous:
        raise ValueError(f"out must be a contiguous uint8 array of at least {n} bytes")
    return out


def bc_encode(rgba, fmt, rdo=0.0, ctx=None, out=None):
    a, w, h, stride = _img(rgba, np.uint8)
    out = _out(out, bc_size(w, h, fmt))
    check(load().zap_tex_cuda_bc_encode(ctx, a.ctypes.data, w, h, stride, fmt, float(rdo), out.ctypes.data), "bc_encode")
    return out


def bc6h_encode(rgba, ctx=None, out=None):
    a, w, h, stride = _img(rgba, np.float32)
    out = _out(out, bc_size(w, h, BC6H))
    check(load().zap_tex_cuda_bc6h_encode(ctx, a.ctypes.data, w, h, stride // 4, out.ctypes.data), "bc6h_encode")
    return out


def astc_encode(rgba, ctx=None, out=None):
    a, w, h, stride = _img(rgba, np.uint8)
    out = _out(out, bc_size(w, h, ASTC4X4))
    check(load().zap_tex_cuda_astc_encode(ctx, a.ctypes.data, w, h, stride, out.ctypes.data), "astc_encode")
    return out


def mip_next(rgba, srgb, ctx=None):
    a, w, h, stride = _img(rgba, np.uint8)
    nw, nh = max(1, w // 2), max(1, h // 2)
    out = np.empty((nh, nw, 4), np.uint8)
    check(load().zap_tex_cuda_mip_next(ctx, a.ctypes.data, w, h, stride, int(srgb), out.ctypes.data, nw * 4), "mip_next")
    return out


def mip_next_f(rgba, ctx=None):
    a, w, h, stride = _img(rgba, np.float32)
    nw, nh = max(1, w // 2), max(1, h // 2)
    out = np.empty((nh, nw, 4), np.float32)
    check(load().zap_tex_cuda_mip_next_f(ctx, a.ctypes.data, w, h, stride // 4, out.ctypes.data, nw * 4), "mip_next_f")
    return out


# ---------------------------------------------------------------- device memory (torch CUDA tensors)
def _stream(stream):
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return C.c_void_p(s.cuda_stream)


def _dev_img(t, channels=(4,)):
    if not t.is_cuda or t.dim() != 3 or t.shape[2] not in channels or t.stride(2) != 1 or t.stride(1) != t.shape[2]:
        raise ValueError(f"expected an HxWxC CUDA tensor with C in {channels} and packed rows, got {tuple(t.shape)}")
    return t.shape[1], t.shape[0], t.stride(0)


def bc_encode_dev(t, fmt, out=None, stream=None, ctx=None):
    """t: HxWxC uint8 CUDA tensor, C in (1, 2, 4); C < 4 reads missing channels as 0 and alpha as 255."""
    import torch
    if t.dtype != torch.uint8:
        raise ValueError("expected uint8")
    w, h, stride = _dev_img(t, (1, 2, 4))
    if out is None:
        out = torch.empty(bc_size(w, h, fmt), dtype=torch.uint8, device=t.device)
    check(load().zap_tex_cuda_bc_encode_u8_dev(ctx, t.data_ptr(), t.shape[2], w, h, stride, fmt, out.data_ptr(), _stream(stream)),
          "bc_encode_dev")
    return out


def bc_encode_rdo_dev(t, fmt, rdo, band_rows=0, out=None, stream=None, ctx=None):
    """Rate-distortion encode (zap_bc_encode with rdo > 0) of an HxWx4 uint8 CUDA tensor: one reference call over
    the whole image (band_rows 0), or one per band of band_rows block rows."""
    import torch
    w, h, stride = _dev_img(t, (4,))
    if out is None:
        out = torch.empty(bc_size(w, h, fmt), dtype=torch.uint8, device=t.device)
    check(load().zap_tex_cuda_bc_encode_rdo_dev(ctx, t.data_ptr(), w, h, stride, fmt, float(rdo), int(band_rows), out.data_ptr(),
                                                _stream(stream)), "bc_encode_rdo_dev")
    return out


def astc_encode_dev(t, out=None, stream=None, ctx=None):
    return bc_encode_dev(t, ASTC4X4, out, stream, ctx)


def bc6h_encode_dev(t, out=None, stream=None, ctx=None):
    """t: HxWx4 float32, or HxWx3 / HxWx4 float16 CUDA tensor."""
    import torch
    if t.dtype == torch.float32:
        w, h, stride = _dev_img(t, (4,))
    elif t.dtype == torch.float16:
        w, h, stride = _dev_img(t, (3, 4))
    else:
        raise ValueError("expected float32 RGBA or float16 RGB(A)")
    if out is None:
        out = torch.empty(bc_size(w, h, BC6H), dtype=torch.uint8, device=t.device)
    lib = load()
    if t.dtype == torch.float32:
        st = lib.zap_tex_cuda_bc6h_encode_dev(ctx, t.data_ptr(), w, h, stride, out.data_ptr(), _stream(stream))
    else:
        st = lib.zap_tex_cuda_bc6h_encode_half_dev(ctx, t.data_ptr(), t.shape[2], w, h, stride, out.data_ptr(), _stream(stream))
    check(st, "bc6h_encode_dev")
    return out


def mip_next_dev(t, srgb, out=None, stream=None, ctx=None):
    import torch
    w, h, stride = _dev_img(t, (4,))
    nw, nh = max(1, w // 2), max(1, h // 2)
    if out is None:
        out = torch.empty((nh, nw, 4), dtype=torch.uint8, device=t.device)
    check(load().zap_tex_cuda_mip_next_dev(ctx, t.data_ptr(), w, h, stride, int(srgb), out.data_ptr(), out.stride(0), _stream(stream)),
          "mip_next_dev")
    return out


def mip_next_f_dev(t, out=None, stream=None, ctx=None):
    import torch
    w, h, stride = _dev_img(t, (4,))
    nw, nh = max(1, w // 2), max(1, h // 2)
    if out is None:
        out = torch.empty((nh, nw, 4), dtype=torch.float32, device=t.device)
    check(load().zap_tex_cuda_mip_next_f_dev(ctx, t.data_ptr(), w, h, stride, out.data_ptr(), out.stride(0), _stream(stream)),
          "mip_next_f_dev")
    return out


def bc_decode_dev(bc, w, h, fmt, stream=None, ctx=None):
    """Device zap_bc_decode: uint8 CUDA tensor of blocks -> HxWx4 uint8 CUDA tensor."""
    import torch
    out = torch.empty((h, w, 4), dtype=torch.uint8, device=bc.device)
    check(load().zap_tex_cuda_bc_decode_dev(ctx, bc.data_ptr(), w, h, fmt, out.data_ptr(), w * 4, _stream(stream)), "bc_decode_dev")
    return out


def bc_split(bc, fmt, ctx=None):
    """zap_bc_split (zap_tex.h:1567) on the device: numpy uint8 blocks -> field planes (same size)."""
    bc = np.ascontiguousarray(bc, dtype=np.uint8)
    out = np.empty_like(bc)
    check(load().zap_tex_cuda_bc_split(ctx, bc.ctypes.data, bc.size, fmt, out.ctypes.data), "bc_split")
    return out


def bc_merge(planes, fmt, ctx=None):
    """zap_bc_merge (zap_tex.h:1568) on the device: numpy uint8 field planes -> blocks."""
    planes = np.ascontiguousarray(planes, dtype=np.uint8)
    out = np.empty_like(planes)
    check(load().zap_tex_cuda_bc_merge(ctx, planes.ctypes.data, planes.size, fmt, out.ctypes.data), "bc_merge")
    return out


def bc_split_dev(bc, fmt, out=None, stream=None, ctx=None):
    """Device split: uint8 CUDA tensor of blocks -> field planes (a new tensor unless out is given)."""
    import torch
    out = torch.empty_like(bc) if out is None else out
    check(load().zap_tex_cuda_bc_split_dev(ctx, bc.data_ptr(), bc.numel(), fmt, out.data_ptr(), _stream(stream)), "bc_split_dev")
    return out


def bc_merge_dev(planes, fmt, out=None, stream=None, ctx=None):
    """Device merge: uint8 CUDA tensor of field planes -> blocks."""
    import torch
    out = torch.empty_like(planes) if out is None else out
    check(load().zap_tex_cuda_bc_merge_dev(ctx, planes.data_ptr(), planes.numel(), fmt, out.data_ptr(), _stream(stream)), "bc_merge_dev")
    return out


def bc_encode_split_dev(t, fmt, out=None, stream=None, ctx=None):
    """Encode an HxWx4 uint8 CUDA tensor straight into the split form (the bytes of bc_split(bc_encode(t)))."""
    import torch
    w, h, stride = _dev_img(t, (4,))
    if out is None:
        out = torch.empty(bc_size(w, h, fmt), dtype=torch.uint8, device=t.device)
    check(load().zap_tex_cuda_bc_encode_split_dev(ctx, t.data_ptr(), w, h, stride, fmt, out.data_ptr(), _stream(stream)),
          "bc_encode_split_dev")
    return out


def bc6h_decode_dev(bc, w, h, stream=None, ctx=None):
    """Device zap_bc6h_decode: blocks -> HxWx4 int16 tensor holding half bits (alpha 0x3C00)."""
    import torch
    out = torch.empty((h, w, 4), dtype=torch.int16, device=bc.device)
    check(load().zap_tex_cuda_bc6h_decode_dev(ctx, bc.data_ptr(), w, h, out.data_ptr(), w * 4, _stream(stream)), "bc6h_decode_dev")
    return out


def astc_decode_dev(bc, w, h, stream=None, ctx=None):
    """Device zap_astc_decode: uint8 CUDA tensor of ASTC 4x4 blocks -> HxWx4 uint8 CUDA tensor."""
    import torch
    out = torch.empty((h, w, 4), dtype=torch.uint8, device=bc.device)
    check(load().zap_tex_cuda_astc_decode_dev(ctx, bc.data_ptr(), w, h, out.data_ptr(), w * 4, _stream(stream)), "astc_decode_dev")
    return out


def dds_header(w, h, fmt, mips=False, srgb=False):
    """The DDS header the CLI's tex command writes (zap.c:344-349): 128 or 148 bytes (DX10 extension) as numpy uint8."""
    hdr = np.zeros(148, np.uint8)
    n = C.c_size_t(0)
    check(load().zap_tex_cuda_dds_header(w, h, fmt, int(mips), int(srgb), hdr.ctypes.data, C.byref(n)), "dds_header")
    return hdr[:n.value]


def astc_header(w, h):
    """The 16-byte .astc header of zap.c:312-321."""
    hdr = np.zeros(16, np.uint8)
    check(load().zap_tex_cuda_astc_header(w, h, hdr.ctypes.data), "astc_header")
    return hdr


def tex_file(img, fmt, rdo=0.0, mips=False, srgb=False, ctx=None):
    """The whole file `zap tex` writes (zap.c:309-355), mip chain and blocks computed on the device: HxWx4 uint8 numpy
    image (rows may be padded) -> numpy uint8 file bytes (DDS for BC1..BC7, .astc for ASTC4X4)."""
    img = np.asarray(img, dtype=np.uint8)
    if img.strides[1:] != (4, 1):
        img = np.ascontiguousarray(img)
    h, w = img.shape[:2]
    n = load().zap_tex_cuda_tex_file_bytes(w, h, fmt, int(mips), int(srgb))
    out = np.empty(max(n, 1), np.uint8)
    check(load().zap_tex_cuda_tex_file(ctx, img.ctypes.data, w, h, img.strides[0], fmt, float(rdo), int(mips), int(srgb),
                                        out.ctypes.data, n), "tex_file")
    return out[:n]


def bc_decode(bc, w, h, fmt, ctx=None):
    """zap_bc_decode (zap_tex.h:1526) through the device: numpy blocks -> HxWx4 uint8 numpy array."""
    bc = np.ascontiguousarray(bc, dtype=np.uint8)
    out = np.empty((h, w, 4), np.uint8)
    check(load().zap_tex_cuda_bc_decode(ctx, bc.ctypes.data, w, h, fmt, out.ctypes.data, w * 4), "bc_decode")
    return out


def bc6h_decode(bc, w, h, ctx=None):
    """zap_bc6h_decode (zap_tex.h:963) through the device: numpy blocks -> HxWx4 uint16 half bits (alpha 0x3C00)."""
    bc = np.ascontiguousarray(bc, dtype=np.uint8)
    out = np.empty((h, w, 4), np.uint16)
    check(load().zap_tex_cuda_bc6h_decode(ctx, bc.ctypes.data, w, h, out.ctypes.data, w * 4), "bc6h_decode")
    return out


def astc_decode(bc, w, h, ctx=None):
    """zap_astc_decode (zap_tex.h:1344) through the device: numpy blocks -> HxWx4 uint8 numpy array."""
    bc = np.ascontiguousarray(bc, dtype=np.uint8)
    out = np.empty((h, w, 4), np.uint8)
    check(load().zap_tex_cuda_astc_decode(ctx, bc.ctypes.data, w, h, out.ctypes.data, w * 4), "astc_decode")
    return out


def endpoint_rows(fmt):
    """Endpoints per block in the differentiable decode: BC1 2 (RGB used), BC7 6 (endpoint 2s + k of subset s)."""
    return 2 if fmt == BC1 else 6


def block_endpoints_dev(blocks, fmt, stream=None, ctx=None):
    """Stored endpoints of BC1 / BC7 blocks, expanded to 8-bit units: float32 [nblocks, endpoint_rows(fmt), 4]."""
    import torch
    n = blocks.numel() // block_bytes(fmt)
    out = torch.empty((n, endpoint_rows(fmt), 4), dtype=torch.float32, device=blocks.device)
    check(load().zap_tex_cuda_block_endpoints_dev(ctx, fmt, blocks.data_ptr(), n, out.data_ptr(), _stream(stream)), "block_endpoints_dev")
    return out


def palette_decode_dev(blocks, fmt, endpoints, stream=None, ctx=None):
    """Linear palette decode with the blocks' indices held fixed: endpoints [n, rows, 4] -> texels float32 [n, 16, 4]."""
    import torch
    n = endpoints.shape[0]
    out = torch.empty((n, 16, 4), dtype=torch.float32, device=endpoints.device)
    check(load().zap_tex_cuda_palette_decode_dev(ctx, fmt, blocks.data_ptr(), n, endpoints.contiguous().data_ptr(), out.data_ptr(),
                                                 _stream(stream)), "palette_decode_dev")
    return out


def palette_adjoint_dev(blocks, fmt, grad_decoded, stream=None, ctx=None):
    """Adjoint of palette_decode_dev: gradient on decoded texels [n, 16, 4] -> gradient on endpoints [n, rows, 4]."""
    import torch
    n = grad_decoded.shape[0]
    out = torch.empty((n, endpoint_rows(fmt), 4), dtype=torch.float32, device=grad_decoded.device)
    check(load().zap_tex_cuda_palette_adjoint_dev(ctx, fmt, blocks.data_ptr(), n, grad_decoded.contiguous().data_ptr(), out.data_ptr(),
                                                  _stream(stream)), "palette_adjoint_dev")
    return out


def refine_dev(t, fmt, blocks, steps=8, lr=1.0, stream=None, ctx=None):
    """Gradient endpoint refinement of encoded blocks in place; returns per-block squared errors (before, after)."""
    import torch
    w, h, stride = _dev_img(t, (4,))
    n = ((w + 3) // 4) * ((h + 3) // 4)
    s0 = torch.empty(n, dtype=torch.int32, device=t.device)
    s1 = torch.empty(n, dtype=torch.int32, device=t.device)
    check(load().zap_tex_cuda_refine_dev(ctx, fmt, t.data_ptr(), w, h, stride, blocks.data_ptr(), int(steps), float(lr), s0.data_ptr(),
                                         s1.data_ptr(), _stream(stream)), "refine_dev")
    return s0, s1


class _Item(C.Structure):
    """zap_tex_cuda_item (include/zap_tex_cuda.h)."""
    _fields_ = [("src", C.c_void_p), ("w", C.c_int), ("h", C.c_int), ("stride", C.c_size_t), ("fmt", C.c_int),
                ("srgb", C.c_int), ("levels", C.c_int), ("dst", C.c_void_p)]


class Batch:
    """Many textures with their mip chains, mixed formats, encoded by one CUDA graph launch.

    textures: HxWx4 uint8 CUDA tensors (level 0); formats / srgb / levels: one per texture (levels 0 = full chain).
    After run(), outputs[i] holds texture i's levels concatenated, largest first (zap_bc_size bytes per level)."""

    PLAN_FLAGS = {"tiles_2d": 4, "regs_loose": 8, "tile_x2": 16, "tile_x4": 32, "cta_64": 64, "cta_256": 128}

    def __init__(self, textures, formats, srgb=None, levels=None, autotune=False, graph=True, ctx=None, plan=()):
        """plan: names from PLAN_FLAGS that fix a launch knob for every format class (without autotune)."""
        import torch
        n = len(textures)
        srgb = [1] * n if srgb is None else list(srgb)
        levels = [0] * n if levels is None else list(levels)
        lib = load()
        self.textures = list(textures)
        self.formats = list(formats)
        self.outputs = []
        items = (_Item * n)()
        for i, t in enumerate(self.textures):
            w, h, stride = _dev_img(t, (4,))
            nbytes = int(lib.zap_tex_cuda_batch_item_bytes(w, h, self.formats[i], levels[i]))
            out = torch.empty(max(1, nbytes), dtype=torch.uint8, device=t.device)
            self.outputs.append(out[:nbytes])
            items[i] = _Item(t.data_ptr(), w, h, stride, self.formats[i], int(srgb[i]), int(levels[i]), out.data_ptr())
        self._items = items
        flags = (1 if autotune else 0) | (0 if graph else 2)
        for name in plan:
            flags |= self.PLAN_FLAGS[name]
        handle = C.c_void_p()
        check(lib.zap_tex_cuda_batch_create(ctx, items, n, flags, C.byref(handle)), "batch_create")
        self._h = handle
        self.levels = [levels[i] or mip_levels(self.textures[i].shape[1], self.textures[i].shape[0]) for i in range(n)]
        self.pixels = 0
        for t, L in zip(self.textures, self.levels):
            w, h = t.shape[1], t.shape[0]
            for _ in range(L):
                self.pixels += w * h
                w, h = max(1, w // 2), max(1, h // 2)

    def run(self, stream=None):
        check(load().zap_tex_cuda_batch_run(self._h, _stream(stream)), "batch_run")

    def run_plain(self, stream=None):
        check(load().zap_tex_cuda_batch_run_plain(self._h, _stream(stream)), "batch_run_plain")

    def info(self):
        buf = C.create_string_buffer(4096)
        load().zap_tex_cuda_batch_info(self._h, buf, len(buf))
        return buf.value.decode()

    def level_views(self, i):
        """Texture i's encoded levels as separate uint8 tensors (views into outputs[i])."""
        t = self.textures[i]
        w, h, off, views = t.shape[1], t.shape[0], 0, []
        for _ in range(self.levels[i]):
            n = bc_size(w, h, self.formats[i])
            views.append(self.outputs[i][off:off + n])
            off += n
            w, h = max(1, w // 2), max(1, h // 2)
        return views

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            load().zap_tex_cuda_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def mip_chain_dev(t, srgb, stream=None, ctx=None):
    """Levels 1.. of t's mip chain as a list of HxWx4 uint8 CUDA tensors (views of one allocation)."""
    import torch
    w, h, stride = _dev_img(t, (4,))
    lib = load()
    buf = torch.empty(max(1, int(lib.zap_tex_cuda_mip_chain_bytes(w, h))), dtype=torch.uint8, device=t.device)
    check(lib.zap_tex_cuda_mip_chain_dev(ctx, t.data_ptr(), w, h, stride, int(srgb), buf.data_ptr(), _stream(stream)), "mip_chain_dev")
    levels, off = [], 0
    while w > 1 or h > 1:
        w, h = max(1, w // 2), max(1, h // 2)
        levels.append(buf[off:off + w * h * 4].view(h, w, 4))
        off += w * h * 4
    return levels
