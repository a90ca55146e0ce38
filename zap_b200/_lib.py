"""Loads the in-tree CUDA library (zap_b200/lib/libzap_tex_cuda.so) and declares its C ABI (include/zap_tex_cuda.h).

There is no CPU fallback: if the library cannot be built or loaded, every call raises.
"""
import ctypes as C
import os
import subprocess
import threading

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
# ZAP_TEX_CUDA_LIB selects another build of the same library (the bounds-check build, libzap_tex_cuda_checks.so)
LIB_PATH = os.environ.get("ZAP_TEX_CUDA_LIB") or os.path.join(PKG, "lib", "libzap_tex_cuda.so")

ZTC_OK = 0
STATUS = {0: "ok", -1: "invalid argument", -2: "unsupported", -3: "CUDA error", -4: "out of memory",
          -6: "no usable CUDA device"}

_lock = threading.Lock()
_lib = None


class ZapTexError(RuntimeError):
    def __init__(self, status, where, detail=""):
        self.status = status
        super().__init__(f"{where}: {STATUS.get(status, status)}" + (f" ({detail})" if detail else ""))


def build(verbose=False):
    """Compile every CUDA source for sm_100a into the in-tree shared library, and its bounds-check build
    (libzap_tex_cuda_checks.so), with nvcc, which cross-compiles without a GPU."""
    jobs = str(min(8, os.cpu_count() or 1))
    r = subprocess.run(["make", "-C", CSRC, "-j", jobs, "all", "checks"], capture_output=not verbose, text=True)
    if r.returncode != 0:
        raise RuntimeError("building libzap_tex_cuda.so failed:\n" + (r.stdout or "") + (r.stderr or ""))
    return LIB_PATH


def _declare(lib):
    vp, i, sz, f, cp = C.c_void_p, C.c_int, C.c_size_t, C.c_float, C.c_char_p
    sig = {
        "zap_tex_cuda_version": ([], i),
        "zap_tex_cuda_status_string": ([i], cp),
        "zap_tex_cuda_last_error": ([], cp),
        "zap_tex_cuda_create": ([i, C.POINTER(vp)], i),
        "zap_tex_cuda_destroy": ([vp], i),
        "zap_tex_cuda_reserve": ([vp, sz], i),
        "zap_tex_cuda_trace_enable": ([i], i),
        "zap_tex_cuda_trace_report": ([C.c_char_p, sz], i),
        "zap_tex_cuda_block_bytes": ([i], sz),
        "zap_tex_cuda_bc_size": ([i, i, i], sz),
        "zap_tex_cuda_mip_levels": ([i, i], i),
        "zap_tex_cuda_bc_encode": ([vp, vp, i, i, sz, i, f, vp], i),
        "zap_tex_cuda_bc6h_encode": ([vp, vp, i, i, sz, vp], i),
        "zap_tex_cuda_astc_encode": ([vp, vp, i, i, sz, vp], i),
        "zap_tex_cuda_mip_next": ([vp, vp, i, i, sz, i, vp, sz], i),
        "zap_tex_cuda_mip_next_f": ([vp, vp, i, i, sz, vp, sz], i),
        "zap_tex_cuda_bc_encode_dev": ([vp, vp, i, i, sz, i, f, vp, vp], i),
        "zap_tex_cuda_bc_encode_rdo_dev": ([vp, vp, i, i, sz, i, f, i, vp, vp], i),
        "zap_tex_cuda_bc6h_encode_dev": ([vp, vp, i, i, sz, vp, vp], i),
        "zap_tex_cuda_astc_encode_dev": ([vp, vp, i, i, sz, vp, vp], i),
        "zap_tex_cuda_mip_next_dev": ([vp, vp, i, i, sz, i, vp, sz, vp], i),
        "zap_tex_cuda_mip_next_f_dev": ([vp, vp, i, i, sz, vp, sz, vp], i),
        "zap_tex_cuda_bc_encode_u8_dev": ([vp, vp, i, i, i, sz, i, vp, vp], i),
        "zap_tex_cuda_bc6h_encode_half_dev": ([vp, vp, i, i, i, sz, vp, vp], i),
        "zap_tex_cuda_mip_chain_bytes": ([i, i], sz),
        "zap_tex_cuda_mip_chain_dev": ([vp, vp, i, i, sz, i, vp, vp], i),
        "zap_tex_cuda_bc7_encode_noalloc_dev": ([vp, i, i, sz, vp, vp], i),
        "zap_tex_cuda_bc_decode_dev": ([vp, vp, i, i, i, vp, sz, vp], i),
        "zap_tex_cuda_bc6h_decode_dev": ([vp, vp, i, i, vp, sz, vp], i),
        "zap_tex_cuda_astc_decode_dev": ([vp, vp, i, i, vp, sz, vp], i),
        "zap_tex_cuda_bc_decode": ([vp, vp, i, i, i, vp, sz], i),
        "zap_tex_cuda_bc6h_decode": ([vp, vp, i, i, vp, sz], i),
        "zap_tex_cuda_astc_decode": ([vp, vp, i, i, vp, sz], i),
        "zap_tex_cuda_bc_split": ([vp, vp, sz, i, vp], i),
        "zap_tex_cuda_bc_merge": ([vp, vp, sz, i, vp], i),
        "zap_tex_cuda_bc_split_dev": ([vp, vp, sz, i, vp, vp], i),
        "zap_tex_cuda_bc_merge_dev": ([vp, vp, sz, i, vp, vp], i),
        "zap_tex_cuda_bc_encode_split_dev": ([vp, vp, i, i, sz, i, vp, vp], i),
        "zap_tex_cuda_block_endpoints_dev": ([vp, i, vp, i, vp, vp], i),
        "zap_tex_cuda_palette_decode_dev": ([vp, i, vp, i, vp, vp, vp], i),
        "zap_tex_cuda_palette_adjoint_dev": ([vp, i, vp, i, vp, vp, vp], i),
        "zap_tex_cuda_refine_dev": ([vp, i, vp, i, i, sz, vp, i, f, vp, vp, vp], i),
        "zap_tex_cuda_batch_item_bytes": ([i, i, i, i], sz),
        "zap_tex_cuda_batch_create": ([vp, vp, i, i, C.POINTER(vp)], i),
        "zap_tex_cuda_batch_run": ([vp, vp], i),
        "zap_tex_cuda_batch_run_plain": ([vp, vp], i),
        "zap_tex_cuda_batch_info": ([vp, C.c_char_p, sz], i),
        "zap_tex_cuda_batch_destroy": ([vp], i),
        "zap_tex_cuda_dds_header": ([i, i, i, i, i, vp, C.POINTER(sz)], i),
        "zap_tex_cuda_astc_header": ([i, i, vp], i),
        "zap_tex_cuda_tex_file_bytes": ([i, i, i, i, i], sz),
        "zap_tex_cuda_tex_file": ([vp, vp, i, i, sz, i, f, i, i, vp, sz], i),
        "zap_tex_cuda_alu_probe_dev": ([i, i, vp, vp, C.POINTER(C.c_double)], i),
        "zap_tex_cuda_debug_fail_allocations": ([i, i], i),
        "zap_tex_cuda_debug_checks": ([C.POINTER(C.c_uint)], i),
    }
    for name, (args, res) in sig.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    return sig


def exported_names():
    """Every entry point this module declares (the test suite checks they match include/zap_tex_cuda.h)."""
    return sorted(_declare(load()).keys())


def load():
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                build()
            lib = C.CDLL(LIB_PATH)
            _declare(lib)
            _lib = lib
        return _lib


def check(status, where):
    if status != ZTC_OK:
        detail = load().zap_tex_cuda_last_error().decode(errors="replace")
        raise ZapTexError(status, where, detail)
