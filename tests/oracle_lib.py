"""ctypes access to the oracle (test infrastructure only).

Two libraries, both built by oracle/Makefile:
  - oracle/liboracle.so      : the C restatement (zt_oracle.c), always buildable from the repo;
  - oracle/_ref/libzapref.so : the reference's own zap_tex.h behind a shim, built where the reference tree exists
                               (it travels with the repo to machines that lack the tree).
Both expose the same numpy-level API below, so a test can check the product against either.
"""
import ctypes as C
import os
import subprocess
import threading

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
PORT_SO = os.path.join(ORACLE_DIR, "liboracle.so")
REF_SO = os.path.join(ORACLE_DIR, "_ref", "libzapref.so")
REF_TREE = os.environ.get("ZAP_REF_DIR", "/root/reference")  # the reference source tree, where one exists

BC1, BC3, BC4, BC5, BC7 = 0, 1, 2, 3, 4
_lock = threading.Lock()
_cache = {}


def _make(target):
    subprocess.run(["make", "-s", "-C", ORACLE_DIR, target], check=True, stdout=subprocess.DEVNULL)


def block_bytes(fmt):
    return 8 if fmt in (BC1, BC4) else 16


def bc_size(w, h, fmt):
    return ((w + 3) // 4) * ((h + 3) // 4) * block_bytes(fmt)


class Oracle:
    """numpy wrapper over one oracle library (prefix zo_ for the restatement, zr_ for the reference)."""

    def __init__(self, path, prefix, kind):
        self.lib = C.CDLL(path)
        self.p = prefix
        self.kind = kind  # "port" or "reference"
        vp, i, sz, f = C.c_void_p, C.c_int, C.c_size_t, C.c_float
        self._fn("bc_encode", [vp, i, i, sz, i, f, vp], None)
        self._fn("bc_decode", [vp, i, i, i, vp, sz], None)
        self._fn("bc6h_encode", [vp, i, i, sz, vp], None)
        self._fn("bc6h_decode", [vp, i, i, vp, sz], None)
        self._fn("astc_encode", [vp, i, i, sz, vp], None)
        self._fn("astc_decode", [vp, i, i, vp, sz], None)
        self._fn("mip_levels", [i, i], C.c_int)
        self._fn("mip_next", [vp, i, i, sz, i, vp, sz], None)
        self._fn("mip_next_f", [vp, i, i, sz, vp, sz], None)
        self._fn("f2h", [C.c_float], C.c_uint16)
        self._fn("h2f", [C.c_uint16], C.c_float)
        self._fn("bc_split", [vp, sz, i, vp], None)
        self._fn("bc_merge", [vp, sz, i, vp], None)
        if kind == "port":
            self._fn("astc_partition", [i, i, i, i], C.c_int)
            self._fn("ise_roundtrip", [i, i, vp, vp], C.c_int)
            self._fn("srgb_tables", [vp, vp], None)
            self._fn("dds_header", [i, i, i, i, i, vp], sz)
            self._fn("astc_header", [i, i, vp], None)
            self._fn("tex_file", [vp, i, i, sz, i, f, i, i, vp], sz)
            self._fn("bc7_fields", [vp, vp, vp, vp, vp, vp], C.c_int)
        else:
            self._fn("astc_part", [i, i, i, i], C.c_int)
            self._fn("srgb_lin", [], C.POINTER(C.c_float))
            self._fn("srgb_thr", [], C.POINTER(C.c_float))
            self._fn("bc_encode_mt", [vp, i, i, sz, i, vp, i], C.c_int)
            self._fn("bc6h_encode_mt", [vp, i, i, sz, vp, i], C.c_int)
            self._fn("astc_encode_mt", [vp, i, i, sz, vp, i], C.c_int)

    def _fn(self, name, argtypes, restype):
        fn = getattr(self.lib, self.p + name)
        fn.argtypes = argtypes
        fn.restype = restype
        setattr(self, "_" + name, fn)

    # ---- encoders (img: HxWx4 uint8 or float32, C-contiguous rows; stride = row pitch)
    def bc_encode(self, img, fmt, threads=1, rdo=0.0):
        img = np.ascontiguousarray(img)
        h, w = img.shape[:2]
        out = np.zeros(bc_size(w, h, fmt), np.uint8)
        if threads > 1 and self.kind == "reference" and rdo <= 0:
            self._bc_encode_mt(img.ctypes.data, w, h, w * 4, fmt, out.ctypes.data, threads)
        else:
            self._bc_encode(img.ctypes.data, w, h, w * 4, fmt, float(rdo), out.ctypes.data)
        return out

    def bc6h_encode(self, img, threads=1):
        img = np.ascontiguousarray(img, dtype=np.float32)
        h, w = img.shape[:2]
        out = np.zeros(bc_size(w, h, BC7), np.uint8)
        if threads > 1 and self.kind == "reference":
            self._bc6h_encode_mt(img.ctypes.data, w, h, w * 4, out.ctypes.data, threads)
        else:
            self._bc6h_encode(img.ctypes.data, w, h, w * 4, out.ctypes.data)
        return out

    def astc_encode(self, img, threads=1):
        img = np.ascontiguousarray(img)
        h, w = img.shape[:2]
        out = np.zeros(bc_size(w, h, BC7), np.uint8)
        if threads > 1 and self.kind == "reference":
            self._astc_encode_mt(img.ctypes.data, w, h, w * 4, out.ctypes.data, threads)
        else:
            self._astc_encode(img.ctypes.data, w, h, w * 4, out.ctypes.data)
        return out

    def bc7_fields(self, blk):
        """One BC7 block's fields (restatement only): mode, subsets, partition, rotation, alpha bits, expanded
        endpoints [6][4] (endpoint 2s + k of subset s), per-texel subset and colour / alpha weights (0..64)."""
        blk = np.ascontiguousarray(blk, dtype=np.uint8)
        info = np.zeros(5, np.int32)
        ep = np.zeros((6, 4), np.int32)
        sub, cw, aw = np.zeros(16, np.int32), np.zeros(16, np.int32), np.zeros(16, np.int32)
        self._bc7_fields(blk.ctypes.data, info.ctypes.data, ep.ctypes.data, sub.ctypes.data, cw.ctypes.data, aw.ctypes.data)
        return {"mode": int(info[0]), "ns": int(info[1]), "part": int(info[2]), "rot": int(info[3]), "ab": int(info[4]),
                "ep": ep.tolist(), "subset": sub.tolist(), "cw": cw.tolist(), "aw": aw.tolist()}

    # ---- the CLI's containers (zap.c:309-355; restatement only)
    def dds_header(self, w, h, fmt, mips, srgb):
        hdr = np.zeros(148, np.uint8)
        n = self._dds_header(w, h, fmt, int(mips), int(srgb), hdr.ctypes.data)
        return hdr[:n]

    def astc_header(self, w, h):
        hdr = np.zeros(16, np.uint8)
        self._astc_header(w, h, hdr.ctypes.data)
        return hdr

    def tex_file(self, img, fmt, rdo=0.0, mips=0, srgb=0):
        img = np.ascontiguousarray(img)
        h, w = img.shape[:2]
        n = self._tex_file(img.ctypes.data, w, h, w * 4, fmt, float(rdo), int(mips), int(srgb), None)
        out = np.zeros(n, np.uint8)
        self._tex_file(img.ctypes.data, w, h, w * 4, fmt, float(rdo), int(mips), int(srgb), out.ctypes.data)
        return out

    # ---- decoders
    def bc_split(self, bc, fmt):
        bc = np.ascontiguousarray(bc, dtype=np.uint8)
        out = np.zeros_like(bc)
        self._bc_split(bc.ctypes.data, bc.size, fmt, out.ctypes.data)
        return out

    def bc_merge(self, planes, fmt):
        planes = np.ascontiguousarray(planes, dtype=np.uint8)
        out = np.zeros_like(planes)
        self._bc_merge(planes.ctypes.data, planes.size, fmt, out.ctypes.data)
        return out

    def bc_decode(self, bc, w, h, fmt):
        out = np.zeros((h, w, 4), np.uint8)
        bc = np.ascontiguousarray(bc)
        self._bc_decode(bc.ctypes.data, w, h, fmt, out.ctypes.data, w * 4)
        return out

    def bc6h_decode(self, bc, w, h):
        out = np.zeros((h, w, 4), np.uint16)
        bc = np.ascontiguousarray(bc)
        self._bc6h_decode(bc.ctypes.data, w, h, out.ctypes.data, w * 4)
        return out

    def astc_decode(self, bc, w, h):
        out = np.zeros((h, w, 4), np.uint8)
        bc = np.ascontiguousarray(bc)
        self._astc_decode(bc.ctypes.data, w, h, out.ctypes.data, w * 4)
        return out

    # ---- mips
    def mip_levels(self, w, h):
        return self._mip_levels(w, h)

    def mip_next(self, img, srgb):
        img = np.ascontiguousarray(img)
        h, w = img.shape[:2]
        nw, nh = max(1, w // 2), max(1, h // 2)
        out = np.zeros((nh, nw, 4), np.uint8)
        self._mip_next(img.ctypes.data, w, h, w * 4, int(srgb), out.ctypes.data, nw * 4)
        return out

    def mip_next_f(self, img):
        img = np.ascontiguousarray(img, dtype=np.float32)
        h, w = img.shape[:2]
        nw, nh = max(1, w // 2), max(1, h // 2)
        out = np.zeros((nh, nw, 4), np.float32)
        self._mip_next_f(img.ctypes.data, w, h, w * 4, out.ctypes.data, nw * 4)
        return out

    # ---- internals pinned by the reference self-test
    def f2h(self, f):
        return self._f2h(f)

    def h2f(self, h):
        return self._h2f(h)

    def astc_partition(self, seed, x, y, count):
        fn = self._astc_partition if self.kind == "port" else self._astc_part
        return fn(seed, x, y, count)

    def srgb_tables(self):
        if self.kind == "port":
            lin = np.zeros(256, np.float32)
            thr = np.zeros(255, np.float32)
            self._srgb_tables(lin.ctypes.data, thr.ctypes.data)
            return lin, thr
        lin = np.ctypeslib.as_array(self._srgb_lin(), (256,)).copy()
        thr = np.ctypeslib.as_array(self._srgb_thr(), (255,)).copy()
        return lin, thr


def port():
    with _lock:
        if "port" not in _cache:
            _make("port")  # cheap when up to date; always rebuilt from the committed restatement
            _cache["port"] = Oracle(PORT_SO, "zo_", "port")
        return _cache["port"]


def reference():
    """The reference library, or None when it is neither built nor buildable here."""
    with _lock:
        if "ref" not in _cache:
            if os.path.isdir(REF_TREE):
                _make("ref")
            _cache["ref"] = Oracle(REF_SO, "zr_", "reference") if os.path.exists(REF_SO) else None
        return _cache["ref"]


def best():
    """The reference when available, else the restatement (which the CPU suite pins to the reference)."""
    return reference() or port()


def psnr(a, b, chmask):
    """tex_bench.c:17-22: PSNR over the channels in chmask; 99 when identical."""
    a = a.reshape(-1, 4).astype(np.float64)
    b = b.reshape(-1, 4).astype(np.float64)
    ch = [c for c in range(4) if (chmask >> c) & 1]
    se = float(np.sum((a[:, ch] - b[:, ch]) ** 2))
    n = a.shape[0] * len(ch)
    return 99.0 if se == 0 else 10 * np.log10(255.0 * 255.0 * n / se)


def chmask(fmt):
    return {BC1: 7, BC4: 1, BC5: 3}.get(fmt, 15)
