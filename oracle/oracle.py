"""ctypes front-end to the CPU oracle -- TEST INFRASTRUCTURE ONLY.

Loads oracle/liboracle.so (this repository's plain-C restatement of the
reference algorithm) and, when it was built here, oracle/_ref (the reference
compiled from its own sources). Only tests/, ``__graft_entry__.smoke()`` and
bench.py's CPU-baseline leg import this module, and only as the checker.
"""
from __future__ import annotations

import ctypes as C
import os
import struct
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")
_u16p = np.ctypeslib.ndpointer(np.uint16, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")

_lib = None
_ref = None


def build(quiet: bool = True) -> None:
    """make -C oracle (the restatement); cheap when up to date."""
    out = subprocess.run(["make", "-C", HERE], capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout + out.stderr)


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        L.orc_branch_levels.argtypes = [C.c_int, C.c_int, _f64p]
        L.orc_fixed_scale.argtypes = [C.c_int]
        L.orc_fixed_scale.restype = C.c_double
        L.orc_refine_tables.argtypes = [C.c_int, C.c_int, _f32p]
        L.orc_scan_class_means.argtypes = [C.c_int, _f64p]
        L.orc_merged_alternating.argtypes = [C.c_int]
        L.orc_encode.argtypes = [_f32p, C.c_size_t, C.c_int, C.c_int, C.c_double, _u16p, _u8p]
        L.orc_pack_coarse.argtypes = [_u16p, C.c_int, C.c_int]
        L.orc_pack_coarse.restype = C.c_uint8
        L.orc_pack_refine.argtypes = [_u16p, C.c_int, C.c_int, _u8p]
        L.orc_decode_split.argtypes = [C.c_int, C.c_uint8, _u8p, _u16p, C.POINTER(C.c_int)]
        L.orc_padded_dim.argtypes = [C.c_size_t]
        L.orc_padded_dim.restype = C.c_size_t
        L.orc_sign_bytes.argtypes = [C.c_size_t]
        L.orc_sign_bytes.restype = C.c_size_t
        L.orc_rotator_signs.argtypes = [C.c_size_t, C.c_uint64, _u8p]
        L.orc_rotate.argtypes = [C.c_size_t, _u8p, _f32p, _f32p]
        L.orc_e8q_build.argtypes = [_f32p, _f32p, _u32p, C.c_size_t, C.c_size_t, C.c_size_t,
                                    C.c_int, C.c_uint64, C.c_int]
        L.orc_e8q_build.restype = C.c_void_p
        L.orc_e8q_free.argtypes = [C.c_void_p]
        L.orc_e8q_prepare_query.argtypes = [C.c_void_p, _f32p, _f32p]
        L.orc_e8q_exact_score.argtypes = [C.c_void_p, C.c_size_t, _f32p]
        L.orc_e8q_exact_score.restype = C.c_float
        L.orc_e8q_estimate.argtypes = [C.c_void_p, _f32p, C.c_uint32]
        L.orc_e8q_estimate.restype = C.c_float
        L.orc_e8q_probe_bound_w.argtypes = [C.c_void_p, _f32p, _f32p, C.c_uint32]
        L.orc_e8q_probe_bound_w.restype = C.c_double
        L.orc_e8q_route.argtypes = [C.c_void_p, _f32p, C.c_size_t, _u32p, _f32p]
        L.orc_e8q_search.argtypes = [C.c_void_p, _f32p, C.c_size_t, C.c_size_t, C.c_size_t,
                                     _u32p, _f32p, C.c_int]
        L.orc_phi_inv.argtypes = [C.c_double]
        L.orc_phi_inv.restype = C.c_double
        L.orc_ortho_quantile.argtypes = [C.c_double, C.c_size_t]
        L.orc_ortho_quantile.restype = C.c_float
        L.orc_e8q_banks.argtypes = [C.c_void_p, C.c_void_p]
        L.orc_e8q_banks.restype = C.c_size_t
        L.orc_e8q_prepare_lut.argtypes = [C.c_int, C.c_int, _f32p, _u8p, _f32p]
        L.orc_e8q_coarse.argtypes = [C.c_void_p, C.c_size_t, _u8p]
        L.orc_e8q_coarse.restype = C.c_int32
        L.orc_e8q_refine_score.argtypes = [C.c_void_p, C.c_size_t, _f32p]
        L.orc_e8q_refine_score.restype = C.c_float
        L.orc_e8q_search_pruned.argtypes = [C.c_void_p, C.c_void_p, C.c_float, C.c_int, _f32p,
                                            C.c_size_t, C.c_size_t, C.c_size_t, _u32p, _f32p,
                                            C.c_void_p, C.c_void_p, C.c_int]
        L.orc_me8q_variance.argtypes = [_f32p, C.c_size_t, C.c_size_t, C.c_size_t, _f32p]
        L.orc_me8q_allocate.argtypes = [_f32p, C.c_size_t, C.c_float, C.c_int, C.c_double,
                                        C.POINTER(C.c_size_t), C.POINTER(C.c_int)]
        L.orc_me8q_allocate.restype = C.c_int
        L.orc_me8q_build.argtypes = [_f32p, _f32p, _u32p, C.c_size_t, C.c_size_t, C.c_size_t,
                                     C.POINTER(C.c_size_t), C.POINTER(C.c_int), C.c_int, C.c_uint64,
                                     C.c_int, C.c_int]
        L.orc_me8q_build.restype = C.c_void_p
        L.orc_me8q_free.argtypes = [C.c_void_p]
        L.orc_me8q_shape.argtypes = [C.c_void_p, C.POINTER(C.c_size_t), C.POINTER(C.c_size_t),
                                     C.POINTER(C.c_int)]
        L.orc_me8q_codes.argtypes = [C.c_void_p, C.c_size_t, _u16p, _u8p, _f32p, _f32p]
        L.orc_me8q_ids.argtypes = [C.c_void_p, _u32p]
        L.orc_me8q_estimate.argtypes = [C.c_void_p, _f32p, C.c_uint32]
        L.orc_me8q_estimate.restype = C.c_float
        L.orc_me8q_search.argtypes = [C.c_void_p, _f32p, C.c_size_t, C.c_size_t, C.c_size_t,
                                      _u32p, _f32p, C.c_int]
        _u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")
        L.orc_me8q_search_pruned.argtypes = [C.c_void_p, _f32p, C.c_size_t, C.c_size_t, C.c_size_t, C.c_float,
                                             _u32p, _f32p, _u64p, _u64p, C.c_int]
        _lib = L
    return _lib


def ref_lib():
    """The reference's own code (oracle/_ref/libe8qref.so) or None."""
    global _ref
    if _ref is None:
        path = os.path.join(REF_DIR, "libe8qref.so")
        if not os.path.exists(path):
            return None
        L = C.CDLL(path)
        L.ref_branch_levels.argtypes = [C.c_int, C.c_int, _f64p]
        L.ref_fixed_scale.argtypes = [C.c_int]
        L.ref_fixed_scale.restype = C.c_double
        L.ref_encode.argtypes = [_f32p, C.c_size_t, C.c_int, C.c_int, C.c_double, _u16p, _u8p]
        L.ref_rotator_sign_bytes.argtypes = [C.c_size_t, C.c_uint64]
        L.ref_rotator_sign_bytes.restype = C.c_size_t
        L.ref_rotator_signs.argtypes = [C.c_size_t, C.c_uint64, _u8p]
        L.ref_rotate.argtypes = [C.c_size_t, C.c_uint64, _f32p, C.c_size_t, _f32p]
        L.ref_refine_tables.argtypes = [C.c_int, C.c_int, _f32p]
        L.ref_pack_block.argtypes = [_u16p, C.c_int, C.c_int, _u8p, _u8p]
        L.ref_scan_class_means.argtypes = [C.c_int, _f64p]
        _ref = L
    return _ref


def ref_module():
    """The reference's pybind11 module (imported as e8qlib_ref) or None."""
    if not os.path.isdir(os.path.join(REF_DIR, "e8qlib_ref")):
        return None
    if REF_DIR not in sys.path:
        sys.path.insert(0, REF_DIR)
    import e8qlib_ref  # noqa: E402

    return e8qlib_ref


# ---- restatement wrappers ---------------------------------------------------

def padded_dim(dim: int) -> int:
    return (dim + 63) // 64 * 64


def branch_levels(bits: int, branch: int, L=None) -> np.ndarray:
    L = L or lib()
    out = np.zeros(1 << bits, np.float64)
    (L.orc_branch_levels if hasattr(L, "orc_branch_levels") else L.ref_branch_levels)(
        bits, branch, out)
    return out


def fixed_scale(bits: int) -> float:
    return lib().orc_fixed_scale(bits)


def refine_tables(bits: int, pd: int) -> np.ndarray:
    out = np.zeros(2 * max(256, 1 << bits), np.float32)
    lib().orc_refine_tables(bits, pd, out)
    return out


def encode(unit: np.ndarray, bits: int, s: float | None = None):
    """unit [n, Dpad] float32 -> (digits [n, B, 8] u16, branch [n, B] u8)."""
    unit = np.ascontiguousarray(unit, np.float32)
    n, pd = unit.shape
    s = fixed_scale(bits) if s is None else s
    dg = np.zeros((n, pd // 8, 8), np.uint16)
    br = np.zeros((n, pd // 8), np.uint8)
    lib().orc_encode(unit, n, pd, bits, s, dg, br)
    return dg, br


def ref_encode(unit: np.ndarray, bits: int, s: float | None = None):
    R = ref_lib()
    unit = np.ascontiguousarray(unit, np.float32)
    n, pd = unit.shape
    s = R.ref_fixed_scale(bits) if s is None else s
    dg = np.zeros((n, pd // 8, 8), np.uint16)
    br = np.zeros((n, pd // 8), np.uint8)
    R.ref_encode(unit, n, pd, bits, s, dg, br)
    return dg, br


def rotator_signs(dim: int, seed: int) -> np.ndarray:
    out = np.zeros(lib().orc_sign_bytes(dim), np.uint8)
    lib().orc_rotator_signs(dim, seed, out)
    return out


def rotate(x: np.ndarray, dim: int, signs: np.ndarray) -> np.ndarray:
    x = np.ascontiguousarray(np.atleast_2d(x), np.float32)
    pd = padded_dim(dim)
    out = np.zeros((x.shape[0], pd), np.float32)
    for i in range(x.shape[0]):
        row = np.ascontiguousarray(x[i])
        o = np.zeros(pd, np.float32)
        lib().orc_rotate(dim, signs, row, o)
        out[i] = o
    return out


class OracleE8qIndex:
    """The restated E8Q index (plain path) as a Python object."""

    def __init__(self, data, centroids, cluster_ids, bits, seed=0, threads=8):
        data = np.ascontiguousarray(data, np.float32)
        centroids = np.ascontiguousarray(centroids, np.float32)
        cluster_ids = np.ascontiguousarray(cluster_ids, np.uint32)
        self.n, self.dim = data.shape
        self.nlist = centroids.shape[0]
        self.bits = bits
        self.pd = padded_dim(self.dim)
        self.blocks = self.pd // 8
        self._p = lib().orc_e8q_build(data, centroids, cluster_ids, self.n, self.dim,
                                      self.nlist, bits, seed, threads)
        if not self._p:
            raise ValueError("oracle build rejected its inputs")
        self._export()

    def _export(self):
        class _S(C.Structure):
            _fields_ = [("n", C.c_size_t), ("dim", C.c_size_t), ("padded_dim", C.c_size_t),
                        ("nlist", C.c_size_t), ("bits", C.c_int), ("blocks", C.c_int),
                        ("signs", C.c_void_p), ("mean_rot", C.c_void_p),
                        ("centroid_rot", C.c_void_p), ("cn2", C.c_void_p),
                        ("list_begin", C.c_void_p), ("ids", C.c_void_p),
                        ("digits", C.c_void_p), ("branch", C.c_void_p), ("g1", C.c_void_p),
                        ("h3", C.c_void_p), ("tab", C.c_void_p), ("tab_stride", C.c_int)]
        s = _S.from_address(self._p)

        def arr(ptr, n, dt):
            return np.ctypeslib.as_array(C.cast(ptr, C.POINTER(np.ctypeslib.as_ctypes_type(dt))),
                                         shape=(n,)).copy()
        B = self.blocks
        self.signs = arr(s.signs, 4 * self.pd // 8, np.uint8)
        self.mean_rot = arr(s.mean_rot, self.pd, np.float32)
        self.centroid_rot = arr(s.centroid_rot, self.nlist * self.pd, np.float32).reshape(
            self.nlist, self.pd)
        self.cn2 = arr(s.cn2, self.nlist, np.float32)
        self.list_begin = arr(s.list_begin, self.nlist + 1, np.uint64)
        self.ids = arr(s.ids, self.n, np.uint32)
        self.digits = arr(s.digits, self.n * B * 8, np.uint16).reshape(self.n, B, 8)
        self.branch = arr(s.branch, self.n * B, np.uint8).reshape(self.n, B)
        self.g1 = arr(s.g1, self.n, np.float32)
        self.h3 = arr(s.h3, self.n, np.float32)
        self.tab_stride = s.tab_stride
        self.tab = arr(s.tab, 2 * s.tab_stride, np.float32)

    def __del__(self):
        if getattr(self, "_p", None):
            lib().orc_e8q_free(self._p)
            self._p = None

    def prepare_query(self, q):
        q = np.ascontiguousarray(q, np.float32)
        out = np.zeros(self.pd, np.float32)
        lib().orc_e8q_prepare_query(self._p, q, out)
        return out

    def exact_score(self, pos, rot_q):
        return lib().orc_e8q_exact_score(self._p, pos, np.ascontiguousarray(rot_q, np.float32))

    def estimate(self, q, gid):
        return lib().orc_e8q_estimate(self._p, np.ascontiguousarray(q, np.float32), gid)

    def probe_bound_w(self, queries, base_rows, qidx, ids):
        """ProbeBoundW per pair i: queries[qidx[i]] against the stored vector
        ids[i] whose raw input is base_rows[i]; NaN where qidx or the id is out
        of range (as the reference's binding)."""
        queries = np.ascontiguousarray(np.atleast_2d(queries), np.float32)
        base_rows = np.ascontiguousarray(np.atleast_2d(base_rows), np.float32)
        out = np.full(len(ids), np.nan)
        for i, (qi, gid) in enumerate(zip(qidx, ids)):
            if qi < queries.shape[0] and gid < self.n:
                out[i] = lib().orc_e8q_probe_bound_w(self._p, queries[qi], base_rows[i], int(gid))
        return out

    def route(self, rot_q, nprobe):
        take = min(nprobe, self.nlist)
        ids = np.zeros(take, np.uint32)
        d2 = np.zeros(take, np.float32)
        lib().orc_e8q_route(self._p, np.ascontiguousarray(rot_q, np.float32), take, ids, d2)
        return ids, d2

    def search(self, queries, k, nprobe, threads=8):
        queries = np.ascontiguousarray(np.atleast_2d(queries), np.float32)
        nq = queries.shape[0]
        ids = np.zeros((nq, k), np.uint32)
        dists = np.zeros((nq, k), np.float32)
        lib().orc_e8q_search(self._p, queries, nq, k, nprobe, ids, dists, threads)
        return ids, dists

    def banks(self):
        """The 128-byte scan-bank header of every 32-row batch, lists in
        order: (nbatches, 128) uint8."""
        nb = lib().orc_e8q_banks(self._p, None)
        out = np.zeros((nb, 128), np.uint8)
        lib().orc_e8q_banks(self._p, out.ctypes.data)
        return out

    def prepare_lut(self, rot_q):
        """PrepareQuery's u8 LUT (blocks x 32) and (delta, base, lut_err, score_max)."""
        lut = np.zeros((self.blocks, 32), np.uint8)
        scal = np.zeros(4, np.float32)
        lib().orc_e8q_prepare_lut(self.bits, self.blocks, np.ascontiguousarray(rot_q, np.float32), lut, scal)
        return lut, scal

    def prepare_query(self, q):
        rq = np.zeros(self.pd, np.float32)
        lib().orc_e8q_prepare_query(self._p, np.ascontiguousarray(q, np.float32), rq)
        return rq

    def coarse(self, pos, lut):
        return int(lib().orc_e8q_coarse(self._p, pos, np.ascontiguousarray(lut)))

    def refine_score(self, pos, rot_q):
        return float(lib().orc_e8q_refine_score(self._p, pos, np.ascontiguousarray(rot_q, np.float32)))


    def search_pruned(self, queries, k, nprobe, alpha=1.0, disable_prune=False, banks=None, threads=8):
        """The reference's shipped sequential pruned search; returns ids,
        dists and per-query (candidates, survivors)."""
        queries = np.ascontiguousarray(np.atleast_2d(queries), np.float32)
        nq = queries.shape[0]
        ids = np.zeros((nq, k), np.uint32)
        dists = np.zeros((nq, k), np.float32)
        cand = np.zeros(nq, np.uint64)
        surv = np.zeros(nq, np.uint64)
        bk = None if banks is None else np.ascontiguousarray(banks, np.uint8)
        lib().orc_e8q_search_pruned(self._p, None if bk is None else bk.ctypes.data, alpha,
                                    1 if disable_prune else 0, queries, nq, k, nprobe, ids, dists,
                                    cand.ctypes.data, surv.ctypes.data, threads)
        return ids, dists, cand, surv


# ---- the reference's on-disk E8Q index (E8AX), read as test input ----------

def parse_e8ax(path: str) -> dict:
    """Fields of a reference-written E8Q index file, in the order
    src/index/e8q_io.cpp:35-80 writes them, plus the per-vector codes decoded
    from its scan/refine arenas (include/e8qlib/index/e8q.hpp:189-266)."""
    with open(path, "rb") as f:
        buf = f.read()
    off = 0

    def take(fmt):
        nonlocal off
        v = struct.unpack_from(fmt, buf, off)
        off += struct.calcsize(fmt)
        return v

    (magic,) = take("<I")
    if magic != 0x58413845:
        raise ValueError("not an E8AX file")
    n, dim, nlist = take("<QQQ")
    (bits,) = take("<i")
    (rot_bytes,) = take("<Q")
    pd = padded_dim(dim)

    def arr(count, dt):
        nonlocal off
        a = np.frombuffer(buf, dtype=dt, count=count, offset=off).copy()
        off += a.nbytes
        return a

    out = dict(n=n, dim=dim, nlist=nlist, bits=bits, padded_dim=pd)
    out["ids"] = arr(n, np.uint32)
    out["signs"] = arr(rot_bytes, np.uint8)
    out["mean_rot"] = arr(pd, np.float32)
    out["centroid_rot"] = arr(nlist * pd, np.float32).reshape(nlist, pd)
    out["cn2"] = arr(nlist, np.float32)
    out["list_begin"] = arr(nlist + 1, np.uint64)
    arena_begin = arr(nlist + 1, np.uint64)
    arena = arr(int(arena_begin[-1]) + 64, np.uint8)
    ref_begin = arr(nlist + 1, np.uint64)
    ref_arena = arr(int(ref_begin[-1]) + 64, np.uint8)
    B = pd // 8
    c = bits - 1
    batch_bytes = (128 + B * 32 + 63) & ~63
    stride = B * c if bits >= 2 else 0
    ref_batch = (stride * 32 + 256 + 63) & ~63
    rowa = np.zeros((n, B), np.uint8)
    banks = []
    refine = np.zeros((n, max(stride, 1)), np.uint8)
    g1 = np.zeros(n, np.float32)
    h3 = np.zeros(n, np.float32)
    lb = out["list_begin"]
    for cl in range(nlist):
        cnt = int(lb[cl + 1] - lb[cl])
        for b0 in range(0, cnt, 32):
            m = min(32, cnt - b0)
            rec = int(arena_begin[cl]) + (b0 // 32) * batch_bytes + 128
            banks.append(arena[rec - 128:rec])
            plane = arena[rec:rec + B * 32].reshape(B, 32)
            rrec = int(ref_begin[cl]) + (b0 // 32) * ref_batch
            base = int(lb[cl]) + b0
            rowa[base:base + m] = plane[:, :m].T
            if stride:
                lanes = ref_arena[rrec:rrec + stride * 32].reshape(32, stride)
                refine[base:base + m] = lanes[:m]
            g1[base:base + m] = np.frombuffer(ref_arena, np.float32, 32, rrec + stride * 32)[:m]
            h3[base:base + m] = np.frombuffer(ref_arena, np.float32, 32,
                                              rrec + stride * 32 + 128)[:m]
    digits = np.zeros((n, B, 8), np.uint16)
    branch = np.zeros((n, B), np.uint8)
    L = lib()
    dbuf = np.zeros(8, np.uint16)
    brv = C.c_int(0)
    for i in range(n):
        for b in range(B):
            fld = np.ascontiguousarray(refine[i, b * c:(b + 1) * c] if stride else
                                       np.zeros(1, np.uint8))
            if fld.size == 0:
                fld = np.zeros(1, np.uint8)
            L.orc_decode_split(bits, int(rowa[i, b]), fld, dbuf, C.byref(brv))
            digits[i, b] = dbuf
            branch[i, b] = brv.value
    out.update(rowa=rowa, refine=refine[:, :stride], g1=g1, h3=h3, digits=digits,
               branch=branch, banks=np.array(banks, np.uint8).reshape(-1, 128))
    return out


# ---- ME8Q (mixed-rate) -----------------------------------------------------

ME8Q_DEFAULT_ROT_SEED = 0x5EED1234  # include/e8qlib/index/me8q.hpp:38 (BuildOptions::rot_seed)


def me8q_variance(base: np.ndarray) -> np.ndarray:
    """detail::DatasetVariance (src/index/me8q_common.cpp:11-35)."""
    base = np.ascontiguousarray(base, np.float32)
    n, dim = base.shape
    out = np.zeros(dim, np.float32)
    lib().orc_me8q_variance(base, dim, n, dim, out)
    return out


def me8q_allocate(var_padded: np.ndarray, avg_bits: float, max_bits: int = 13, extra_bits: float = 0.0):
    """SAQ DP plan over the padded dimension: [(len, bits), ...]."""
    v = np.ascontiguousarray(var_padded, np.float32)
    pd = v.shape[0]
    lens = (C.c_size_t * (pd // 64 + 1))()
    bits = (C.c_int * (pd // 64 + 1))()
    nr = lib().orc_me8q_allocate(v, pd, avg_bits, max_bits, extra_bits, lens, bits)
    return [(int(lens[i]), int(bits[i])) for i in range(nr)]


def parse_plan_spec(spec: str, pd: int):
    """detail::ParsePlanSpec (src/index/me8q_common.cpp:37-68)."""
    plan = []
    for tok in spec.split(","):
        if not tok:
            continue
        ln, b = tok.split(":")
        ln, b = int(ln), int(b)
        if ln <= 0 or ln % 64 or b < 0 or b > 13:
            raise ValueError("plan_spec: bad run " + tok)
        plan.append((ln, b))
    if sum(p[0] for p in plan) != pd:
        raise ValueError("plan_spec: runs do not cover the padded dims")
    return plan


class OracleMe8qIndex:
    """The restated ME8Q index as a Python object: the plain SearchIVF path
    (search) and the reference's production FastScan cascade
    (search_pruned)."""

    def __init__(self, data, centroids, cluster_ids, avg_bits=4.0, seed=0, variance=None, drop_energy=True,
                 plan_spec="", extra_budget_bits=0.0, max_bits=13, threads=8):
        data = np.ascontiguousarray(data, np.float32)
        centroids = np.ascontiguousarray(centroids, np.float32)
        cluster_ids = np.ascontiguousarray(cluster_ids, np.uint32)
        self.n, self.dim = data.shape
        self.nlist = centroids.shape[0]
        self.pd = padded_dim(self.dim)
        if plan_spec:
            self.plan = parse_plan_spec(plan_spec, self.pd)
        else:
            var = np.zeros(self.pd, np.float32)
            var[:self.dim] = me8q_variance(data) if variance is None else np.asarray(variance, np.float32)
            self.plan = me8q_allocate(var, avg_bits, max_bits, extra_budget_bits)
        rot_seed = seed if seed != 0 else ME8Q_DEFAULT_ROT_SEED
        lens = (C.c_size_t * len(self.plan))(*[p[0] for p in self.plan])
        bits = (C.c_int * len(self.plan))(*[p[1] for p in self.plan])
        self._p = lib().orc_me8q_build(data, centroids, cluster_ids, self.n, self.dim, self.nlist, lens, bits,
                                       len(self.plan), rot_seed, 1 if drop_energy else 0, threads)
        n, pd, nc = C.c_size_t(), C.c_size_t(), C.c_int()
        lib().orc_me8q_shape(self._p, C.byref(n), C.byref(pd), C.byref(nc))
        self.ncoded = nc.value
        self.ids = np.zeros(self.n, np.uint32)
        lib().orc_me8q_ids(self._p, self.ids)

    def __del__(self):
        if getattr(self, "_p", None):
            lib().orc_me8q_free(self._p)
            self._p = None

    def codes(self, pos):
        """(digits [pd] u16, branch [pd/8] u8, coef [ncoded], h2 [ncoded]) at cluster-major pos."""
        dg = np.zeros(self.pd, np.uint16)
        br = np.zeros(self.pd // 8, np.uint8)
        cf = np.zeros(max(self.ncoded, 1), np.float32)
        h2 = np.zeros(max(self.ncoded, 1), np.float32)
        lib().orc_me8q_codes(self._p, pos, dg, br, cf, h2)
        return dg, br, cf[:self.ncoded], h2[:self.ncoded]

    def estimate(self, q, gid):
        return lib().orc_me8q_estimate(self._p, np.ascontiguousarray(q, np.float32), gid)

    def search(self, queries, k, nprobe, threads=8):
        queries = np.ascontiguousarray(np.atleast_2d(queries), np.float32)
        nq = queries.shape[0]
        ids = np.zeros((nq, k), np.uint32)
        dists = np.zeros((nq, k), np.float32)
        lib().orc_me8q_search(self._p, queries, nq, k, nprobe, ids, dists, threads)
        return ids, dists

    def search_pruned(self, queries, k, nprobe, alpha=1.0, threads=8):
        """(ids, dists, candidates, survivors) of the production search; alpha
        is the build's prune_alpha (1 when not positive)."""
        queries = np.ascontiguousarray(np.atleast_2d(queries), np.float32)
        nq = queries.shape[0]
        ids = np.zeros((nq, k), np.uint32)
        dists = np.zeros((nq, k), np.float32)
        cand = np.zeros(nq, np.uint64)
        surv = np.zeros(nq, np.uint64)
        lib().orc_me8q_search_pruned(self._p, queries, nq, k, nprobe, alpha, ids, dists, cand, surv, threads)
        return ids, dists, cand, surv


def parse_me8q(path: str) -> dict:
    """Fields of a reference-written ME8Q index file (src/index/me8q_io.cpp:29-65,
    ME8QIDXX), with every row's segment codes unpacked (digits 0..6 at `bits`
    each, digit 7 without its parity bit at bits-1, branch in the block's top
    bit: src/quantization/me8q_codec.cpp:109-127) and its (coef, h2) pairs."""
    with open(path, "rb") as f:
        raw = f.read()
    off = [0]

    def take(fmt):
        v = struct.unpack_from(fmt, raw, off[0])
        off[0] += struct.calcsize(fmt)
        return v

    assert raw[:8] == b"ME8QIDXX"
    off[0] = 8
    n, dim, pd, nlist, bpv = take("<5Q")
    take("<f")
    take("<4i")
    (nplan,) = take("<Q")
    plan = []
    for _ in range(nplan):
        ln, b = take("<Qi")
        plan.append((ln, b))

    def arr(count, dt):
        a = np.frombuffer(raw, dt, count, off[0]).copy()
        off[0] += a.nbytes
        return a

    centroids = arr(nlist * pd, np.float32).reshape(nlist, pd)
    ids = arr(n, np.uint32)
    list_begin = arr(nlist + 1, np.uint64)
    byte_begin = arr(nlist + 1, np.uint64)
    codes = arr(int(byte_begin[-1]), np.uint8)
    coded = [(sum(p[0] for p in plan[:i]), p[0], p[1]) for i, p in enumerate(plan) if p[1] > 0]
    nseg = len(coded)
    stride = nseg * 8 + sum(ln // 8 * b for _, ln, b in coded)
    digits = np.zeros((n, pd), np.uint16)
    branch = np.zeros((n, pd // 8), np.uint8)
    coef = np.zeros((n, nseg), np.float32)
    h2 = np.zeros((n, nseg), np.float32)
    for c in range(nlist):
        for r in range(int(list_begin[c + 1] - list_begin[c])):
            pos = int(list_begin[c]) + r
            row = codes[int(byte_begin[c]) + r * stride:int(byte_begin[c]) + (r + 1) * stride]
            fac = row[:nseg * 8].view(np.float32)
            coef[pos] = fac[0::2]
            h2[pos] = fac[1::2]
            cur = nseg * 8
            for doff, ln, b in coded:
                for blk in range(ln // 8):
                    x = int.from_bytes(row[cur:cur + b].tobytes(), "little")
                    cur += b
                    par = 0
                    for i in range(7):
                        f = (x >> (b * i)) & ((1 << b) - 1)
                        digits[pos, doff + blk * 8 + i] = f
                        par ^= f & 1
                    f7 = (x >> (b * 7)) & ((1 << (b - 1)) - 1)
                    digits[pos, doff + blk * 8 + 7] = (f7 << 1) | par
                    branch[pos, doff // 8 + blk] = (x >> (8 * b - 1)) & 1
    return {"n": n, "dim": dim, "pd": pd, "nlist": nlist, "plan": plan, "centroids": centroids, "ids": ids,
            "list_begin": list_begin, "digits": digits, "branch": branch, "coef": coef, "h2": h2}
