"""ctypes access to the CPU oracle (phem_oracle.c) and to the reference's own
CPU code compiled from source into oracle/_ref (see oracle/Makefile).

TEST INFRASTRUCTURE ONLY.  Every function here is a checker or a CPU
baseline; nothing in the product calls it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF_DIR = HERE / "_ref"
FOREST_EMPTY = np.uint64(0x7FFFFFFF)

_u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")

_lib = None


def build(reference: str | None = None) -> None:
    """Compiles liboracle.so, and oracle/_ref when the reference tree exists."""
    subprocess.run(["make", "-s", "-C", str(HERE), "oracle"], check=True)
    ref = reference or os.environ.get("PHEM_REFERENCE", "/root/reference")
    if Path(ref, "CC", "host_spanning_tree.cu").exists():
        subprocess.run(["make", "-s", "-C", str(HERE), f"REF={ref}", "ref"], check=True)
        if (HERE.parent / "phem_graph_b200" / "libphem.so").exists():
            # the reference drivers linked with the compat layer (checks of the boundary)
            subprocess.run(["make", "-s", "-C", str(HERE), f"REF={ref}", "compat"], check=True)


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        path = HERE / "liboracle.so"
        if not path.exists():
            build()
        L = C.CDLL(str(path))
        L.oracle_cc_init.argtypes = [C.c_int32, _i32p, _u64p]
        L.oracle_cc_unite.argtypes = [_u64p, C.c_int64, C.c_int32, _i32p, _u64p]
        L.oracle_cc_unite.restype = C.c_int64
        L.oracle_cc_labels.argtypes = [C.c_int32, _i32p, _i32p]
        L.oracle_msf_kruskal.argtypes = [_u32p, C.c_uint64, C.c_uint32, _u8p, C.POINTER(C.c_uint64),
                                         C.POINTER(C.c_uint64)]
        L.oracle_msf_kruskal.restype = C.c_int
        L.oracle_msf_boruvka.argtypes = [_u32p, C.c_uint64, C.c_uint32, _u8p, C.POINTER(C.c_uint64),
                                         C.POINTER(C.c_uint64), _u64p, _u64p, C.c_int32,
                                         C.POINTER(C.c_int32)]
        L.oracle_msf_boruvka.restype = C.c_int
        L.oracle_csr_to_coo.argtypes = [_i64p, _u32p, C.c_int32, C.c_void_p]
        L.oracle_csr_to_coo.restype = C.c_int64
        _lib = L
    return _lib


# ---------------------------------------------------------------- CC

def cc_state(n: int):
    parent = np.empty(n, np.int32)
    forest = np.empty(n, np.uint64)
    lib().oracle_cc_init(n, parent, forest)
    return parent, forest


def cc_unite(edges: np.ndarray, n: int, parent: np.ndarray, forest: np.ndarray) -> int:
    edges = np.ascontiguousarray(edges, np.uint64)
    h = lib().oracle_cc_unite(edges, len(edges), n, parent, forest)
    if h < 0:
        raise ValueError("edge endpoint outside [0, n)")
    return int(h)


def cc_labels(parent: np.ndarray) -> np.ndarray:
    labels = np.empty(len(parent), np.int32)
    lib().oracle_cc_labels(len(parent), parent, labels)
    return labels


def cc_solve(edges: np.ndarray, n: int):
    """Sequential union-find in edge-index order: (labels, forest slots).
    The forest edge set is the canonical (index-order) spanning forest."""
    parent, forest = cc_state(n)
    cc_unite(edges, n, parent, forest)
    return cc_labels(parent), forest


def forest_set(forest: np.ndarray) -> np.ndarray:
    """Sorted packed edges of the filled forest slots."""
    f = np.asarray(forest, np.uint64)
    return np.sort(f[f != FOREST_EMPTY])


# ---------------------------------------------------------------- MSF

def _edges3(E) -> np.ndarray:
    E = np.ascontiguousarray(E, np.uint32)
    if E.ndim == 1:
        E = E.reshape(-1, 3)
    return E


def msf_kruskal(E, n: int):
    """(in_msf bool[m], count, total) of the unique MSF under (w, id)."""
    E = _edges3(E)
    m = len(E)
    flags = np.zeros(max(m, 1), np.uint8)
    cnt, tot = C.c_uint64(), C.c_uint64()
    if lib().oracle_msf_kruskal(E.reshape(-1), m, n, flags, C.byref(cnt), C.byref(tot)) != 0:
        raise ValueError("bad MSF input")
    return flags[:m].astype(bool), int(cnt.value), int(tot.value)


def msf_boruvka(E, n: int, max_rounds: int = 64):
    """Boruvka restatement: (in_msf, count, total, m_r, n_r)."""
    E = _edges3(E)
    m = len(E)
    flags = np.zeros(max(m, 1), np.uint8)
    cnt, tot, rounds = C.c_uint64(), C.c_uint64(), C.c_int32()
    m_r = np.zeros(max_rounds, np.uint64)
    n_r = np.zeros(max_rounds, np.uint64)
    rc = lib().oracle_msf_boruvka(E.reshape(-1), m, n, flags, C.byref(cnt), C.byref(tot), m_r, n_r, max_rounds,
                                  C.byref(rounds))
    if rc != 0:
        raise ValueError(f"boruvka restatement failed ({rc})")
    r = rounds.value
    return flags[:m].astype(bool), int(cnt.value), int(tot.value), m_r[:r].copy(), n_r[:r].copy()


def msf_chunked(E, n: int, chunk: int):
    """Chunked MSF of streamline_boruvka (MST/src/kernels.cu:849-1154): each
    chunk is solved together with the forest of the chunks before it
    (kernels.cu:942-997 appends the previous MSF to the next chunk).  The
    carried forest goes first, ascending by global edge id, so Kruskal's
    (w, position) order is the global (w, id) order.  Returns (in_msf, count,
    total) over the global ids."""
    E = _edges3(E)
    m = len(E)
    carried = np.zeros(0, np.int64)  # global ids of the forest so far
    count = total = 0
    for off in range(0, m, chunk):
        ids = np.concatenate([carried, np.arange(off, min(m, off + chunk), dtype=np.int64)])
        flags, count, total = msf_kruskal(E[ids], n)
        carried = ids[flags]
    in_msf = np.zeros(m, bool)
    in_msf[carried] = True
    return in_msf, count, total


def msf_bytes(m_r, n_r, n: int, components: int) -> int:
    """Algorithmic bytes of one MSF solve:
    sum_r (32 m_r + 16 m_{r+1}) + 16 sum_r n_r + 12 (n - c)."""
    m_r = [int(x) for x in m_r]
    total = 0
    for r, mr in enumerate(m_r):
        nxt = m_r[r + 1] if r + 1 < len(m_r) else 0
        total += 32 * mr + 16 * nxt
    total += 16 * sum(int(x) for x in n_r) + 12 * (n - components)
    return total


def csr_to_coo(offsets: np.ndarray, cols: np.ndarray, n: int) -> np.ndarray:
    offsets = np.ascontiguousarray(offsets, np.int64)
    cols = np.ascontiguousarray(cols, np.uint32)
    k = lib().oracle_csr_to_coo(offsets, cols, n, None)
    out = np.empty(k, np.uint64)
    lib().oracle_csr_to_coo(offsets, cols, n, out.ctypes.data_as(C.c_void_p))
    return out


# ---------------------------------------------------------------- reference code (oracle/_ref)

def ref_available() -> bool:
    return all((REF_DIR / f).exists() for f in ("libref_cc.so", "libref_mst.so", "libref_serial_mst.so"))


_ref = {}


def _ref_lib(name: str) -> C.CDLL:
    if name not in _ref:
        path = REF_DIR / name
        if not path.exists():
            raise FileNotFoundError(f"{path} missing: build it with `make -C oracle ref`")
        L = C.CDLL(str(path))
        if name == "libref_cc.so":
            L.ref_cc_create.argtypes = [C.c_int32]
            L.ref_cc_create.restype = C.c_void_p
            L.ref_cc_destroy.argtypes = [C.c_void_p]
            L.ref_cc_set_edges.argtypes = [C.c_void_p, _u64p, C.c_int64]
            L.ref_cc_run.argtypes = [C.c_void_p]
            L.ref_cc_run.restype = C.c_double
            L.ref_cc_reset.argtypes = [C.c_void_p]
            L.ref_cc_get.argtypes = [C.c_void_p, _i32p, _u64p]
            L.ref_cc_workers.restype = C.c_int32
        elif name == "libref_gpu_mst.so":
            L.ref_gpu_mst_create.argtypes = [_u32p, C.c_uint64, C.c_uint32]
            L.ref_gpu_mst_create.restype = C.c_void_p
            L.ref_gpu_mst_run.argtypes = [C.c_void_p, C.POINTER(C.c_float), C.POINTER(C.c_uint64),
                                          C.POINTER(C.c_uint64)]
            L.ref_gpu_mst_run.restype = C.c_int
            L.ref_gpu_mst_destroy.argtypes = [C.c_void_p]
        elif name == "libref_mst.so":
            L.ref_mst_create.argtypes = [_u32p, C.c_uint64]
            L.ref_mst_create.restype = C.c_void_p
            L.ref_mst_destroy.argtypes = [C.c_void_p]
            L.ref_mst_run.argtypes = [C.c_void_p, C.c_int32, C.POINTER(C.c_double)]
            L.ref_mst_run.restype = C.c_int
            L.ref_mst_count.argtypes = [C.c_void_p]
            L.ref_mst_count.restype = C.c_uint64
            L.ref_mst_ids.argtypes = [C.c_void_p, _u32p]
            L.ref_mst_workers.restype = C.c_int32
        else:
            L.ref_serial_mst.argtypes = [_u32p, C.c_uint64, _u32p]
            L.ref_serial_mst.restype = C.c_uint64
        _ref[name] = L
    return _ref[name]


class RefCC:
    """The reference's host_spanning_tree (CC/host_spanning_tree.cu:89) on one
    state of n vertices; the worker count comes from PARLAY_NUM_THREADS."""

    def __init__(self, n: int):
        self.L = _ref_lib("libref_cc.so")
        self.n = n
        self.h = self.L.ref_cc_create(n)

    def set_edges(self, edges: np.ndarray) -> None:
        edges = np.ascontiguousarray(edges, np.uint64)
        self.L.ref_cc_set_edges(self.h, edges, len(edges))

    def run(self) -> float:
        return float(self.L.ref_cc_run(self.h))

    def reset(self) -> None:
        self.L.ref_cc_reset(self.h)

    def state(self):
        parent = np.empty(self.n, np.int32)
        sptree = np.empty(self.n, np.uint64)
        self.L.ref_cc_get(self.h, parent, sptree)
        return parent, sptree

    def workers(self) -> int:
        return int(self.L.ref_cc_workers())

    def close(self) -> None:
        if self.h:
            self.L.ref_cc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class RefGpuMST:
    """The reference's GPU Boruvka device_boruvka (MST/src/kernels.cu:507-689),
    built for sm_100a: device copies of the edges made once, each run() times
    the call alone with CUDA events on fresh copies; returns (ms, count, total)."""

    def __init__(self, E, n: int):
        self.L = _ref_lib("libref_gpu_mst.so")
        E = _edges3(E)
        self.h = self.L.ref_gpu_mst_create(E.reshape(-1), len(E), n)
        if not self.h:
            raise RuntimeError("ref_gpu_mst_create failed (device memory)")

    def run(self):
        ms, cnt, tot = C.c_float(), C.c_uint64(), C.c_uint64()
        if self.L.ref_gpu_mst_run(self.h, C.byref(ms), C.byref(cnt), C.byref(tot)) != 0:
            raise RuntimeError("device_boruvka failed")
        return float(ms.value), int(cnt.value), int(tot.value)

    def close(self) -> None:
        if self.h:
            self.L.ref_gpu_mst_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def ref_gpu_available() -> bool:
    return (REF_DIR / "libref_gpu_mst.so").exists()


class RefPBBS:
    """The reference's PBBS mst() (MST/src/utils.cu:794-841) on one edge array."""

    def __init__(self, E):
        self.L = _ref_lib("libref_mst.so")
        self.E = _edges3(E)
        self.h = self.L.ref_mst_create(self.E.reshape(-1), len(self.E))

    def run(self, threads: int = 0) -> float:
        secs = C.c_double()
        rc = self.L.ref_mst_run(self.h, threads, C.byref(secs))
        if rc != 0:
            raise RuntimeError("PBBS mst() gave up (speculative_for: too many iterations)")
        return secs.value

    def ids(self) -> np.ndarray:
        k = int(self.L.ref_mst_count(self.h))
        out = np.empty(k, np.uint32)
        if k:
            self.L.ref_mst_ids(self.h, out)
        return out

    def workers(self) -> int:
        return int(self.L.ref_mst_workers())

    def close(self) -> None:
        if self.h:
            self.L.ref_mst_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def ref_pbbs_mst(E, threads: int = 0) -> np.ndarray:
    """MSF edge ids (ascending) from the reference's PBBS mst()."""
    r = RefPBBS(E)
    r.run(threads)
    ids = r.ids()
    r.close()
    return ids


def ref_serial_mst(E) -> np.ndarray:
    """MSF edge ids (ascending) from the reference's serial Kruskal."""
    E = _edges3(E)
    out = np.empty(max(len(E), 1), np.uint32)
    k = _ref_lib("libref_serial_mst.so").ref_serial_mst(E.reshape(-1), len(E), out)
    return np.sort(out[:k])


def ref_mtx_read(path, generate_weights: bool = False):
    """The MST driver's own MatrixMarket reader (getGraphInfo +
    mmapPopulateEdgeArray, MST/src/utils.cu:160-180, 896-1036) on `path`:
    ((m, 3) uint32 records, n), slots of missing lines left zero."""
    L = _ref_lib("libref_mst.so")
    L.ref_mtx_read.argtypes = [C.c_char_p, C.c_int, C.c_void_p, C.c_uint64, C.POINTER(C.c_uint32),
                               C.POINTER(C.c_uint64)]
    L.ref_mtx_read.restype = C.c_int
    p = str(path).encode()
    n, m = C.c_uint32(), C.c_uint64()
    if L.ref_mtx_read(p, int(generate_weights), None, 0, C.byref(n), C.byref(m)) != 0:
        raise ValueError("reference reader failed")
    out = np.zeros((max(m.value, 1), 3), np.uint32)
    if L.ref_mtx_read(p, int(generate_weights), out.ctypes.data, m.value, C.byref(n), C.byref(m)) != 0:
        raise ValueError("reference reader failed")
    return out[: m.value], n.value
