"""ctypes front end of the CPU oracle (TEST INFRASTRUCTURE ONLY).

The oracle (oracle/oracle.c) is a plain-C restatement of the reference's plan
compiler (src/pattern.h) and DFS count semantics (src/gpu_match.cu,
cu_test.cu:100-105).  Only tests/, the smoke check and bench.py's CPU baseline
use this module, as the checker or the timed CPU baseline; the product never
imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
PAT = 7


class _Plan(C.Structure):
    _fields_ = [
        ("k", C.c_int),
        ("labeled", C.c_int),
        ("adj", (C.c_int * PAT) * PAT),
        ("vlabel", C.c_int * PAT),
        ("degree", C.c_int * PAT),
        ("nbn", C.c_int * PAT),
        ("bn", (C.c_int * PAT) * PAT),
        ("shared_lvl", C.c_int * PAT),
        ("nbn_sh", C.c_int * PAT),
        ("bn_sh", (C.c_int * PAT) * PAT),
        ("cond_op", (C.c_int * PAT) * PAT),
        ("ncond_pairs", C.c_int),
        ("cond_a", C.c_int * 64),
        ("cond_b", C.c_int * 64),
        ("orient", C.c_int),
        ("multiplicity", C.c_longlong),
        ("aut_size", C.c_int),
    ]


class _Graph(C.Structure):
    _fields_ = [
        ("n", C.c_int64),
        ("nedges", C.c_int64),
        ("rowptr", C.POINTER(C.c_int64)),
        ("colidx", C.POINTER(C.c_int32)),
        ("label", C.POINTER(C.c_int32)),
        ("max_degree", C.c_int32),
    ]


_lib = None


def build():
    subprocess.run(["make", "-s", "-C", _HERE, "oracle"], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        L.orc_last_error.restype = C.c_char_p
        L.orc_plan_from_text.argtypes = [C.c_char_p, C.c_int, C.POINTER(_Plan)]
        L.orc_graph_wrap.argtypes = [C.c_int64, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p,
                                     C.POINTER(_Graph)]
        L.orc_count.argtypes = [C.POINTER(_Graph), C.POINTER(_Plan), C.c_int, C.c_int64, C.c_int64,
                                C.POINTER(C.c_ulonglong), C.POINTER(C.c_ulonglong)]
        L.orc_bruteforce.argtypes = [C.POINTER(_Graph), C.POINTER(_Plan), C.POINTER(C.c_ulonglong)]
        _lib = L
    return _lib


class OracleError(RuntimeError):
    pass


class Plan:
    """Compiled plan of one .g pattern (reference semantics)."""

    def __init__(self, text: str, labeled: bool):
        self._p = _Plan()
        rc = lib().orc_plan_from_text(text.encode(), int(labeled), C.byref(self._p))
        if rc:
            raise OracleError(lib().orc_last_error().decode())

    def as_dict(self) -> dict:
        p = self._p
        k = p.k
        return {
            "k": k,
            "labeled": p.labeled,
            "multiplicity": p.multiplicity,
            "orient": p.orient,
            "degree": list(p.degree[:k]),
            "vertex_labels": list(p.vlabel[:k]),
            "num_BN": [0] + [p.nbn[i] for i in range(1, k)],
            "backward_neighbors": [[]] + [list(p.bn[i][: p.nbn[i]]) for i in range(1, k)],
            "shared_lvl": list(p.shared_lvl[:k]),
            "backward_neighbors_sh": [
                list(p.bn_sh[i][: p.nbn_sh[i]]) if p.shared_lvl[i] != -1 else [] for i in range(k)
            ],
            "condition_cnt": list(range(k)),
            "condition_order": [[[p.cond_op[i][j], j] for j in range(i)] for i in range(k)],
            "conditions": [[p.cond_a[c], p.cond_b[c]] for c in range(p.ncond_pairs)],
        }


class Graph:
    """CSR graph held in numpy arrays (int64 rowptr, int32 colidx, int32 labels)."""

    def __init__(self, rowptr, colidx, labels=None):
        self.rowptr = np.ascontiguousarray(rowptr, dtype=np.int64)
        self.colidx = np.ascontiguousarray(colidx, dtype=np.int32)
        self.labels = None if labels is None else np.ascontiguousarray(labels, dtype=np.int32)
        self._g = _Graph()
        lib().orc_graph_wrap(
            len(self.rowptr) - 1, len(self.colidx), self.rowptr.ctypes.data,
            self.colidx.ctypes.data, None if self.labels is None else self.labels.ctypes.data,
            C.byref(self._g))


def count(graph: Graph, plan: Plan, threads: int = 0, edge_begin: int = 0, edge_end: int = -1,
          with_bytes: bool = False):
    c = C.c_ulonglong()
    b = C.c_ulonglong()
    rc = lib().orc_count(C.byref(graph._g), C.byref(plan._p), threads, edge_begin, edge_end,
                         C.byref(c), C.byref(b))
    if rc:
        raise OracleError(lib().orc_last_error().decode())
    return (c.value, b.value) if with_bytes else c.value


def bruteforce(graph: Graph, plan: Plan) -> int:
    c = C.c_ulonglong()
    rc = lib().orc_bruteforce(C.byref(graph._g), C.byref(plan._p), C.byref(c))
    if rc:
        raise OracleError(lib().orc_last_error().decode())
    return c.value
