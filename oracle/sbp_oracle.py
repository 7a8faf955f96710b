"""ctypes binding of the CPU oracle (oracle/sbp_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, by the smoke check and by the CPU-baseline leg
of bench.py as the parity checker.  The product engine never imports this module.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD_DIR = os.path.join(HERE, "_build")
LIB_PATH = os.path.join(BUILD_DIR, "libsbp_oracle.so")
SRC_PATH = os.path.join(HERE, "sbp_oracle.c")

MH, GIBBS, HYBRID = 0, 1, 2
_i32p = ctypes.POINTER(ctypes.c_int32)
_u32p = ctypes.POINTER(ctypes.c_uint32)
_f64p = ctypes.POINTER(ctypes.c_double)
_i64p = ctypes.POINTER(ctypes.c_int64)


def build(force=False):
    """Compile the oracle with gcc into oracle/_build/ (no GPU needed)."""
    os.makedirs(BUILD_DIR, exist_ok=True)
    if not force and os.path.exists(LIB_PATH) and os.path.getmtime(LIB_PATH) >= os.path.getmtime(SRC_PATH):
        return LIB_PATH
    cmd = ["gcc", "-O2", "-fPIC", "-shared", "-fno-fast-math", "-o", LIB_PATH, SRC_PATH, "-lm"]
    subprocess.check_call(cmd)
    return LIB_PATH


class _Stats(ctypes.Structure):
    _fields_ = [("visits", ctypes.c_int64), ("proposals_moved", ctypes.c_int64),
                ("accepted", ctypes.c_int64), ("sweeps", ctypes.c_int), ("mdl", ctypes.c_double),
                ("rng_error", ctypes.c_int)]


class _MergeStats(ctypes.Structure):
    _fields_ = [("proposals", ctypes.c_int64), ("avoided", ctypes.c_int64)]


class _Options(ctypes.Structure):
    _fields_ = [("algo", ctypes.c_int), ("batches", ctypes.c_int), ("approximate", ctypes.c_int),
                ("asynciterations", ctypes.c_int), ("seed", ctypes.c_uint64)]


class _RunStats(ctypes.Structure):
    _fields_ = [("mdl", ctypes.c_double), ("num_blocks", ctypes.c_int), ("outer_iterations", ctypes.c_int),
                ("mcmc_sweeps", ctypes.c_int), ("visits", ctypes.c_int64), ("accepted", ctypes.c_int64)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(LIB_PATH)
        vp = ctypes.c_void_p
        L.sbpo_graph_create.restype = vp
        L.sbpo_graph_create.argtypes = [ctypes.c_int, ctypes.c_int64, _i32p, _i32p]
        L.sbpo_graph_destroy.argtypes = [vp]
        L.sbpo_graph_num_edges.restype = ctypes.c_int
        L.sbpo_graph_num_edges.argtypes = [vp]
        L.sbpo_graph_num_high.restype = ctypes.c_int
        L.sbpo_graph_num_high.argtypes = [vp]
        L.sbpo_graph_get_split.argtypes = [vp, _i32p, _i32p]
        L.sbpo_graph_set_split.restype = ctypes.c_int
        L.sbpo_graph_set_split.argtypes = [vp, ctypes.c_int, _i32p, ctypes.c_int, _i32p]
        L.sbpo_bm_create.restype = vp
        L.sbpo_bm_create.argtypes = [vp, ctypes.c_int, _i32p]
        L.sbpo_bm_copy.restype = vp
        L.sbpo_bm_copy.argtypes = [vp]
        L.sbpo_bm_destroy.argtypes = [vp]
        L.sbpo_bm_num_blocks.restype = ctypes.c_int
        L.sbpo_bm_num_blocks.argtypes = [vp]
        L.sbpo_bm_get_assignment.argtypes = [vp, _i32p]
        L.sbpo_bm_get_matrix.argtypes = [vp, _i32p]
        L.sbpo_bm_get_degrees.argtypes = [vp, _i32p, _i32p, _i32p]
        L.sbpo_bm_overall_entropy.restype = ctypes.c_float
        L.sbpo_bm_overall_entropy.argtypes = [vp]
        L.sbpo_bm_set_num_blocks_to_merge.argtypes = [vp, ctypes.c_int]
        L.sbpo_mdl.restype = ctypes.c_double
        L.sbpo_mdl.argtypes = [vp, ctypes.c_int, ctypes.c_int]
        L.sbpo_null_mdl_v1.restype = ctypes.c_double
        L.sbpo_null_mdl_v1.argtypes = [ctypes.c_long]
        L.sbpo_null_mdl_v2.restype = ctypes.c_double
        L.sbpo_null_mdl_v2.argtypes = [ctypes.c_long, ctypes.c_long]
        L.sbpo_philox.argtypes = [_u32p, _u32p, _u32p]
        L.sbpo_u53.restype = ctypes.c_double
        L.sbpo_u53.argtypes = [ctypes.c_uint32, ctypes.c_uint32]
        L.sbpo_eval_vertex.restype = ctypes.c_int
        L.sbpo_eval_vertex.argtypes = [vp, vp, ctypes.c_int, _u32p, _i32p, _f64p, _f64p, _i32p]
        L.sbpo_delta_mdl_move.restype = ctypes.c_double
        L.sbpo_delta_mdl_move.argtypes = [vp, vp, ctypes.c_int, ctypes.c_int, _f64p]
        L.sbpo_move_vertex.argtypes = [vp, vp, ctypes.c_int, ctypes.c_int]
        L.sbpo_finetune.restype = ctypes.c_int
        L.sbpo_finetune.argtypes = [vp, vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_uint64,
                                    ctypes.c_uint32, _u32p, ctypes.c_int64, ctypes.c_int, ctypes.POINTER(_Stats)]
        L.sbpo_merge_delta_mdl.restype = ctypes.c_double
        L.sbpo_merge_delta_mdl.argtypes = [vp, ctypes.c_int, ctypes.c_int]
        L.sbpo_merge_blocks.restype = ctypes.c_int
        L.sbpo_merge_blocks.argtypes = [vp, vp, ctypes.c_int, ctypes.c_uint64, ctypes.c_uint32, _u32p,
                                        ctypes.c_int64, _i32p, _f64p, ctypes.POINTER(_MergeStats)]
        L.sbpo_finetune_moves.restype = ctypes.c_int
        L.sbpo_finetune_moves.argtypes = [vp, vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, _u32p, ctypes.c_int64,
                                          ctypes.c_int, ctypes.POINTER(_Stats)]
        L.sbpo_merge_blocks_moves.restype = ctypes.c_int
        L.sbpo_merge_blocks_moves.argtypes = [vp, vp, ctypes.c_int, _u32p, ctypes.c_int64, _i32p, _f64p,
                                              ctypes.POINTER(_MergeStats)]
        L.sbpo_sbp_moves.restype = ctypes.c_int
        L.sbpo_sbp_moves.argtypes = [vp, ctypes.POINTER(_Options), ctypes.c_int,
                                     ctypes.POINTER(ctypes.POINTER(ctypes.c_uint32)), _i64p, ctypes.c_int, _i32p,
                                     _i32p, ctypes.POINTER(_RunStats)]
        L.sbpo_sbp.restype = ctypes.c_int
        L.sbpo_sbp.argtypes = [vp, ctypes.POINTER(_Options), _i32p, ctypes.POINTER(_RunStats)]
        L.sbpo_nmi.restype = ctypes.c_double
        L.sbpo_nmi.argtypes = [ctypes.c_int, _i32p, _i32p]
        _lib = L
    return _lib


def _p(a, t=_i32p):
    return a.ctypes.data_as(t)


def philox(ctr, key):
    c = np.ascontiguousarray(ctr, dtype=np.uint32)
    k = np.ascontiguousarray(key, dtype=np.uint32)
    out = np.zeros(4, dtype=np.uint32)
    lib().sbpo_philox(_p(c, _u32p), _p(k, _u32p), _p(out, _u32p))
    return out


class Graph:
    """Directed graph with the reference's de-duplicated adjacency lists (src/graph.cpp)."""

    def __init__(self, V, src, dst):
        self.src = np.ascontiguousarray(src, dtype=np.int32)
        self.dst = np.ascontiguousarray(dst, dtype=np.int32)
        self.V = int(V)
        self.h = lib().sbpo_graph_create(self.V, len(self.src), _p(self.src), _p(self.dst))
        if not self.h:
            raise ValueError("invalid edge list")
        self.E = lib().sbpo_graph_num_edges(self.h)

    def split(self):
        nh = lib().sbpo_graph_num_high(self.h)
        hi = np.zeros(nh, np.int32)
        lo = np.zeros(self.V - nh, np.int32)
        lib().sbpo_graph_get_split(self.h, _p(hi), _p(lo))
        return hi, lo

    def set_split(self, high, low):
        hi = np.ascontiguousarray(high, np.int32)
        lo = np.ascontiguousarray(low, np.int32)
        if lib().sbpo_graph_set_split(self.h, len(hi), _p(hi), len(lo), _p(lo)) != 0:
            raise ValueError("split does not cover V")

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.sbpo_graph_destroy(self.h)
            self.h = None


class Blockmodel:
    """Dense-matrix blockmodel with the reference's state (include/blockmodel/blockmodel.hpp)."""

    def __init__(self, graph, B=None, assignment=None, _handle=None):
        self.graph = graph
        if _handle is not None:
            self.h = _handle
            return
        a = np.ascontiguousarray(assignment, dtype=np.int32)
        self.h = lib().sbpo_bm_create(graph.h, int(B), _p(a))
        if not self.h:
            raise ValueError("invalid assignment")

    def copy(self):
        return Blockmodel(self.graph, _handle=lib().sbpo_bm_copy(self.h))

    @property
    def B(self):
        return lib().sbpo_bm_num_blocks(self.h)

    def assignment(self):
        out = np.zeros(self.graph.V, np.int32)
        lib().sbpo_bm_get_assignment(self.h, _p(out))
        return out

    def matrix(self):
        B = self.B
        out = np.zeros(B * B, np.int32)
        lib().sbpo_bm_get_matrix(self.h, _p(out))
        return out.reshape(B, B)

    def degrees(self):
        B = self.B
        do, di, d = (np.zeros(B, np.int32) for _ in range(3))
        lib().sbpo_bm_get_degrees(self.h, _p(do), _p(di), _p(d))
        return do, di, d

    def overall_entropy(self):
        return lib().sbpo_bm_overall_entropy(self.h)

    def set_num_blocks_to_merge(self, n):
        lib().sbpo_bm_set_num_blocks_to_merge(self.h, int(n))

    def mdl(self):
        return lib().sbpo_mdl(self.h, self.graph.V, self.graph.E)

    def delta_mdl_move(self, v, s):
        H = ctypes.c_double(0)
        dS = lib().sbpo_delta_mdl_move(self.h, self.graph.h, int(v), int(s), ctypes.byref(H))
        return dS, H.value

    def merge_delta_mdl(self, r, s):
        return lib().sbpo_merge_delta_mdl(self.h, int(r), int(s))

    def move_vertex(self, v, s):
        lib().sbpo_move_vertex(self.h, self.graph.h, int(v), int(s))

    def eval_vertex(self, v, record):
        x = np.ascontiguousarray(record, np.uint32)
        s = ctypes.c_int32(0)
        dS = ctypes.c_double(0)
        H = ctypes.c_double(0)
        acc = ctypes.c_int32(0)
        moved = lib().sbpo_eval_vertex(self.h, self.graph.h, int(v), _p(x, _u32p), ctypes.byref(s),
                                       ctypes.byref(dS), ctypes.byref(H), ctypes.byref(acc))
        return dict(s=s.value, moved=bool(moved), dS=dS.value, H=H.value, accepted=bool(acc.value))

    def finetune(self, algo, batches=10, bracket=False, seed=0, call=0, replay=None, max_sweeps=0):
        st = _Stats()
        if replay is not None:
            rp = np.ascontiguousarray(replay, np.uint32).reshape(-1)
            rc = lib().sbpo_finetune(self.h, self.graph.h, algo, batches, int(bracket), seed, call,
                                     _p(rp, _u32p), len(rp) // 4, max_sweeps, ctypes.byref(st))
        else:
            rc = lib().sbpo_finetune(self.h, self.graph.h, algo, batches, int(bracket), seed, call,
                                     None, 0, max_sweeps, ctypes.byref(st))
        if rc != 0:
            raise RuntimeError("oracle finetune failed (replay buffer too short?)")
        return dict(visits=st.visits, proposals_moved=st.proposals_moved, accepted=st.accepted,
                    sweeps=st.sweeps, mdl=st.mdl)

    def merge_blocks(self, approximate=True, seed=0, call=0, replay=None):
        B = self.B
        best = np.zeros(B, np.int32)
        dS = np.zeros(B, np.float64)
        ms = _MergeStats()
        if replay is not None:
            rp = np.ascontiguousarray(replay, np.uint32).reshape(-1)
            rc = lib().sbpo_merge_blocks(self.h, self.graph.h, int(approximate), seed, call, _p(rp, _u32p),
                                         len(rp) // 4, _p(best), _p(dS, _f64p), ctypes.byref(ms))
        else:
            rc = lib().sbpo_merge_blocks(self.h, self.graph.h, int(approximate), seed, call, None, 0,
                                         _p(best), _p(dS, _f64p), ctypes.byref(ms))
        if rc != 0:
            raise RuntimeError("oracle merge failed")
        return dict(best=best, dS=dS, proposals=ms.proposals, avoided=ms.avoided)

    def finetune_replayed(self, algo, proposal, uniform, batches=10, bracket=False, max_sweeps=0):
        """The finetune driven by a recorded proposal stream: proposal[t*V + v] and uniform[t*V + v]
        are the proposed block and the accept uniform of vertex v's visit in sweep t (2.0 where
        the stream has none: never accepts)."""
        rp = move_records(proposal, uniform)
        st = _Stats()
        rc = lib().sbpo_finetune_moves(self.h, self.graph.h, algo, batches, int(bracket), _p(rp, _u32p),
                                       len(rp) // 4, max_sweeps, ctypes.byref(st))
        if rc != 0:
            raise RuntimeError("oracle finetune failed (a visit with no recorded proposal, or one out of range)")
        return dict(visits=st.visits, proposals_moved=st.proposals_moved, accepted=st.accepted,
                    sweeps=st.sweeps, mdl=st.mdl)

    def merge_blocks_replayed(self, proposal, approximate=True):
        """The merge step with proposal[r*10 + i] as proposal i of block r."""
        B = self.B
        best = np.zeros(B, np.int32)
        dS = np.zeros(B, np.float64)
        ms = _MergeStats()
        rp = move_records(proposal, None)
        rc = lib().sbpo_merge_blocks_moves(self.h, self.graph.h, int(approximate), _p(rp, _u32p), len(rp) // 4,
                                           _p(best), _p(dS, _f64p), ctypes.byref(ms))
        if rc != 0:
            raise RuntimeError("oracle merge failed (a proposal missing or out of range)")
        return dict(best=best, dS=dS, proposals=ms.proposals, avoided=ms.avoided)

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.sbpo_bm_destroy(self.h)
            self.h = None


def move_records(proposal, uniform):
    """4-word records (s, 0, u_hi, u_lo) of a recorded proposal stream: the proposed block and
    the bits of the accept uniform (2.0, which never accepts, where there is none)."""
    prop = np.ascontiguousarray(proposal, np.int32)
    uni = np.full(len(prop), 2.0) if uniform is None else np.ascontiguousarray(uniform, np.float64)
    if uni.shape != prop.shape:
        raise ValueError("proposal and uniform streams differ in length")
    bits = uni.view(np.uint64)
    rec = np.zeros((len(prop), 4), np.uint32)
    rec[:, 0] = prop.view(np.uint32)
    rec[:, 2] = (bits >> np.uint64(32)).astype(np.uint32)
    rec[:, 3] = (bits & np.uint64(0xFFFFFFFF)).astype(np.uint32)
    return rec.reshape(-1)


def null_mdl_v1(E):
    return lib().sbpo_null_mdl_v1(int(E))


def null_mdl_v2(V, E):
    return lib().sbpo_null_mdl_v2(int(V), int(E))


def nmi(a, b):
    a = np.ascontiguousarray(a, np.int32)
    b = np.ascontiguousarray(b, np.int32)
    return lib().sbpo_nmi(len(a), _p(a), _p(b))


def sbp(graph, algo=GIBBS, batches=10, approximate=True, asynciterations=2**31 - 1, seed=0):
    opt = _Options(algo, batches, int(approximate), asynciterations, seed)
    rs = _RunStats()
    out = np.zeros(graph.V, np.int32)
    if lib().sbpo_sbp(graph.h, ctypes.byref(opt), _p(out), ctypes.byref(rs)) != 0:
        raise RuntimeError("oracle sbp failed")
    return out, dict(mdl=rs.mdl, num_blocks=rs.num_blocks, outer_iterations=rs.outer_iterations,
                     mcmc_sweeps=rs.mcmc_sweeps, visits=rs.visits, accepted=rs.accepted)


def sbp_replayed(graph, streams, algo=GIBBS, batches=10, approximate=True, max_sweeps=0):
    """sbp with every merge and finetune call driven by a recorded stream, in call order:
    streams[k] = (proposal, uniform) of call k (uniform None for a merge call).  Returns
    (assignment, stats, block count after every call)."""
    recs = [move_records(p, u) for p, u in streams]
    ptrs = (ctypes.POINTER(ctypes.c_uint32) * max(1, len(recs)))(*[_p(r, _u32p) for r in recs])
    counts = np.array([len(r) // 4 for r in recs] or [0], np.int64)
    blocks = np.zeros(max(1, len(recs)), np.int32)
    opt = _Options(algo, batches, int(approximate), 2**31 - 1, 0)
    rs = _RunStats()
    out = np.zeros(graph.V, np.int32)
    made = lib().sbpo_sbp_moves(graph.h, ctypes.byref(opt), len(recs), ptrs, counts.ctypes.data_as(_i64p),
                                int(max_sweeps), _p(out), _p(blocks), ctypes.byref(rs))
    if made < 0:
        raise RuntimeError("oracle sbp replay failed (the partition needed more calls than were recorded, or a "
                           "stream lacked a proposal)")
    return out, dict(mdl=rs.mdl, num_blocks=rs.num_blocks, outer_iterations=rs.outer_iterations,
                     mcmc_sweeps=rs.mcmc_sweeps, visits=rs.visits, accepted=rs.accepted), blocks[:made].copy()


# ------------------------------------------------------------------------------------------
# Partition quality (src/evaluate.cpp:7-178), restated in numpy; the block <-> community
# matching of the accuracy is scipy's linear_sum_assignment (the reference uses the Hungarian
# method of extern/hungarian).
# ------------------------------------------------------------------------------------------
def contingency(alg, truth):
    """Table with rows = algorithm blocks, columns = true communities numbered in order of first
    appearance (evaluate::hungarian's translator); vertices with truth < 0 are not counted."""
    alg = np.asarray(alg, np.int64)
    truth = np.asarray(truth, np.int64)
    known = truth >= 0
    _, first = np.unique(truth[known], return_index=True)
    order = np.unique(truth[known])[np.argsort(first)]
    col = {int(t): i for i, t in enumerate(order)}
    cols = np.array([col[int(t)] for t in truth[known]], np.int64)
    table = np.zeros((int(alg.max()) + 1, len(order)), np.int64)
    np.add.at(table, (alg[known], cols), 1)
    return table


def contingency_metrics(table, num_vertices):
    """calculate_f1_score and calculate_nmi (src/evaluate.cpp:7-96) with exact integer pair counts."""
    from scipy.optimize import linear_sum_assignment
    t = np.asarray(table, np.int64)
    N = float(num_vertices)
    rows, cols = t.sum(1).astype(np.float64), t.sum(0).astype(np.float64)
    cell_pairs = float((t * (t - 1)).sum()) / 2.0
    row_pairs = float((rows * (rows - 1)).sum()) / 2.0
    col_pairs = float((cols * (cols - 1)).sum()) / 2.0
    agree_diff = (N * N + float((t * t).sum()) - float((rows ** 2).sum() + (cols ** 2).sum())) / 2.0
    recall, precision = cell_pairs / row_pairs, cell_pairs / col_pairs
    p = t / N
    pr, pc = rows / N, cols / N
    h = lambda q: -float(np.sum(q[q > 0] * np.log(q[q > 0])))
    nz = p > 0
    mi = float(np.sum(p[nz] * np.log(p[nz] / np.outer(pr, pc)[nz])))
    ri, ci = linear_sum_assignment(t, maximize=True)
    return {"f1": 2 * precision * recall / (precision + recall), "precision": precision, "recall": recall,
            "rand_index": (cell_pairs + agree_diff) / (N * (N - 1) / 2.0), "nmi": mi / np.sqrt(h(pr) * h(pc)),
            "accuracy": float(t[ri, ci].sum()) / N}


def evaluate(alg, truth):
    t = contingency(alg, truth)
    return dict(contingency_metrics(t, len(alg)), table=t)
