"""Python binding of libsbp_b200.so (the C ABI in include/sbp_b200.h).

Mirrors the reference's C++ API (vtsynergy/Hybrid-Stochastic-Block-Partitioning):
  Graph                      include/graph.hpp:15-113
  Blockmodel                 include/blockmodel/blockmodel.hpp:45-184
  entropy.mdl                src/entropy.cpp:584-589
  block_merge.merge_blocks   src/block_merge.cpp:278-311
  finetune.metropolis_hastings / asynchronous_gibbs / hybrid_mcmc   src/finetune.cpp
  sbp.stochastic_block_partition                                    src/sbp.cpp:61-98
All compute runs on the GPU; without the built library or a CUDA device every call raises.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsbp_b200.so")

METROPOLIS_HASTINGS, ASYNC_GIBBS, HYBRID_MCMC = 0, 1, 2
ALGORITHMS = {"metropolis_hastings": METROPOLIS_HASTINGS, "async_gibbs": ASYNC_GIBBS, "hybrid_mcmc": HYBRID_MCMC}

STATUS = {0: "SBP_OK", 1: "SBP_ERR_INVALID_ARGUMENT", 2: "SBP_ERR_CUDA", 3: "SBP_ERR_UNSUPPORTED",
          4: "SBP_ERR_REPLAY", 5: "SBP_ERR_DEVICE", 6: "SBP_ERR_OUT_OF_MEMORY"}

EXPORTED = [
    "sbp_last_error", "sbp_device_count", "sbp_set_option", "sbp_get_stream", "sbp_release_cached_memory",
    "sbp_profile_enable", "sbp_profile_read",
    "sbp_graph_create", "sbp_graph_destroy", "sbp_graph_num_edges",
    "sbp_graph_get_split", "sbp_graph_set_split", "sbp_blockmodel_create", "sbp_blockmodel_copy",
    "sbp_blockmodel_destroy", "sbp_blockmodel_num_blocks", "sbp_blockmodel_set_num_blocks_to_merge",
    "sbp_blockmodel_overall_entropy", "sbp_get_assignment", "sbp_get_block_matrix", "sbp_get_degrees", "sbp_mdl",
    "sbp_evaluate_vertices", "sbp_move_vertex", "sbp_finetune", "sbp_merge_blocks", "sbp_partition",
    "sbp_mlp_create", "sbp_mlp_destroy", "sbp_mlp_get_params", "sbp_mlp_set_params", "sbp_mlp_forward",
    "sbp_mlp_gradients", "sbp_mlp_train", "sbp_dataset_create", "sbp_dataset_destroy", "sbp_dataset_size",
    "sbp_dataset_append", "sbp_dataset_read", "sbp_vertex_features", "sbp_learned_evaluate", "sbp_learned_q",
    "sbp_collect_moves", "sbp_finetune_learned", "sbp_partition_learned", "sbp_partition_batched",
    "sbp_batched_reset_tuning", "sbp_mdl_device_noalloc", "sbp_finetune_replayed", "sbp_merge_blocks_replayed",
    "sbp_partition_replayed", "sbp_set_degrees", "sbp_mdl_of_cells", "sbp_contingency_metrics",
    "sbp_evaluate_blockmodel", "sbp_get_intermediates", "sbp_clear_intermediates",
]

MLP_FEATURES, MLP_OUTPUTS, MLP_SLOTS, MLP_ESCAPE, MLP_PARAMS = 64, 16, 14, 14, 26896


class SbpError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{STATUS.get(code, code)}: {msg}")
        self.code = code


class Replay(ctypes.Structure):
    _fields_ = [("words", ctypes.POINTER(ctypes.c_uint32)), ("records", ctypes.c_int64)]


class MoveReplay(ctypes.Structure):
    _fields_ = [("proposal", ctypes.POINTER(ctypes.c_int32)), ("uniform", ctypes.POINTER(ctypes.c_double)),
                ("records", ctypes.c_int64)]


class Evaluation(ctypes.Structure):
    _fields_ = [("f1_score", ctypes.c_double), ("nmi", ctypes.c_double), ("accuracy", ctypes.c_double),
                ("rand_index", ctypes.c_double), ("precision", ctypes.c_double), ("recall", ctypes.c_double),
                ("true_mdl", ctypes.c_double), ("counted_vertices", ctypes.c_int64), ("num_blocks", ctypes.c_int32),
                ("true_num_blocks", ctypes.c_int32)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class Intermediate(ctypes.Structure):
    _fields_ = [("iteration", ctypes.c_float), ("num_blocks", ctypes.c_int32), ("mdl", ctypes.c_double),
                ("normalized_mdl_v1", ctypes.c_double), ("normalized_mdl_v2", ctypes.c_double),
                ("modularity", ctypes.c_double), ("interblock_edges", ctypes.c_double),
                ("block_size_variation", ctypes.c_double), ("mcmc_iterations", ctypes.c_int32), ("_pad", ctypes.c_int32),
                ("mcmc_time", ctypes.c_double), ("visits", ctypes.c_int64), ("seconds", ctypes.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if not k.startswith("_")}


class Stats(ctypes.Structure):
    _fields_ = [("visits", ctypes.c_int64), ("proposals_moved", ctypes.c_int64), ("accepted", ctypes.c_int64),
                ("sweeps", ctypes.c_int32), ("outer_iterations", ctypes.c_int32), ("num_blocks", ctypes.c_int32),
                ("overflow_rebuilds", ctypes.c_int32), ("mdl", ctypes.c_double), ("mcmc_seconds", ctypes.c_double),
                ("merge_seconds", ctypes.c_double), ("merge_proposals", ctypes.c_int64),
                ("merge_avoided", ctypes.c_int64), ("total_seconds", ctypes.c_double),
                ("learned_sweeps", ctypes.c_int32), ("_reserved", ctypes.c_int32)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if not k.startswith("_")}


class Profile(ctypes.Structure):
    _fields_ = [("launches", ctypes.c_int64), ("eval_launches", ctypes.c_int64), ("eval_visits", ctypes.c_int64),
                ("eval_ms", ctypes.c_double), ("eval_bytes", ctypes.c_double), ("h2d_bytes", ctypes.c_int64),
                ("d2h_bytes", ctypes.c_int64)]


class Options(ctypes.Structure):
    _fields_ = [("algorithm", ctypes.c_int32), ("batches", ctypes.c_int32), ("approximate", ctypes.c_int32),
                ("asynciterations", ctypes.c_int32), ("seed", ctypes.c_uint64)]


class FinetuneOptions(ctypes.Structure):
    _fields_ = [("batches", ctypes.c_int32), ("bracket_established", ctypes.c_int32),
                ("max_sweeps", ctypes.c_int32), ("call", ctypes.c_uint32), ("seed", ctypes.c_uint64)]


class MergeOptions(ctypes.Structure):
    _fields_ = [("approximate", ctypes.c_int32), ("call", ctypes.c_uint32), ("seed", ctypes.c_uint64)]


class TrainOptions(ctypes.Structure):
    _fields_ = [("epochs", ctypes.c_int32), ("batch", ctypes.c_int32), ("lr", ctypes.c_float),
                ("_pad", ctypes.c_int32), ("seed", ctypes.c_uint64)]


class TrainStats(ctypes.Structure):
    _fields_ = [("steps", ctypes.c_int64), ("first_loss", ctypes.c_double), ("last_loss", ctypes.c_double),
                ("seconds", ctypes.c_double)]


class LearnedOptions(ctypes.Structure):
    _fields_ = [("epsilon", ctypes.c_float), ("fallback_acceptance", ctypes.c_float), ("stop_rule", ctypes.c_int32),
                ("_pad", ctypes.c_int32)]


class BatchInfo(ctypes.Structure):
    _fields_ = [("rounds", ctypes.c_int32), ("batched_finetunes", ctypes.c_int32),
                ("fallback_finetunes", ctypes.c_int32), ("sweep_launches", ctypes.c_int32), ("chunk", ctypes.c_int32),
                ("ctas_per_sm", ctypes.c_int32), ("tuned", ctypes.c_int32), ("candidates", ctypes.c_int32),
                ("candidate_ms", ctypes.c_double * 8), ("sweep_seconds", ctypes.c_double), ("seconds", ctypes.c_double),
                ("overlapped_seconds", ctypes.c_double), ("serial_seconds", ctypes.c_double)]


class Trace(ctypes.Structure):
    _fields_ = [("capacity", ctypes.c_int32), ("count", ctypes.c_int32), ("seconds", ctypes.POINTER(ctypes.c_double)),
                ("mdl", ctypes.POINTER(ctypes.c_double))]


_lib = None
_i32p = ctypes.POINTER(ctypes.c_int32)
_u32p = ctypes.POINTER(ctypes.c_uint32)
_f64p = ctypes.POINTER(ctypes.c_double)


def load(path=LIB_PATH):
    """Load the CUDA library (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise SbpError(2, f"{path} is missing: run __graft_entry__.build() (no CPU fallback exists)")
    L = ctypes.CDLL(path)
    vp = ctypes.c_void_p
    pp = ctypes.POINTER(ctypes.c_void_p)
    L.sbp_last_error.restype = ctypes.c_char_p
    L.sbp_device_count.restype = ctypes.c_int32
    for name in EXPORTED[2:]:
        getattr(L, name).restype = ctypes.c_int
    L.sbp_set_option.argtypes = [ctypes.c_char_p, ctypes.c_int64]
    L.sbp_get_stream.argtypes = [pp]
    L.sbp_profile_enable.argtypes = [ctypes.c_int32]
    L.sbp_profile_read.argtypes = [ctypes.POINTER(Profile), ctypes.c_int32]
    L.sbp_graph_create.argtypes = [ctypes.c_int32, ctypes.c_int64, _i32p, _i32p, pp]
    L.sbp_graph_destroy.argtypes = [vp]
    L.sbp_graph_num_edges.argtypes = [vp, ctypes.POINTER(ctypes.c_int64)]
    L.sbp_graph_get_split.argtypes = [vp, _i32p, _i32p, _i32p]
    L.sbp_graph_set_split.argtypes = [vp, ctypes.c_int32, _i32p, ctypes.c_int32, _i32p]
    L.sbp_blockmodel_create.argtypes = [vp, ctypes.c_int32, _i32p, pp]
    L.sbp_blockmodel_copy.argtypes = [vp, pp]
    L.sbp_blockmodel_destroy.argtypes = [vp]
    L.sbp_blockmodel_num_blocks.argtypes = [vp, _i32p]
    L.sbp_blockmodel_set_num_blocks_to_merge.argtypes = [vp, ctypes.c_int32]
    L.sbp_blockmodel_overall_entropy.argtypes = [vp, ctypes.POINTER(ctypes.c_float)]
    L.sbp_get_assignment.argtypes = [vp, _i32p]
    L.sbp_get_block_matrix.argtypes = [vp, _i32p]
    L.sbp_get_degrees.argtypes = [vp, _i32p, _i32p, _i32p]
    L.sbp_mdl.argtypes = [vp, vp, _f64p]
    L.sbp_evaluate_vertices.argtypes = [vp, vp, ctypes.c_int32, _i32p, _u32p, _i32p, _f64p, _f64p, _i32p]
    L.sbp_move_vertex.argtypes = [vp, vp, ctypes.c_int32, ctypes.c_int32]
    L.sbp_finetune.argtypes = [vp, vp, ctypes.c_int32, ctypes.POINTER(FinetuneOptions), ctypes.POINTER(Replay),
                               ctypes.POINTER(Stats)]
    L.sbp_merge_blocks.argtypes = [vp, vp, ctypes.POINTER(MergeOptions), ctypes.POINTER(Replay), _i32p, _f64p,
                                   ctypes.POINTER(Stats)]
    L.sbp_partition.argtypes = [vp, ctypes.POINTER(Options), _i32p, ctypes.POINTER(Stats)]
    L.sbp_finetune_replayed.argtypes = [vp, vp, ctypes.c_int32, ctypes.POINTER(FinetuneOptions),
                                        ctypes.POINTER(MoveReplay), ctypes.POINTER(Stats)]
    L.sbp_merge_blocks_replayed.argtypes = [vp, vp, ctypes.POINTER(MergeOptions), ctypes.POINTER(MoveReplay), _i32p,
                                            _f64p, ctypes.POINTER(Stats)]
    L.sbp_set_degrees.argtypes = [vp, _i32p]
    L.sbp_get_intermediates.argtypes = [ctypes.POINTER(Intermediate), ctypes.c_int32, _i32p]
    L.sbp_clear_intermediates.argtypes = []
    i64p = ctypes.POINTER(ctypes.c_int64)
    L.sbp_contingency_metrics.argtypes = [ctypes.c_int32, ctypes.c_int32, i64p, ctypes.c_int64,
                                          ctypes.POINTER(Evaluation)]
    L.sbp_evaluate_blockmodel.argtypes = [vp, vp, _i32p, ctypes.POINTER(Evaluation), i64p]
    L.sbp_mdl_of_cells.argtypes = [ctypes.c_int32, ctypes.c_int64, _i32p, _i32p, _i32p, _i32p, _i32p, ctypes.c_int32,
                                   ctypes.c_int64, _f64p]
    L.sbp_partition_replayed.argtypes = [vp, ctypes.POINTER(Options), ctypes.c_int32, ctypes.c_int32,
                                         ctypes.POINTER(MoveReplay), _i32p, _i32p, _i32p, ctypes.POINTER(Stats)]
    L.sbp_mdl_device_noalloc.argtypes = [vp, ctypes.c_int32, ctypes.c_int64, vp, vp, ctypes.c_int32, ctypes.c_int64,
                                         vp, vp]
    f32p = ctypes.POINTER(ctypes.c_float)
    L.sbp_mlp_create.argtypes = [ctypes.c_uint64, pp]
    L.sbp_mlp_destroy.argtypes = [vp]
    L.sbp_mlp_get_params.argtypes = [vp, f32p]
    L.sbp_mlp_set_params.argtypes = [vp, f32p]
    L.sbp_mlp_forward.argtypes = [vp, ctypes.c_int64, f32p, f32p]
    L.sbp_mlp_gradients.argtypes = [vp, ctypes.c_int64, f32p, _i32p, _i32p, f32p, _f64p]
    L.sbp_mlp_train.argtypes = [vp, vp, ctypes.POINTER(TrainOptions), ctypes.POINTER(TrainStats)]
    L.sbp_dataset_create.argtypes = [ctypes.c_int64, pp]
    L.sbp_dataset_destroy.argtypes = [vp]
    L.sbp_dataset_size.argtypes = [vp, ctypes.POINTER(ctypes.c_int64)]
    L.sbp_dataset_append.argtypes = [vp, ctypes.c_int64, f32p, _i32p, _i32p]
    L.sbp_dataset_read.argtypes = [vp, ctypes.c_int64, ctypes.c_int64, ctypes.POINTER(ctypes.c_uint16), _i32p, _i32p]
    L.sbp_vertex_features.argtypes = [vp, vp, ctypes.c_int32, _i32p, f32p, _i32p, _i32p]
    L.sbp_learned_evaluate.argtypes = [vp, vp, vp, ctypes.c_int32, _i32p, _u32p, ctypes.c_float, _i32p, _f64p, _f64p,
                                       _f64p, _i32p]
    L.sbp_learned_q.argtypes = [vp, vp, vp, ctypes.c_int32, _i32p, _i32p, ctypes.c_float, _f64p]
    L.sbp_collect_moves.argtypes = [vp, vp, vp, ctypes.POINTER(FinetuneOptions), ctypes.POINTER(Stats)]
    L.sbp_finetune_learned.argtypes = [vp, vp, ctypes.c_int32, ctypes.POINTER(FinetuneOptions), vp,
                                       ctypes.POINTER(LearnedOptions), ctypes.POINTER(Trace), ctypes.POINTER(Stats)]
    L.sbp_partition_learned.argtypes = [vp, ctypes.POINTER(Options), vp, ctypes.POINTER(LearnedOptions), _i32p,
                                        ctypes.POINTER(Stats)]
    L.sbp_partition_batched.argtypes = [ctypes.c_int32, ctypes.POINTER(vp), ctypes.POINTER(Options),
                                        ctypes.POINTER(_i32p), ctypes.POINTER(Stats), ctypes.POINTER(BatchInfo)]
    L.sbp_batched_reset_tuning.argtypes = []
    _lib = L
    return L


def _check(rc):
    if rc != 0:
        raise SbpError(rc, _lib.sbp_last_error().decode())


def last_error():
    """sbp_last_error(): the text of the calling thread's last failure."""
    return _lib.sbp_last_error().decode()


def _p(a, t=_i32p):
    return a.ctypes.data_as(t)


def _replay(records):
    if records is None:
        return None, None
    arr = np.ascontiguousarray(records, dtype=np.uint32).reshape(-1)
    rp = Replay(arr.ctypes.data_as(_u32p), len(arr) // 4)
    return arr, ctypes.byref(rp)


def device_count():
    return load().sbp_device_count()


def set_option(name, value):
    """Engine option, e.g. set_option("dense_max_blocks", 65536) (include/sbp_b200.h lists them)."""
    _check(load().sbp_set_option(name.encode(), int(value)))


def release_cached_memory():
    """Free the device buffers the library keeps cached for reuse."""
    _check(load().sbp_release_cached_memory())


def stream_handle():
    """cudaStream_t of the library (use with torch.cuda.ExternalStream for events)."""
    h = ctypes.c_void_p()
    _check(load().sbp_get_stream(ctypes.byref(h)))
    return h.value


def profile_enable(on=True):
    _check(load().sbp_profile_enable(int(bool(on))))


def profile_read(reset=False):
    p = Profile()
    _check(load().sbp_profile_read(ctypes.byref(p), int(bool(reset))))
    return {k: getattr(p, k) for k, _ in p._fields_}


class Graph:
    """Device-resident directed graph (Graph::load_text semantics: first occurrence of each edge kept)."""

    def __init__(self, num_vertices, src, dst):
        L = load()
        s = np.ascontiguousarray(src, dtype=np.int32)
        d = np.ascontiguousarray(dst, dtype=np.int32)
        if s.shape != d.shape:
            raise SbpError(1, "src and dst differ in length")
        h = ctypes.c_void_p()
        _check(L.sbp_graph_create(int(num_vertices), len(s), _p(s), _p(d), ctypes.byref(h)))
        self.h = h
        self.V = int(num_vertices)
        e = ctypes.c_int64()
        _check(L.sbp_graph_num_edges(h, ctypes.byref(e)))
        self.E = e.value

    def num_vertices(self):
        return self.V

    def num_edges(self):
        return self.E

    def split(self):
        nh = ctypes.c_int32()
        hi = np.zeros(self.V, np.int32)
        lo = np.zeros(self.V, np.int32)
        _check(_lib.sbp_graph_get_split(self.h, ctypes.byref(nh), _p(hi), _p(lo)))
        return hi[:nh.value].copy(), lo[:self.V - nh.value].copy()

    def set_split(self, high, low):
        hi = np.ascontiguousarray(high, np.int32)
        lo = np.ascontiguousarray(low, np.int32)
        _check(_lib.sbp_graph_set_split(self.h, len(hi), _p(hi), len(lo), _p(lo)))

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.sbp_graph_destroy(self.h)
            self.h = None


class Blockmodel:
    """Device-resident blockmodel: assignment, B x B counts, degrees (Blockmodel)."""

    def __init__(self, graph, num_blocks=None, assignment=None, _handle=None):
        self.graph = graph
        if _handle is not None:
            self.h = _handle
            return
        a = np.ascontiguousarray(assignment, dtype=np.int32)
        h = ctypes.c_void_p()
        _check(load().sbp_blockmodel_create(graph.h, int(num_blocks), _p(a), ctypes.byref(h)))
        self.h = h

    def copy(self):
        h = ctypes.c_void_p()
        _check(_lib.sbp_blockmodel_copy(self.h, ctypes.byref(h)))
        return Blockmodel(self.graph, _handle=h)

    def getNum_blocks(self):
        b = ctypes.c_int32()
        _check(_lib.sbp_blockmodel_num_blocks(self.h, ctypes.byref(b)))
        return b.value

    B = property(getNum_blocks)

    def setNum_blocks_to_merge(self, n):
        _check(_lib.sbp_blockmodel_set_num_blocks_to_merge(self.h, int(n)))

    def getOverall_entropy(self):
        f = ctypes.c_float()
        _check(_lib.sbp_blockmodel_overall_entropy(self.h, ctypes.byref(f)))
        return f.value

    def block_assignment(self):
        out = np.zeros(self.graph.V, np.int32)
        _check(_lib.sbp_get_assignment(self.h, _p(out)))
        return out

    def blockmatrix(self):
        B = self.B
        out = np.zeros(B * B, np.int32)
        _check(_lib.sbp_get_block_matrix(self.h, _p(out)))
        return out.reshape(B, B)

    def degrees_all(self):
        B = self.B
        do, di, d = (np.zeros(B, np.int32) for _ in range(3))
        _check(_lib.sbp_get_degrees(self.h, _p(do), _p(di), _p(d)))
        return do, di, d

    def degrees_out(self):
        return self.degrees_all()[0]

    def degrees_in(self):
        return self.degrees_all()[1]

    def degrees(self):
        return self.degrees_all()[2]

    def move_vertex(self, vertex, block):
        _check(_lib.sbp_move_vertex(self.h, self.graph.h, int(vertex), int(block)))

    def evaluate_vertices(self, vertices, records):
        v = np.ascontiguousarray(vertices, np.int32)
        r = np.ascontiguousarray(records, np.uint32).reshape(-1)
        n = len(v)
        s = np.zeros(n, np.int32)
        dS = np.zeros(n, np.float64)
        H = np.zeros(n, np.float64)
        acc = np.zeros(n, np.int32)
        _check(_lib.sbp_evaluate_vertices(self.h, self.graph.h, n, _p(v), _p(r, _u32p), _p(s), _p(dS, _f64p),
                                          _p(H, _f64p), _p(acc)))
        return s, dS, H, acc.astype(bool)

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.sbp_blockmodel_destroy(self.h)
            self.h = None


class entropy:
    @staticmethod
    def mdl(blockmodel, graph=None):
        out = ctypes.c_double()
        _check(_lib.sbp_mdl(blockmodel.h, (graph or blockmodel.graph).h, ctypes.byref(out)))
        return out.value


class finetune:
    @staticmethod
    def run(blockmodel, algorithm, batches=10, bracket=False, seed=0, call=0, replay=None, max_sweeps=0):
        opt = FinetuneOptions(int(batches), int(bool(bracket)), int(max_sweeps), int(call), int(seed))
        keep, rp = _replay(replay)
        st = Stats()
        _check(_lib.sbp_finetune(blockmodel.h, blockmodel.graph.h, int(algorithm), ctypes.byref(opt), rp,
                                 ctypes.byref(st)))
        del keep
        return st.as_dict()

    @staticmethod
    def replayed(blockmodel, algorithm, proposal, uniform, batches=10, bracket=False, max_sweeps=0):
        """finetune with the proposals and accept uniforms of a recorded stream
        (sbp_finetune_replayed): proposal[t*V + v], uniform[t*V + v] for vertex v in sweep t."""
        prop = np.ascontiguousarray(proposal, np.int32)
        uni = np.ascontiguousarray(uniform, np.float64)
        if prop.shape != uni.shape:
            raise ValueError("proposal and uniform streams differ in length")
        opt = FinetuneOptions(int(batches), int(bool(bracket)), int(max_sweeps), 0, 0)
        rp = MoveReplay(_p(prop), _p(uni, _f64p), len(prop))
        st = Stats()
        algo = ALGORITHMS[algorithm] if isinstance(algorithm, str) else int(algorithm)
        _check(_lib.sbp_finetune_replayed(blockmodel.h, blockmodel.graph.h, algo, ctypes.byref(opt), ctypes.byref(rp),
                                          ctypes.byref(st)))
        return st.as_dict()

    @staticmethod
    def metropolis_hastings(blockmodel, **kw):
        return finetune.run(blockmodel, METROPOLIS_HASTINGS, **kw)

    @staticmethod
    def asynchronous_gibbs(blockmodel, **kw):
        return finetune.run(blockmodel, ASYNC_GIBBS, **kw)

    @staticmethod
    def hybrid_mcmc(blockmodel, **kw):
        return finetune.run(blockmodel, HYBRID_MCMC, **kw)


class block_merge:
    @staticmethod
    def merge_blocks(blockmodel, approximate=True, seed=0, call=0, replay=None):
        B = blockmodel.B
        best = np.zeros(B, np.int32)
        dS = np.zeros(B, np.float64)
        opt = MergeOptions(int(bool(approximate)), int(call), int(seed))
        keep, rp = _replay(replay)
        st = Stats()
        _check(_lib.sbp_merge_blocks(blockmodel.h, blockmodel.graph.h, ctypes.byref(opt), rp, _p(best),
                                     _p(dS, _f64p), ctypes.byref(st)))
        del keep
        return dict(best=best, dS=dS, **st.as_dict())

    @staticmethod
    def merge_blocks_replayed(blockmodel, proposal, approximate=True):
        """merge_blocks with every proposal taken from a recorded stream (sbp_merge_blocks_replayed):
        proposal[block*10 + i] is proposal i of a block."""
        B = blockmodel.B
        best = np.zeros(B, np.int32)
        dS = np.zeros(B, np.float64)
        prop = np.ascontiguousarray(proposal, np.int32)
        opt = MergeOptions(int(bool(approximate)), 0, 0)
        rp = MoveReplay(_p(prop), None, len(prop))
        st = Stats()
        _check(_lib.sbp_merge_blocks_replayed(blockmodel.h, blockmodel.graph.h, ctypes.byref(opt), ctypes.byref(rp),
                                              _p(best), _p(dS, _f64p), ctypes.byref(st)))
        return dict(best=best, dS=dS, **st.as_dict())


def mdl_device_noalloc(d_matrix, num_blocks, ld, d_degrees_out, d_degrees_in, num_vertices, num_edges, d_result,
                       stream=None):
    """MDL of device-resident counts without any GPU allocation (sbp_mdl_device_noalloc).
    Pointer arguments are raw device addresses (ints); the result is written to d_result on
    `stream` (a cudaStream_t as int, or None for the legacy default stream)."""
    rc = load().sbp_mdl_device_noalloc(d_matrix, int(num_blocks), int(ld), d_degrees_out, d_degrees_in,
                                       int(num_vertices), int(num_edges), d_result, stream)
    if rc != 0:
        raise SbpError(rc, last_error())


class evaluate:
    """evaluate::evaluate_blockmodel / calculate_f1_score / calculate_nmi (src/evaluate.cpp:7-178)."""

    @staticmethod
    def contingency_metrics(table, num_vertices):
        t = np.ascontiguousarray(table, np.int64)
        ev = Evaluation()
        _check(load().sbp_contingency_metrics(t.shape[0], t.shape[1], t.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                                              int(num_vertices), ctypes.byref(ev)))
        return ev.as_dict()

    @staticmethod
    def evaluate_blockmodel(blockmodel, true_assignment, with_table=False):
        truth = np.ascontiguousarray(true_assignment, np.int32)
        ev = Evaluation()
        known = truth[truth >= 0]
        K = len(np.unique(known))
        table = np.zeros((blockmodel.B, max(K, 1)), np.int64)
        _check(_lib.sbp_evaluate_blockmodel(blockmodel.h, blockmodel.graph.h, _p(truth), ctypes.byref(ev),
                                            table.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))))
        out = ev.as_dict()
        if with_table:
            out["table"] = table
        return out


def set_degrees(blockmodel, d):
    """sbp_set_degrees: overwrite the block degrees d of a blockmodel."""
    dd = np.ascontiguousarray(d, np.int32)
    _check(_lib.sbp_set_degrees(blockmodel.h, _p(dd)))


def mdl_of_cells(num_blocks, rows, cols, counts, d_out, d_in, num_vertices, num_edges):
    """sbp_mdl_of_cells: entropy::mdl of host cell lists and degrees."""
    r, c, v = (np.ascontiguousarray(x, np.int32) for x in (rows, cols, counts))
    do, di = np.ascontiguousarray(d_out, np.int32), np.ascontiguousarray(d_in, np.int32)
    out = ctypes.c_double()
    _check(load().sbp_mdl_of_cells(int(num_blocks), len(v), _p(r), _p(c), _p(v), _p(do), _p(di), int(num_vertices),
                                   int(num_edges), ctypes.byref(out)))
    return out.value


class sbp:
    @staticmethod
    def stochastic_block_partition(graph, algorithm="async_gibbs", batches=10, approximate=True,
                                   asynciterations=2**31 - 1, seed=0):
        algo = ALGORITHMS[algorithm] if isinstance(algorithm, str) else int(algorithm)
        opt = Options(algo, int(batches), int(bool(approximate)), int(asynciterations), int(seed))
        out = np.zeros(graph.V, np.int32)
        st = Stats()
        _check(_lib.sbp_partition(graph.h, ctypes.byref(opt), _p(out), ctypes.byref(st)))
        return out, st.as_dict()

    @staticmethod
    def get_intermediates():
        """sbp::get_intermediates: the records of every partition of this process (list of dicts)."""
        n = ctypes.c_int32()
        _check(load().sbp_get_intermediates(None, 0, ctypes.byref(n)))
        arr = (Intermediate * max(1, n.value))()
        _check(_lib.sbp_get_intermediates(arr, n.value, ctypes.byref(n)))
        return [arr[i].as_dict() for i in range(n.value)]

    @staticmethod
    def clear_intermediates():
        _check(load().sbp_clear_intermediates())

    @staticmethod
    def stochastic_block_partition_replayed(graph, calls, algorithm="async_gibbs", batches=10, approximate=True,
                                            max_sweeps=0):
        """sbp_partition_replayed: `calls` lists the recorded stream of every merge and finetune
        call in call order, each (proposal, uniform) with uniform None for a merge.  Returns
        (assignment, stats, blocks after each call)."""
        algo = ALGORITHMS[algorithm] if isinstance(algorithm, str) else int(algorithm)
        opt = Options(algo, int(batches), int(bool(approximate)), 2**31 - 1, 0)
        keep = []
        arr = (MoveReplay * len(calls))()
        for k, (prop, uni) in enumerate(calls):
            p = np.ascontiguousarray(prop, np.int32)
            u = None if uni is None else np.ascontiguousarray(uni, np.float64)
            keep.append((p, u))
            arr[k] = MoveReplay(_p(p), None if u is None else _p(u, _f64p), len(p))
        out = np.zeros(graph.V, np.int32)
        counts = np.zeros(len(calls), np.int32)
        made = ctypes.c_int32()
        st = Stats()
        _check(_lib.sbp_partition_replayed(graph.h, ctypes.byref(opt), int(max_sweeps), len(calls), arr, _p(out),
                                           _p(counts), ctypes.byref(made), ctypes.byref(st)))
        del keep
        return out, st.as_dict(), counts[:made.value]


# ------------------------------------------------------------------------------------------
# Learned proposal (no counterpart in the reference)
# ------------------------------------------------------------------------------------------
_f32p = ctypes.POINTER(ctypes.c_float)


class Mlp:
    """Proposal network 64 -> 128 -> 128 -> 16 (BF16 weights, FP32 accumulation, tensor cores)."""

    def __init__(self, seed=0):
        L = load()
        self.h = ctypes.c_void_p()
        _check(L.sbp_mlp_create(int(seed), ctypes.byref(self.h)))

    def params(self):
        out = np.zeros(MLP_PARAMS, np.float32)
        _check(_lib.sbp_mlp_get_params(self.h, _p(out, _f32p)))
        return out

    def set_params(self, params):
        arr = np.ascontiguousarray(params, dtype=np.float32)
        if arr.size != MLP_PARAMS:
            raise ValueError(f"expected {MLP_PARAMS} parameters")
        _check(_lib.sbp_mlp_set_params(self.h, _p(arr, _f32p)))

    def forward(self, features):
        X = np.ascontiguousarray(features, dtype=np.float32).reshape(-1, MLP_FEATURES)
        out = np.zeros((len(X), MLP_OUTPUTS), np.float32)
        _check(_lib.sbp_mlp_forward(self.h, len(X), _p(X, _f32p), _p(out, _f32p)))
        return out

    def gradients(self, features, target, nvalid):
        X = np.ascontiguousarray(features, dtype=np.float32).reshape(-1, MLP_FEATURES)
        t = np.ascontiguousarray(target, dtype=np.int32)
        nv = np.ascontiguousarray(nvalid, dtype=np.int32)
        g = np.zeros(MLP_PARAMS, np.float32)
        loss = ctypes.c_double()
        _check(_lib.sbp_mlp_gradients(self.h, len(X), _p(X, _f32p), _p(t), _p(nv), _p(g, _f32p), ctypes.byref(loss)))
        return g, loss.value

    def train(self, dataset, epochs=1, batch=1024, lr=1e-3, seed=0):
        opt = TrainOptions(int(epochs), int(batch), float(lr), 0, int(seed))
        st = TrainStats()
        _check(_lib.sbp_mlp_train(self.h, dataset.h, ctypes.byref(opt), ctypes.byref(st)))
        return {k: getattr(st, k) for k, _ in st._fields_}

    def __del__(self):
        if _lib is not None and getattr(self, "h", None):
            _lib.sbp_mlp_destroy(self.h)
            self.h = None


class Dataset:
    """Device-resident training samples (features, target slot, valid slots)."""

    def __init__(self, capacity):
        L = load()
        self.h = ctypes.c_void_p()
        _check(L.sbp_dataset_create(int(capacity), ctypes.byref(self.h)))

    def __len__(self):
        n = ctypes.c_int64()
        _check(_lib.sbp_dataset_size(self.h, ctypes.byref(n)))
        return n.value

    def append(self, features, target, nvalid):
        X = np.ascontiguousarray(features, dtype=np.float32).reshape(-1, MLP_FEATURES)
        t = np.ascontiguousarray(target, dtype=np.int32)
        nv = np.ascontiguousarray(nvalid, dtype=np.int32)
        _check(_lib.sbp_dataset_append(self.h, len(X), _p(X, _f32p), _p(t), _p(nv)))

    def read(self, offset=0, n=None):
        n = len(self) - offset if n is None else n
        fb = np.zeros((n, MLP_FEATURES), np.uint16)
        t = np.zeros(n, np.int32)
        nv = np.zeros(n, np.int32)
        _check(_lib.sbp_dataset_read(self.h, int(offset), int(n), fb.ctypes.data_as(ctypes.POINTER(ctypes.c_uint16)),
                                     _p(t), _p(nv)))
        X = (fb.astype(np.uint32) << 16).view(np.float32)
        return X, t, nv

    def __del__(self):
        if _lib is not None and getattr(self, "h", None):
            _lib.sbp_dataset_destroy(self.h)
            self.h = None


class learned:
    @staticmethod
    def vertex_features(blockmodel, vertices):
        v = np.ascontiguousarray(vertices, dtype=np.int32)
        n = len(v)
        F = np.zeros((n, MLP_FEATURES), np.float32)
        S = np.zeros((n, MLP_SLOTS), np.int32)
        nv = np.zeros(n, np.int32)
        _check(_lib.sbp_vertex_features(blockmodel.h, blockmodel.graph.h, n, _p(v), _p(F, _f32p), _p(S), _p(nv)))
        return F, S, nv

    @staticmethod
    def evaluate(blockmodel, mlp, vertices, records, epsilon=0.05):
        v = np.ascontiguousarray(vertices, dtype=np.int32)
        rec = np.ascontiguousarray(records, dtype=np.uint32).reshape(-1, 4)
        n = len(v)
        s = np.zeros(n, np.int32)
        qf = np.zeros(n, np.float64)
        dS = np.zeros(n, np.float64)
        H = np.zeros(n, np.float64)
        acc = np.zeros(n, np.int32)
        _check(_lib.sbp_learned_evaluate(blockmodel.h, blockmodel.graph.h, mlp.h, n, _p(v), _p(rec, _u32p),
                                         float(epsilon), _p(s), _p(qf, _f64p), _p(dS, _f64p), _p(H, _f64p), _p(acc)))
        return s, qf, dS, H, acc

    @staticmethod
    def q(blockmodel, mlp, vertices, blocks, epsilon=0.05):
        v = np.ascontiguousarray(vertices, dtype=np.int32)
        b = np.ascontiguousarray(blocks, dtype=np.int32)
        out = np.zeros(len(v), np.float64)
        _check(_lib.sbp_learned_q(blockmodel.h, blockmodel.graph.h, mlp.h, len(v), _p(v), _p(b), float(epsilon),
                                  _p(out, _f64p)))
        return out

    @staticmethod
    def collect_moves(blockmodel, dataset, batches=10, sweeps=10, seed=0, call=0):
        opt = FinetuneOptions(int(batches), 0, int(sweeps), int(call), int(seed))
        st = Stats()
        _check(_lib.sbp_collect_moves(blockmodel.h, blockmodel.graph.h, dataset.h, ctypes.byref(opt),
                                      ctypes.byref(st)))
        return st.as_dict()

    @staticmethod
    def finetune(blockmodel, mlp=None, algorithm="async_gibbs", batches=10, bracket=False, seed=0, call=0,
                 max_sweeps=0, epsilon=0.05, fallback_acceptance=0.0, stop_rule=0, trace=True):
        algo = ALGORITHMS[algorithm] if isinstance(algorithm, str) else int(algorithm)
        opt = FinetuneOptions(int(batches), int(bool(bracket)), int(max_sweeps), int(call), int(seed))
        lo = LearnedOptions(float(epsilon), float(fallback_acceptance), int(stop_rule), 0)
        cap = 128
        secs = np.zeros(cap, np.float64)
        mdls = np.zeros(cap, np.float64)
        tr = Trace(cap, 0, secs.ctypes.data_as(_f64p), mdls.ctypes.data_as(_f64p)) if trace else None
        st = Stats()
        _check(_lib.sbp_finetune_learned(blockmodel.h, blockmodel.graph.h, algo, ctypes.byref(opt),
                                         mlp.h if mlp is not None else None, ctypes.byref(lo),
                                         ctypes.byref(tr) if tr is not None else None, ctypes.byref(st)))
        out = st.as_dict()
        if tr is not None:
            out["trace_seconds"] = secs[:tr.count].copy()
            out["trace_mdl"] = mdls[:tr.count].copy()
        return out

    @staticmethod
    def stochastic_block_partition(graph, mlp=None, algorithm="async_gibbs", batches=10, approximate=True,
                                   asynciterations=2**31 - 1, seed=0, epsilon=0.05, fallback_acceptance=0.0,
                                   stop_rule=1):
        algo = ALGORITHMS[algorithm] if isinstance(algorithm, str) else int(algorithm)
        opt = Options(algo, int(batches), int(bool(approximate)), int(asynciterations), int(seed))
        lo = LearnedOptions(float(epsilon), float(fallback_acceptance), int(stop_rule), 0)
        out = np.zeros(graph.V, np.int32)
        st = Stats()
        _check(_lib.sbp_partition_learned(graph.h, ctypes.byref(opt), mlp.h if mlp is not None else None,
                                          ctypes.byref(lo), _p(out), ctypes.byref(st)))
        return out, st.as_dict()


# ------------------------------------------------------------------------------------------
# Batched partitioning (no counterpart in the reference)
# ------------------------------------------------------------------------------------------
class batched:
    @staticmethod
    def stochastic_block_partition(graphs, algorithm="async_gibbs", batches=10, approximate=True,
                                   asynciterations=2**31 - 1, seed=0):
        """Partition every graph (each exactly as sbp.stochastic_block_partition would) with the
        finetunes of all graphs in one persistent launch per sweep.  Returns (assignments, stats,
        info)."""
        load()
        algo = ALGORITHMS[algorithm] if isinstance(algorithm, str) else int(algorithm)
        opt = Options(algo, int(batches), int(bool(approximate)), int(asynciterations), int(seed))
        n = len(graphs)
        outs = [np.zeros(g.V, np.int32) for g in graphs]
        hs = (ctypes.c_void_p * n)(*[g.h.value if isinstance(g.h, ctypes.c_void_p) else g.h for g in graphs])
        ps = (_i32p * n)(*[_p(o) for o in outs])
        st = (Stats * n)()
        info = BatchInfo()
        _check(_lib.sbp_partition_batched(n, hs, ctypes.byref(opt), ps, st, ctypes.byref(info)))
        inf = {k: getattr(info, k) for k, _ in info._fields_}
        inf["candidate_ms"] = list(info.candidate_ms)[:info.candidates]
        return outs, [x.as_dict() for x in st], inf

    @staticmethod
    def reset_tuning():
        _check(load().sbp_batched_reset_tuning())
