"""Expression selection on the GPU (include/fls_select.h): the exact-size wizard and the learned selector.

The reference picks an expression per column by encoding it with every expression of its pool and keeping the
smallest (src/encoder/exp_col_encoder.cpp:18-28 encode_all, :117-129 GetBest).  ``SelectionPlan.wizard`` does
that exactly on the GPU for the six no-patch candidates of ``CANDIDATES`` per (column, row-group) chunk;
``SelectionPlan.learned`` replaces the trial encodes by 32 statistics of a sample of every chunk's vectors and
an MLP trained on wizard labels (``train_selector``).
"""
import ctypes

import numpy as np
import torch

from ._lib import check, declare

_p = ctypes.c_void_p
_u8 = ctypes.c_uint8
_u32 = ctypes.c_uint32
_u64 = ctypes.c_uint64
_f = ctypes.c_float
_i = ctypes.c_int

CANDIDATES = ("UNCOMPRESSED", "FFOR", "RLE", "DELTA", "DICT", "DICT_RLE")
POOL_IDS = (0, 1, 6, 11, 17, 27)  # reference i64 pool ids (src/cor/exp_pool.cpp:25-52)
K = len(CANDIDATES)
N_FEATURES = 32
HIDDEN = 128


class SelColumn(ctypes.Structure):
    _fields_ = [("d_values", _p), ("n_vec", _u64), ("width", _u8), ("is_signed", _u8), ("pad", _u8 * 6)]


_plan_create = declare("fls_sel_plan_create", _i, [ctypes.POINTER(SelColumn), _u32, _u32, ctypes.POINTER(_p)])
_plan_info = declare("fls_sel_plan_info", _i, [_p, ctypes.POINTER(_u64), ctypes.POINTER(_u64)])
_plan_chunks = declare("fls_sel_plan_chunks", _i, [_p, _p, _p, _p])
_plan_destroy = declare("fls_sel_plan_destroy", _i, [_p])
_parts = declare("fls_sel_vector_parts", _i, [_p, _p, _p])
_wizard = declare("fls_sel_wizard", _i, [_p, _p, _p, _p, _p])
_features = declare("fls_sel_features", _i, [_p, _u32, _p, _p, ctypes.POINTER(_u64), _p])
_learned = declare("fls_sel_learned", _i, [_p, _p, _u32, _f, _p, _p, ctypes.POINTER(_u64), _p])
_param_count = declare("fls_sel_param_count", _u64, [])
_mlp_init = declare("fls_sel_mlp_init", _i, [_p, _u64])
_mlp_forward = declare("fls_sel_mlp_forward", _i, [_p, _p, _u64, _p, _p])
_mlp_grad = declare("fls_sel_mlp_grad", _i, [_p, _p, _p, _u64, _p, _p, _p])
_adam = declare("fls_sel_adam_step", _i, [_p, _p, _p, _p, _f, _f, _f, _f, _u32, _p])
_train = declare("fls_sel_train", _i, [_p, _p, _p, _p, _u32, _u32, _f, _p, _p])

_WIDTH = {torch.int32: (32, 1), torch.int64: (64, 1)}

STR_CANDIDATES = ("BYTE_ARR", "DICT", "FSST", "DICT_RLE")
STR_POOL_IDS = (0, 3, 13, 15)  # reference string pool ids (src/cor/exp_pool.cpp:66-101)
STR_K = len(STR_CANDIDATES)


class SelStrColumn(ctypes.Structure):
    _fields_ = [("d_bytes", _p), ("d_offsets", _p), ("n_rows", _u64), ("table", _p), ("table_size", _u64)]


_plan_create_str = declare("fls_sel_plan_create_strings", _i, [ctypes.POINTER(SelStrColumn), _u32, _u32,
                                                                ctypes.POINTER(_p)])


def _stream(stream):
    return stream if stream is not None else torch.cuda.current_stream().cuda_stream


class SelectionPlan:
    """Chunks of a set of integer columns.  columns: list of (tensor, is_signed) or tensors (int32 / int64
    on the GPU, whole vectors; int tensors stand for unsigned columns when is_signed is False)."""

    def __init__(self, columns, chunk_vectors=64):
        cols = (SelColumn * max(len(columns), 1))()
        self._keep = []
        for i, c in enumerate(columns):
            t, sgn = (c if isinstance(c, tuple) else (c, True))
            if t.dtype not in _WIDTH or not t.is_cuda or t.numel() % 1024:
                raise ValueError("columns are int32 / int64 CUDA tensors of whole 1024-value vectors")
            t = t.contiguous()
            self._keep.append(t)
            cols[i].d_values = t.data_ptr()
            cols[i].n_vec = t.numel() // 1024
            cols[i].width = _WIDTH[t.dtype][0]
            cols[i].is_signed = 1 if sgn else 0
        h = _p()
        check(_plan_create(cols, len(columns), chunk_vectors, ctypes.byref(h)), "fls_sel_plan_create")
        self.handle = h
        nc, nv = _u64(), _u64()
        check(_plan_info(h, ctypes.byref(nc), ctypes.byref(nv)), "plan_info")
        self.n_chunks, self.n_vectors = nc.value, nv.value

    def chunks(self):
        col = np.zeros(self.n_chunks, np.uint32)
        first = np.zeros(self.n_chunks, np.uint64)
        count = np.zeros(self.n_chunks, np.uint32)
        check(_plan_chunks(self.handle, col.ctypes.data, first.ctypes.data, count.ctypes.data), "plan_chunks")
        return col, first, count

    def vector_parts(self, stream=None):
        out = torch.empty(self.n_vectors, dtype=torch.int32, device="cuda")
        check(_parts(self.handle, out.data_ptr(), _stream(stream)), "vector_parts")
        return out

    def wizard(self, stream=None):
        """(sizes[n_chunks, K] int64 bytes, best[n_chunks] uint8, distinct values per chunk int32)"""
        sizes = torch.empty((self.n_chunks, K), dtype=torch.int64, device="cuda")
        best = torch.empty(self.n_chunks, dtype=torch.uint8, device="cuda")
        dn = torch.empty(self.n_chunks, dtype=torch.int32, device="cuda")
        check(_wizard(self.handle, sizes.data_ptr(), best.data_ptr(), dn.data_ptr(), _stream(stream)), "wizard")
        return sizes, best, dn

    def features(self, stride=1, stream=None):
        """(features[rows, 32] float32, chunk of every row) of vectors 0, stride, ... of every chunk"""
        n = _u64()
        check(_features(self.handle, stride, None, None, ctypes.byref(n), _stream(stream)), "features")
        feat = torch.empty((n.value, N_FEATURES), dtype=torch.float32, device="cuda")
        rc = torch.empty(n.value, dtype=torch.int32, device="cuda")
        check(_features(self.handle, stride, feat.data_ptr(), rc.data_ptr(), ctypes.byref(n), _stream(stream)),
              "features")
        return feat, rc

    def learned(self, params, stride=8, threshold=0.0, stream=None):
        """(choice[n_chunks] uint8, confidence[n_chunks] float32, chunks sent to the wizard)"""
        choice = torch.empty(self.n_chunks, dtype=torch.uint8, device="cuda")
        conf = torch.empty(self.n_chunks, dtype=torch.float32, device="cuda")
        nf = _u64()
        check(_learned(self.handle, params.data_ptr(), stride, threshold, choice.data_ptr(), conf.data_ptr(),
                       ctypes.byref(nf), _stream(stream)), "learned")
        return choice, conf, nf.value

    def close(self):
        if getattr(self, "handle", None) and _plan_destroy is not None:
            _plan_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # interpreter shutdown: the library may already be gone
            pass


class StrSelectionPlan(SelectionPlan):
    """Chunks of a set of string columns: list of (bytes uint8 CUDA tensor, offsets int64 CUDA tensor of
    n_rows + 1, the column's FSST table as host bytes).  wizard(): sizes n_chunks x 6 with the string
    candidates (``STR_CANDIDATES``) in 0..3; features / learned as for integer columns."""

    def __init__(self, columns, chunk_vectors=64):
        cols = (SelStrColumn * max(len(columns), 1))()
        self._keep = []
        for i, (byts, offs, table) in enumerate(columns):
            offs = offs.contiguous()
            table = np.ascontiguousarray(table, np.uint8)
            if offs.dtype != torch.int64 or not offs.is_cuda or (offs.numel() - 1) % 1024:
                raise ValueError("offsets: int64 CUDA tensor of n_rows + 1, n_rows whole vectors")
            self._keep += [byts, offs, table]
            cols[i].d_bytes = byts.data_ptr()
            cols[i].d_offsets = offs.data_ptr()
            cols[i].n_rows = offs.numel() - 1
            cols[i].table = table.ctypes.data
            cols[i].table_size = table.size
        h = _p()
        check(_plan_create_str(cols, len(columns), chunk_vectors, ctypes.byref(h)), "fls_sel_plan_create_strings")
        self.handle = h
        nc, nv = _u64(), _u64()
        check(_plan_info(h, ctypes.byref(nc), ctypes.byref(nv)), "plan_info")
        self.n_chunks, self.n_vectors = nc.value, nv.value


# ---- the MLP ----------------------------------------------------------------------------------------------
def param_count():
    return int(_param_count())


def mlp_init(seed=0):
    p = torch.empty(param_count(), dtype=torch.float32, device="cuda")
    check(_mlp_init(p.data_ptr(), seed), "mlp_init")
    return p


def mlp_forward(params, x, stream=None):
    x = x.contiguous()
    prob = torch.empty((x.shape[0], K), dtype=torch.float32, device="cuda")
    check(_mlp_forward(params.data_ptr(), x.data_ptr(), x.shape[0], prob.data_ptr(), _stream(stream)), "forward")
    return prob


def mlp_grad(params, x, y, stream=None):
    x, y = x.contiguous(), y.to(torch.int32).contiguous()
    g = torch.empty_like(params)
    loss = torch.empty(1, dtype=torch.float32, device="cuda")
    check(_mlp_grad(params.data_ptr(), x.data_ptr(), y.data_ptr(), x.shape[0], g.data_ptr(), loss.data_ptr(),
                    _stream(stream)), "grad")
    return float(loss.item()), g


def adam_step(params, grad, m, v, step, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8, stream=None):
    check(_adam(params.data_ptr(), grad.data_ptr(), m.data_ptr(), v.data_ptr(), lr, b1, b2, eps, step,
                _stream(stream)), "adam")


def train(params, x, y, epochs=8, batch=1024, lr=1e-3, seed=0, stream=None):
    """Minibatch Adam over (x, y) (one CUDA-graph replay per step); returns the per-step losses."""
    n = x.shape[0]
    steps_per_epoch = n // batch
    rng = np.random.default_rng(seed)
    perm = np.concatenate([rng.permutation(n)[:steps_per_epoch * batch] for _ in range(epochs)]).astype(np.uint32)
    perm_d = torch.from_numpy(perm.view(np.int32)).to("cuda")
    steps = steps_per_epoch * epochs
    hist = torch.empty(max(steps, 1), dtype=torch.float32, device="cuda")
    x, y = x.contiguous(), y.to(torch.int32).contiguous()
    check(_train(params.data_ptr(), x.data_ptr(), y.data_ptr(), perm_d.data_ptr(), batch, steps, lr, hist.data_ptr(),
                 _stream(stream)), "train")
    return hist[:steps].cpu().numpy()


# ---- training data and the trained selector ---------------------------------------------------------------
def labelled_vectors(n_chunks=3125, seed=0, chunk_vectors=64):
    """Features and wizard labels of n_chunks seeded synthetic chunks (one column each, families of
    ``workloads.selection_column``); every vector carries its chunk's best candidate."""
    from . import workloads as W
    rng = np.random.default_rng(seed)
    cols = [W.selection_column(rng, chunk_vectors) for _ in range(n_chunks)]
    plan = SelectionPlan(cols, chunk_vectors)
    sizes, best, _ = plan.wizard()
    feat, row_chunk = plan.features(1)
    y = best.long()[row_chunk.long()]
    out = (feat, y.to(torch.int32), sizes, best)
    plan.close()
    return out


def train_selector(n_chunks=3125, seed=0, epochs=10, batch=1024, lr=2e-3):
    """Parameters of the learned selector trained on n_chunks * 64 wizard-labelled vectors, and the losses."""
    feat, y, _, _ = labelled_vectors(n_chunks, seed)
    params = mlp_init(seed)
    hist = train(params, feat, y, epochs=epochs, batch=batch, lr=lr, seed=seed)
    return params, hist


def labelled_string_vectors(n_chunks=400, seed=0, chunk_vectors=16):
    """Features and wizard labels of n_chunks seeded synthetic string chunks (one column each, families of
    ``workloads.string_selection_column``); every vector carries its chunk's best string candidate."""
    from . import workloads as W
    rng = np.random.default_rng(seed)
    cols = []
    for _ in range(n_chunks):
        byts, offs, table = W.string_selection_column(rng, chunk_vectors)
        cols.append((torch.from_numpy(byts).cuda(), torch.from_numpy(offs.astype(np.int64)).cuda(), table))
    plan = StrSelectionPlan(cols, chunk_vectors)
    sizes, best, _ = plan.wizard()
    feat, row_chunk = plan.features(1)
    y = best.long()[row_chunk.long()]
    out = (feat, y.to(torch.int32), sizes, best)
    plan.close()
    return out


def ratio_loss(sizes, choice):
    """Relative excess of the chosen candidates' total bytes over the smallest possible."""
    s = sizes.double()
    chosen = s.gather(1, choice.long().view(-1, 1)).sum()
    return float(chosen / s.min(dim=1).values.sum() - 1.0)
