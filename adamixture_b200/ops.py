"""Torch-facing wrappers of the CUDA library (device tensors in, device tensors out).

Every function launches on the current torch CUDA stream of the tensors' device and
raises on any error; nothing here runs on the CPU. Operator names registered with
``register_reference_ops()`` match the reference's ``TORCH_LIBRARY`` schemas
(adamixture/src/utils_c/cuda/pack2bit.cu:147-160) so its Python resolves to these kernels.
"""
from __future__ import annotations

import torch

from . import _lib
from ._lib import ADX_BF16, ADX_F16, ADX_F32, ADX_F64, call, query_size

PRECISIONS = {"f64": ADX_F64, "f32": ADX_F32, "bf16": ADX_BF16, "f16": ADX_F16}
_TORCH_OF = {ADX_F64: torch.float64, ADX_F32: torch.float32, ADX_BF16: torch.float32, ADX_F16: torch.float32}


def precision_code(p) -> int:
    if isinstance(p, int):
        return p
    try:
        return PRECISIONS[p]
    except KeyError:
        raise ValueError(f"unknown precision {p!r}; use one of {sorted(PRECISIONS)}") from None


def input_dtype(precision) -> torch.dtype:
    """dtype of the P/Q operands an E-step of this precision reads."""
    return _TORCH_OF[precision_code(precision)]


def _ptr(t: torch.Tensor | None) -> int | None:
    return None if t is None else t.data_ptr()


def _stream(dev: torch.device) -> int:
    return torch.cuda.current_stream(dev).cuda_stream


def _check(t: torch.Tensor, name: str, dtype=None, device=None) -> None:
    if not t.is_cuda:
        raise ValueError(f"{name} must be a CUDA tensor (got {t.device})")
    if not t.is_contiguous():
        raise ValueError(f"{name} must be contiguous")
    if dtype is not None and t.dtype != dtype:
        raise ValueError(f"{name} must be {dtype} (got {t.dtype})")
    if device is not None and t.device != device:
        raise ValueError(f"{name} is on {t.device}, expected {device}")


class Workspace:
    """Grow-only device scratch buffer per device (caller-owned memory for the C ABI)."""

    _bufs: dict = {}

    @classmethod
    def get(cls, device: torch.device, nbytes: int, tag: str = "em") -> torch.Tensor:
        """Buffers of different tags never alias. The "em" buffer belongs to the E-step
        alone: its first word is the sweep's sticky status, which other scratch users
        would overwrite."""
        key = (device.type, device.index, tag)
        buf = cls._bufs.get(key)
        if buf is None or buf.numel() < nbytes:
            cls._bufs[key] = None
            # zero-filled: the E-step workspace ends with a sticky status word
            buf = torch.zeros(max(nbytes, 256), dtype=torch.uint8, device=device)
            cls._bufs[key] = buf
        return buf

    @classmethod
    def release(cls) -> None:
        cls._bufs.clear()


# ---------------------------------------------------------------- genotype layout

def unpack_u8(G: torch.Tensor, m_start: int, count: int, M: int, byte_offset: int = 0) -> torch.Tensor:
    """Decode SNP rows [m_start, m_start+count) of packed ``G`` to ``[count, N]`` uint8."""
    _check(G, "G", torch.uint8)
    N = G.shape[1]
    count = max(0, min(count, M - m_start))
    out = torch.empty((count, N), dtype=torch.uint8, device=G.device)
    if count:
        call("adx_unpack_u8", G.data_ptr(), G.shape[0], N, M, m_start, count, byte_offset,
             out.data_ptr(), _stream(G.device))
    return out


def unpack_center(G: torch.Tensor, f: torch.Tensor, m_start: int, count: int, M: int,
                  byte_offset: int = 0) -> torch.Tensor:
    """Decode and centre: ``g - 2 f_j`` (0 where missing), float32 ``[count, N]``."""
    _check(G, "G", torch.uint8)
    _check(f, "f", torch.float32, G.device)
    N = G.shape[1]
    count = max(0, min(count, M - m_start))
    out = torch.empty((count, N), dtype=torch.float32, device=G.device)
    if count:
        call("adx_unpack_center_f32", G.data_ptr(), G.shape[0], N, M, m_start, count,
             byte_offset, f.data_ptr(), out.data_ptr(), _stream(G.device))
    return out


def allele_frequency(G: torch.Tensor, M: int) -> torch.Tensor:
    _check(G, "G", torch.uint8)
    f = torch.empty(M, dtype=torch.float32, device=G.device)
    call("adx_allele_frequency", G.data_ptr(), M, G.shape[1], f.data_ptr(), _stream(G.device))
    return f


def sample_counts(G: torch.Tensor, M: int) -> torch.Tensor:
    """q_bat: 2 x observed SNPs per sample (float64)."""
    _check(G, "G", torch.uint8)
    q = torch.empty(G.shape[1], dtype=torch.float64, device=G.device)
    call("adx_sample_counts", G.data_ptr(), M, G.shape[1], q.data_ptr(), _stream(G.device))
    return q


def sample_het_counts(G: torch.Tensor, M: int) -> torch.Tensor:
    """Heterozygous genotype count per sample (float64, exact)."""
    _check(G, "G", torch.uint8)
    h = torch.empty(G.shape[1], dtype=torch.float64, device=G.device)
    call("adx_sample_het_counts", G.data_ptr(), M, G.shape[1], h.data_ptr(), _stream(G.device))
    return h


def bed_to_packed(bed_rows: torch.Tensor, N: int, M: int) -> torch.Tensor:
    """PLINK BED rows ``[M, ceil(N/4)]`` (device) -> packed ``[ceil(M/4), N]``, flipped
    0<->2 when the mean dosage/2 is >= 0.5 (the reference reader's rule)."""
    _check(bed_rows, "bed_rows", torch.uint8)
    dev = bed_rows.device
    G = torch.empty(((M + 3) // 4, N), dtype=torch.uint8, device=dev)
    nbytes = query_size("adx_bed_workspace_bytes", M, N)
    ws = Workspace.get(dev, nbytes, "bed")
    flipped = torch.zeros(1, dtype=torch.int32, device=dev)
    call("adx_bed_to_packed", bed_rows.data_ptr(), M, N, G.data_ptr(), flipped.data_ptr(),
         ws.data_ptr(), ws.numel(), _stream(dev))
    return G


def simulate_packed(Pq: torch.Tensor, Qq: torch.Tensor, miss_q: int, keys: tuple[int, int]) -> torch.Tensor:
    """Sample packed genotypes on the device from fixed-point P/Q (see src/simulate.py)."""
    _check(Pq, "Pq", torch.int32)
    _check(Qq, "Qq", torch.int32, Pq.device)
    M, K = Pq.shape
    N = Qq.shape[0]
    G = torch.empty(((M + 3) // 4, N), dtype=torch.uint8, device=Pq.device)
    call("adx_simulate_packed", Pq.data_ptr(), Qq.data_ptr(), M, N, K, keys[0], keys[1],
         miss_q, G.data_ptr(), _stream(Pq.device))
    return G


# ---------------------------------------------------------------- Adam-EM

def em_workspace_bytes(M: int, N: int, K: int, precision) -> int:
    return query_size("adx_em_workspace_bytes", M, N, K, precision_code(precision))


def em_workspace(M: int, N: int, K: int, precision, device) -> torch.Tensor:
    """A zeroed E-step workspace of its own (not the shared cache): for callers that keep
    its address, e.g. in a captured graph (``EmGraph``)."""
    return torch.zeros(max(em_workspace_bytes(M, N, K, precision), 256), dtype=torch.uint8, device=device)


def em_stats(G: torch.Tensor, P: torch.Tensor, Q: torch.Tensor, M: int, precision="f64"):
    """Sufficient statistics (A, B, T) of one E-step sweep, float64."""
    pc = precision_code(precision)
    dt = input_dtype(pc)
    _check(G, "G", torch.uint8)
    _check(P, "P", dt, G.device)
    _check(Q, "Q", dt, G.device)
    N, K = Q.shape
    dev = G.device
    A = torch.empty((M, K), dtype=torch.float64, device=dev)
    B = torch.empty((M, K), dtype=torch.float64, device=dev)
    T = torch.empty((N, K), dtype=torch.float64, device=dev)
    ws = Workspace.get(dev, em_workspace_bytes(M, N, K, pc))
    call("adx_em_stats", G.data_ptr(), M, N, K, pc, P.data_ptr(), Q.data_ptr(), A.data_ptr(),
         B.data_ptr(), T.data_ptr(), ws.data_ptr(), ws.numel(), _stream(dev))
    return A, B, T


def em_status(workspace: torch.Tensor, M: int, N: int, K: int, precision) -> int:
    """Read and clear the sweep status word of ``workspace`` (0 = ok, 5 = a bounded
    in-kernel wait timed out). Synchronises the current stream."""
    import ctypes

    out = ctypes.c_int(0)
    call("adx_em_status", workspace.data_ptr(), workspace.numel(), M, N, K,
         precision_code(precision), ctypes.addressof(out), _stream(workspace.device))
    return int(out.value)


def tc_wait_selftest(arrive: bool, limit: int, device=None) -> list[int]:
    """Run the tensor-core sweep's bounded-wait self-test on ``device``: ``[first wait's
    status, abort word, second wait's status]`` (ADX_OK = 0, ADX_ERR_TIMEOUT = 5)."""
    dev = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
    status = torch.full((3,), -1, dtype=torch.int32, device=dev)
    call("adx_tc_wait_selftest", int(bool(arrive)), int(limit), status.data_ptr(), _stream(dev))
    return [int(v) for v in status.cpu().tolist()]


def em_sweep(G: torch.Tensor, P: torch.Tensor, Q: torch.Tensor, M: int, precision,
             workspace: torch.Tensor) -> None:
    """The E-step sweep alone (partials left in ``workspace``)."""
    pc = precision_code(precision)
    N, K = Q.shape
    call("adx_em_sweep", G.data_ptr(), M, N, K, pc, P.data_ptr(), Q.data_ptr(),
         workspace.data_ptr(), workspace.numel(), _stream(G.device))


def em_sweep_loglik(G: torch.Tensor, P: torch.Tensor, Q: torch.Tensor, M: int, workspace: torch.Tensor) -> None:
    """The float64 sweep (K <= 16) with the log-likelihood of its input (P, Q) folded in."""
    N, K = Q.shape
    call("adx_em_sweep_loglik", G.data_ptr(), M, N, K, ADX_F64, P.data_ptr(), Q.data_ptr(),
         workspace.data_ptr(), workspace.numel(), _stream(G.device))


def em_sweep_blocks_info(M: int, N: int, K: int) -> tuple[int, int, int]:
    """(SNPs per block, number of blocks, CTAs per block) of the float64 sweep's partition
    (K <= 16); each CTA occupies one SM."""
    import ctypes

    spb, nb, cpb = ctypes.c_int64(0), ctypes.c_int(0), ctypes.c_int(0)
    call("adx_em_sweep_blocks_info", M, N, K, ADX_F64, ctypes.addressof(spb), ctypes.addressof(nb),
         ctypes.addressof(cpb))
    return int(spb.value), int(nb.value), int(cpb.value)


def em_sweep_blocks(G: torch.Tensor, P: torch.Tensor, Q: torch.Tensor, M: int, b0: int, b1: int,
                    workspace: torch.Tensor) -> None:
    """The float64 sweep over SNP blocks [b0, b1) into ``workspace``'s partials: only the
    packed rows of those blocks are read, and the ranges of one workspace add up to exactly
    the full sweep (``em_sweep``)."""
    _check(G, "G", torch.uint8)
    _check(P, "P", torch.float64, G.device)
    _check(Q, "Q", torch.float64, G.device)
    N, K = Q.shape
    call("adx_em_sweep_blocks", G.data_ptr(), M, N, K, ADX_F64, P.data_ptr(), Q.data_ptr(), int(b0), int(b1),
         workspace.data_ptr(), workspace.numel(), _stream(G.device))


def em_loglik_from_sweep(workspace: torch.Tensor, M: int, N: int, K: int, out: torch.Tensor | None = None):
    """The log-likelihood left by the last em_sweep_loglik in ``workspace`` (device float64)."""
    out = torch.empty((), dtype=torch.float64, device=workspace.device) if out is None else out
    call("adx_em_loglik_from_sweep", workspace.data_ptr(), workspace.numel(), M, N, K, ADX_F64, out.data_ptr(),
         _stream(workspace.device))
    return out


def em_adam_update(P, Q, P32, Q32, mP, vP, mQ, vQ, q_bat, M, t, lr, beta1, beta2, eps, precision,
                   workspace: torch.Tensor) -> None:
    """EM targets + Adam move from the partial sums of the last sweep in ``workspace``."""
    N, K = Q.shape
    call("adx_em_adam_update", M, N, K, precision_code(precision), P.data_ptr(), Q.data_ptr(), _ptr(P32),
         _ptr(Q32), mP.data_ptr(), vP.data_ptr(), mQ.data_ptr(), vQ.data_ptr(), q_bat.data_ptr(), float(t),
         float(lr), float(beta1), float(beta2), float(eps), workspace.data_ptr(), workspace.numel(),
         _stream(P.device))


def em_targets(P, Q, A, B, T, q_bat, P_EM=None, Q_EM=None):
    M, K = P.shape
    N = Q.shape[0]
    for t, n in ((P, "P"), (Q, "Q"), (A, "A"), (B, "B"), (T, "T"), (q_bat, "q_bat")):
        _check(t, n, torch.float64, P.device)
    P_EM = torch.empty_like(P) if P_EM is None else P_EM
    Q_EM = torch.empty_like(Q) if Q_EM is None else Q_EM
    call("adx_em_targets", P.data_ptr(), Q.data_ptr(), A.data_ptr(), B.data_ptr(), T.data_ptr(),
         q_bat.data_ptr(), M, N, K, P_EM.data_ptr(), Q_EM.data_ptr(), _stream(P.device))
    return P_EM, Q_EM


def adam_step(P, Q, P_EM, Q_EM, mP, vP, mQ, vQ, t, lr, beta1, beta2, eps, P32=None, Q32=None):
    M, K = P.shape
    N = Q.shape[0]
    for x, n in ((P, "P"), (Q, "Q"), (P_EM, "P_EM"), (Q_EM, "Q_EM"), (mP, "m_P"), (vP, "v_P"),
                 (mQ, "m_Q"), (vQ, "v_Q")):
        _check(x, n, torch.float64, P.device)
    call("adx_adam_step", P.data_ptr(), Q.data_ptr(), P_EM.data_ptr(), Q_EM.data_ptr(),
         mP.data_ptr(), vP.data_ptr(), mQ.data_ptr(), vQ.data_ptr(), M, N, K, float(t),
         float(lr), float(beta1), float(beta2), float(eps), _ptr(P32), _ptr(Q32), _stream(P.device))


def em_adam_iteration(G, P, Q, P32, Q32, mP, vP, mQ, vQ, q_bat, M, t, lr, beta1, beta2, eps,
                      precision="f32", workspace: torch.Tensor | None = None):
    """One fused Adam-EM iteration (E-step sweep + targets + Adam move), in place."""
    pc = precision_code(precision)
    N, K = Q.shape
    dev = G.device
    ws = workspace if workspace is not None else Workspace.get(dev, em_workspace_bytes(M, N, K, pc))
    call("adx_em_adam_iteration", G.data_ptr(), M, N, K, pc, P.data_ptr(), Q.data_ptr(),
         _ptr(P32), _ptr(Q32), mP.data_ptr(), vP.data_ptr(), mQ.data_ptr(), vQ.data_ptr(),
         q_bat.data_ptr(), float(t), float(lr), float(beta1), float(beta2), float(eps),
         ws.data_ptr(), ws.numel(), _stream(dev))


class EmGraph:
    """``n_iters`` fused Adam-EM iterations (``em_adam_iteration``) captured into one CUDA
    graph by the library. ``launch(t0)`` replays them as steps t0+1 .. t0+n_iters, bit for
    bit the eager iterations. The graph keeps a reference to every tensor it was captured
    with (they must keep their storage: no resizing or reassignment of the buffers), and
    ``workspace`` must be a buffer of its own, not the shared ``Workspace`` cache, which
    may be reallocated."""

    def __init__(self, G, P, Q, P32, Q32, mP, vP, mQ, vQ, q_bat, M, n_iters, lr, beta1, beta2, eps, precision,
                 workspace: torch.Tensor):
        import ctypes

        pc = precision_code(precision)
        N, K = Q.shape
        dev = G.device
        _check(G, "G", torch.uint8)
        for x, n in ((P, "P"), (Q, "Q"), (mP, "m_P"), (vP, "v_P"), (mQ, "m_Q"), (vQ, "v_Q"), (q_bat, "q_bat")):
            _check(x, n, torch.float64, dev)
        if workspace.numel() < em_workspace_bytes(M, N, K, pc):
            raise ValueError("EmGraph: workspace too small")
        self.counter = torch.zeros(1, dtype=torch.float64, device=dev)
        self._keep = (G, P, Q, P32, Q32, mP, vP, mQ, vQ, q_bat, workspace)
        self.n_iters, self.lr, self.device = int(n_iters), float(lr), dev
        h = ctypes.c_void_p(0)
        call("adx_em_graph_create", G.data_ptr(), M, N, K, pc, P.data_ptr(), Q.data_ptr(), _ptr(P32), _ptr(Q32),
             mP.data_ptr(), vP.data_ptr(), mQ.data_ptr(), vQ.data_ptr(), q_bat.data_ptr(), self.n_iters,
             self.lr, float(beta1), float(beta2), float(eps), self.counter.data_ptr(), workspace.data_ptr(),
             workspace.numel(), ctypes.addressof(h))
        self._h = h.value

    def launch(self, t0: int) -> None:
        if not self._h:
            raise RuntimeError("EmGraph: launched after close()")
        call("adx_em_graph_launch", self._h, float(t0), _stream(self.device))

    def close(self) -> None:
        if getattr(self, "_h", None):
            from ._lib import load

            load().adx_em_graph_destroy(self._h)
            self._h = None
            self._keep = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------- batched float64 E-step

class EmBatch:
    """Host-side description of a batch of float64 E-step problems on one cohort (the
    C arrays the batch entry points take) and its partial-sum workspace."""

    def __init__(self, M: int, N: int, Ks, device=None):
        import ctypes

        self.M, self.N = int(M), int(N)
        self.n = len(Ks)
        self.K = (ctypes.c_int * self.n)(*[int(k) for k in Ks])
        nbytes = query_size("adx_em_batch_workspace_bytes", self.M, self.N, self.n, ctypes.addressof(self.K))
        dev = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
        self.workspace = Workspace.get(dev, nbytes, tag="em_batch")

    def sweep(self, Gs, Ps, Qs) -> None:
        """One batched sweep: problem p on packed genotypes Gs[p] with Ps[p], Qs[p] (float64)."""
        import ctypes

        for G, P, Q, k in zip(Gs, Ps, Qs, self.K):
            _check(G, "G", torch.uint8)
            _check(P, "P", torch.float64, G.device)
            _check(Q, "Q", torch.float64, G.device)
            if P.shape != (self.M, k) or Q.shape != (self.N, k) or G.shape != ((self.M + 3) // 4, self.N):
                raise ValueError("G/P/Q shapes do not match the batch")
        gg = (ctypes.c_void_p * self.n)(*[G.data_ptr() for G in Gs])
        pp = (ctypes.c_void_p * self.n)(*[P.data_ptr() for P in Ps])
        qq = (ctypes.c_void_p * self.n)(*[Q.data_ptr() for Q in Qs])
        call("adx_em_sweep_batch", self.M, self.N, self.n, ctypes.addressof(self.K), ctypes.addressof(gg),
             ctypes.addressof(pp), ctypes.addressof(qq), self.workspace.data_ptr(), self.workspace.numel(),
             _stream(Gs[0].device))

    def stats(self, p: int):
        """A, B, T of problem p from the last sweep."""
        import ctypes

        dev = self.workspace.device
        K = self.K[p]
        A = torch.empty((self.M, K), dtype=torch.float64, device=dev)
        B = torch.empty_like(A)
        T = torch.empty((self.N, K), dtype=torch.float64, device=dev)
        call("adx_em_batch_apply", self.M, self.N, self.n, ctypes.addressof(self.K), p, 0, A.data_ptr(),
             B.data_ptr(), T.data_ptr(), None, None, None, None, None, None, None, 1.0, 0.0, 0.0, 0.0, 0.0,
             self.workspace.data_ptr(), self.workspace.numel(), _stream(dev))
        return A, B, T

    def adam(self, p: int, P, Q, mP, vP, mQ, vQ, q_bat, t, lr, beta1, beta2, eps) -> None:
        """EM targets and the Adam move of problem p from the last sweep, in place."""
        import ctypes

        call("adx_em_batch_apply", self.M, self.N, self.n, ctypes.addressof(self.K), p, 1, None, None, None,
             q_bat.data_ptr(), P.data_ptr(), Q.data_ptr(), mP.data_ptr(), vP.data_ptr(), mQ.data_ptr(),
             vQ.data_ptr(), float(t), float(lr), float(beta1), float(beta2), float(eps),
             self.workspace.data_ptr(), self.workspace.numel(), _stream(P.device))


def loglik_device(G: torch.Tensor, P: torch.Tensor, Q: torch.Tensor, M: int, precision="f64",
                  out: torch.Tensor | None = None) -> torch.Tensor:
    """Log-likelihood as a device float64 scalar (no host sync)."""
    pc = precision_code(precision)
    dt = input_dtype(pc)
    _check(G, "G", torch.uint8)
    _check(P, "P", dt, G.device)
    _check(Q, "Q", dt, G.device)
    N, K = Q.shape
    dev = G.device
    out = torch.empty((), dtype=torch.float64, device=dev) if out is None else out
    nbytes = query_size("adx_loglik_workspace_bytes", M, N, K, pc)
    ws = _ll_ws(dev, nbytes)
    call("adx_loglik", G.data_ptr(), M, N, K, pc, P.data_ptr(), Q.data_ptr(), out.data_ptr(),
         ws.data_ptr(), ws.numel(), _stream(dev))
    return out


_LL_WS: dict = {}


def _ll_ws(dev, nbytes):
    key = (dev.type, dev.index)
    buf = _LL_WS.get(key)
    if buf is None or buf.numel() < nbytes:
        buf = torch.empty(max(nbytes, 256), dtype=torch.uint8, device=dev)
        _LL_WS[key] = buf
    return buf


# ---------------------------------------------------------------- reference operator names

_registered = False


def register_reference_ops() -> None:
    """Register the reference's extension operators (same schemas) on the CUDA dispatch key,
    backed by this library: ``pack2bit::unpack2bit_gpu_chunk_uint8``,
    ``pack2bit::unpack2bit_gpu_chunk_center``, ``bvls_kernel::batch_bvls_bpp_cuda``,
    ``sqp_kernel::sqp_solve_q_cuda`` and ``sqp_kernel::sqp_solve_p_cuda``."""
    global _registered
    if _registered:
        return
    lib = torch.library.Library("pack2bit", "DEF")
    lib.define("unpack2bit_gpu_chunk_uint8(Tensor input, int m_start, int chunk_size, int M_total, "
               "int byte_offset, int threads_per_block) -> Tensor")
    lib.define("unpack2bit_gpu_chunk_center(Tensor input, Tensor f, int m_start, int chunk_size, "
               "int M_total, int byte_offset, int threads_per_block) -> Tensor")

    def _u8(inp, m_start, chunk_size, M_total, byte_offset, threads_per_block):
        return unpack_u8(inp.contiguous(), m_start, chunk_size, M_total, byte_offset)

    def _center(inp, f, m_start, chunk_size, M_total, byte_offset, threads_per_block):
        return unpack_center(inp.contiguous(), f.contiguous(), m_start, chunk_size, M_total, byte_offset)

    lib.impl("unpack2bit_gpu_chunk_uint8", _u8, "CUDA")
    lib.impl("unpack2bit_gpu_chunk_center", _center, "CUDA")

    # bvls_kernel.cu:224-230 and sqp_kernel.cu:377-385
    blib = torch.library.Library("bvls_kernel", "DEF")
    blib.define("batch_bvls_bpp_cuda(Tensor A, Tensor B, float lower, float upper) -> Tensor")
    blib.impl("batch_bvls_bpp_cuda",
              lambda A, B, lower, upper: bvls(A.contiguous(), B.contiguous(), lower, upper), "CUDA")
    slib = torch.library.Library("sqp_kernel", "DEF")
    slib.define("sqp_solve_q_cuda(Tensor XtX_q, Tensor Xtz_q, Tensor Q, Tensor v_kk, int N, int K) -> Tensor")
    slib.define("sqp_solve_p_cuda(Tensor XtX_p, Tensor Xtz_p, Tensor P, int M, int K) -> Tensor")
    slib.impl("sqp_solve_q_cuda", lambda H, g, Q, v, N, K: sqp_solve_q(
        H.contiguous(), g.contiguous(), Q.contiguous(), v.contiguous(), N, K), "CUDA")
    slib.impl("sqp_solve_p_cuda", lambda H, g, P, M, K: sqp_solve_p(
        H.contiguous(), g.contiguous(), P.contiguous(), M, K), "CUDA")
    register_reference_ops._lib = (lib, blib, slib)  # keep the registrations alive
    _registered = True


# ---------------------------------------------------------------- initialisation

def rsvd_rows(G: torch.Tensor, f: torch.Tensor, B: torch.Tensor, M: int,
              out: torch.Tensor | None = None) -> torch.Tensor:
    """``Xc @ B`` for the centred genotypes (float32 ``[M, L]``), B float32 ``[N, L]``."""
    _check(G, "G", torch.uint8)
    _check(f, "f", torch.float32, G.device)
    _check(B, "B", torch.float32, G.device)
    N, L = B.shape
    Y = torch.empty((M, L), dtype=torch.float32, device=G.device) if out is None else out
    _check(Y, "out", torch.float32, G.device)
    call("adx_rsvd_rows", G.data_ptr(), M, N, f.data_ptr(), B.data_ptr(), L, Y.data_ptr(),
         _stream(G.device))
    return Y


def rsvd_cols(G: torch.Tensor, f: torch.Tensor, Y: torch.Tensor, M: int,
              out: torch.Tensor | None = None, accumulate: bool = False) -> torch.Tensor:
    """``Xc.T @ Y`` (float32 ``[N, L]``; added to ``out`` when ``accumulate``)."""
    _check(G, "G", torch.uint8)
    _check(f, "f", torch.float32, G.device)
    _check(Y, "Y", torch.float32, G.device)
    N = G.shape[1]
    L = Y.shape[1]
    Z = torch.empty((N, L), dtype=torch.float32, device=G.device) if out is None else out
    _check(Z, "out", torch.float32, G.device)
    nb = query_size("adx_rsvd_workspace_bytes", M, N, L)
    ws = Workspace.get(G.device, nb, "rsvd")
    call("adx_rsvd_cols", G.data_ptr(), M, N, f.data_ptr(), Y.data_ptr(), L, int(bool(accumulate)),
         Z.data_ptr(), ws.data_ptr(), ws.numel(), _stream(G.device))
    return Z


def bvls(A: torch.Tensor, B: torch.Tensor, lower: float, upper: float) -> torch.Tensor:
    """Row-batched bounded least squares (float64): ``argmin 1/2 x'Ax - b'x`` in the box."""
    _check(A, "A", torch.float64)
    _check(B, "B", torch.float64, A.device)
    M, K = B.shape
    if A.shape != (K, K):
        raise ValueError("A must be K x K")
    X = torch.empty_like(B)
    call("adx_bvls", A.data_ptr(), B.data_ptr(), M, K, float(lower), float(upper), X.data_ptr(),
         _stream(A.device))
    return X


# ---------------------------------------------------------------- original ADMIXTURE (BR-QN)

def grad_hess_q(G: torch.Tensor, P: torch.Tensor, Q: torch.Tensor, M: int, XtX_q=None, Xtz_q=None):
    _check(G, "G", torch.uint8)
    _check(P, "P", torch.float64, G.device)
    _check(Q, "Q", torch.float64, G.device)
    N, K = Q.shape
    XtX_q = torch.empty((N, K, K), dtype=torch.float64, device=G.device) if XtX_q is None else XtX_q
    Xtz_q = torch.empty((N, K), dtype=torch.float64, device=G.device) if Xtz_q is None else Xtz_q
    call("adx_grad_hess_q", G.data_ptr(), M, N, K, P.data_ptr(), Q.data_ptr(), XtX_q.data_ptr(),
         Xtz_q.data_ptr(), _stream(G.device))
    return XtX_q, Xtz_q


def grad_hess_p(G: torch.Tensor, P: torch.Tensor, Q: torch.Tensor, M: int, XtX_p=None, Xtz_p=None):
    _check(G, "G", torch.uint8)
    _check(P, "P", torch.float64, G.device)
    _check(Q, "Q", torch.float64, G.device)
    N, K = Q.shape
    XtX_p = torch.empty((M, K, K), dtype=torch.float64, device=G.device) if XtX_p is None else XtX_p
    Xtz_p = torch.empty((M, K), dtype=torch.float64, device=G.device) if Xtz_p is None else Xtz_p
    call("adx_grad_hess_p", G.data_ptr(), M, N, K, P.data_ptr(), Q.data_ptr(), XtX_p.data_ptr(),
         Xtz_p.data_ptr(), _stream(G.device))
    return XtX_p, Xtz_p


def sqp_solve_q(XtX_q: torch.Tensor, Xtz_q: torch.Tensor, Q: torch.Tensor, v_kk: torch.Tensor,
                N: int, K: int) -> torch.Tensor:
    """Same contract as ``sqp_kernel::sqp_solve_q_cuda`` (Xtz_q already negated)."""
    for t, nm in ((XtX_q, "XtX_q"), (Xtz_q, "Xtz_q"), (Q, "Q"), (v_kk, "v_kk")):
        _check(t, nm, torch.float64, Q.device)
    out = torch.empty((N, K), dtype=torch.float64, device=Q.device)
    call("adx_sqp_q", XtX_q.data_ptr(), Xtz_q.data_ptr(), Q.data_ptr(), v_kk.data_ptr(), N, K,
         out.data_ptr(), _stream(Q.device))
    return out


def sqp_solve_p(XtX_p: torch.Tensor, Xtz_p: torch.Tensor, P: torch.Tensor, M: int, K: int) -> torch.Tensor:
    """Same contract as ``sqp_kernel::sqp_solve_p_cuda`` (Xtz_p already negated)."""
    for t, nm in ((XtX_p, "XtX_p"), (Xtz_p, "Xtz_p"), (P, "P")):
        _check(t, nm, torch.float64, P.device)
    out = torch.empty((M, K), dtype=torch.float64, device=P.device)
    call("adx_sqp_p", XtX_p.data_ptr(), Xtz_p.data_ptr(), P.data_ptr(), M, K, out.data_ptr(),
         _stream(P.device))
    return out


def project_simplex_(Q: torch.Tensor) -> torch.Tensor:
    """Project float64 Q rows onto {q >= 1e-5, sum q = 1} in place."""
    _check(Q, "Q", torch.float64)
    call("adx_project_simplex", Q.data_ptr(), Q.shape[0], Q.shape[1], _stream(Q.device))
    return Q


def project_box_(P: torch.Tensor) -> torch.Tensor:
    """Clamp float64 P into [1e-5, 1 - 1e-5] in place."""
    _check(P, "P", torch.float64)
    call("adx_project_box", P.data_ptr(), P.shape[0], P.shape[1], _stream(P.device))
    return P


# ---------------------------------------------------------------- cross-validation

def masked_copy(G: torch.Tensor) -> torch.Tensor:
    """A copy of packed G in a buffer padded to whole 32-bit words (the masking kernels
    hide entries with 32-bit atomics); returns the [rows, N] view."""
    _check(G, "G", torch.uint8)
    n = G.numel()
    buf = torch.empty(((n + 3) // 4) * 4, dtype=torch.uint8, device=G.device)
    view = buf[:n].view(G.shape)
    view.copy_(G)
    return view


def _padded_bytes(Gm: torch.Tensor) -> int:
    return Gm.untyped_storage().nbytes() - Gm.storage_offset()


def cv_mask_list(Gm: torch.Tensor, M: int, idx: torch.Tensor) -> None:
    """Hide the entries at flat indices ``idx`` (int64, j*N + i) in the masked copy ``Gm``."""
    _check(idx, "idx", torch.int64, Gm.device)
    ws = Workspace.get(Gm.device, query_size("adx_cv_workspace_bytes"), "cv")
    call("adx_cv_mask_list", Gm.data_ptr(), _padded_bytes(Gm) // 4 * 4, M, Gm.shape[1], idx.data_ptr(),
         idx.numel(), ws.data_ptr(), ws.numel(), _stream(Gm.device))


def cv_mask_hash(Gm: torch.Tensor, G0: torch.Tensor, M: int, seed: int, n_folds: int, fold: int) -> None:
    """Hide fold ``fold`` of the hash rule (observed entries of ``G0``) in ``Gm``."""
    call("adx_cv_mask_hash", Gm.data_ptr(), _padded_bytes(Gm) // 4 * 4, G0.data_ptr(), M, G0.shape[1],
         int(seed) & 0xFFFFFFFFFFFFFFFF, n_folds, fold, _stream(Gm.device))


def cv_deviance_list(G0, P, Q, M, idx) -> float:
    ws = Workspace.get(G0.device, query_size("adx_cv_workspace_bytes"), "cv")
    out = torch.empty(1, dtype=torch.float64, device=G0.device)
    call("adx_cv_deviance_list", G0.data_ptr(), M, G0.shape[1], Q.shape[1], P.data_ptr(), Q.data_ptr(),
         idx.data_ptr(), idx.numel(), out.data_ptr(), ws.data_ptr(), ws.numel(), _stream(G0.device))
    return float(out.item())


def cv_deviance_hash(G0, P, Q, M, seed, n_folds, fold) -> float:
    ws = Workspace.get(G0.device, query_size("adx_cv_workspace_bytes"), "cv")
    out = torch.empty(1, dtype=torch.float64, device=G0.device)
    call("adx_cv_deviance_hash", G0.data_ptr(), M, G0.shape[1], Q.shape[1], P.data_ptr(), Q.data_ptr(),
         int(seed) & 0xFFFFFFFFFFFFFFFF, n_folds, fold, out.data_ptr(), ws.data_ptr(), ws.numel(),
         _stream(G0.device))
    return float(out.item())
