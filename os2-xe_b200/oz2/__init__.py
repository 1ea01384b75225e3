"""Python binding of liboz2.so, the B200-native Ozaki Scheme II FP64 GEMM emulator.

Mirrors the reference's C++ class oz2::Ozaki2 (MacraMacra/OS2-Xe, src/ozaki2_gpu.hpp:678-1188):
the same member names, argument meaning and error behaviour. Reference exceptions map to
Python ones: std::invalid_argument -> ValueError, std::runtime_error -> RuntimeError
(MemoryError when the workspace does not fit), std::overflow_error -> OverflowError.

Matrices are column-major device buffers: a torch CUDA tensor (its data_ptr is used) or a raw
integer device address. This module calls only the C ABI; it has no CPU fallback and raises
ImportError when the library is missing.
"""
import ctypes as C
import os
from dataclasses import dataclass

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboz2.so")

OK, EINVAL, ENOMEM, EINTERNAL, ETIMEOUT, EOVERFLOW, ECUDA = range(7)
K_MAX_MODULI = 24
K_MAX_MODULI_EXT = 32  # the adaptive path's extended sets (s = 25..32, no counterpart in the reference)
NATIVE_S = 33  # adaptive s of a tile run as a native FP64 GEMM

if not os.path.exists(LIB_PATH):
    raise ImportError(f"{LIB_PATH} is not built: run python os2-xe_b200/build.py")
_lib = C.CDLL(LIB_PATH)

_i64, _i32, _dbl, _vp, _chr, _sz = C.c_int64, C.c_int, C.c_double, C.c_void_p, C.c_char, C.c_size_t
_lib.oz2_create.argtypes = [_vp, C.POINTER(_vp)]
_lib.oz2_destroy.argtypes = [_vp]
_lib.oz2_set_stream.argtypes = [_vp, _vp]
_lib.oz2_dgemm.argtypes = [_vp, _chr, _chr, _i64, _i64, _i64, _dbl, _vp, _i64, _vp, _i64, _dbl, _vp, _i64, _i32,
                           _vp, _i32, _vp]
_lib.oz2_zgemm.argtypes = [_vp, _chr, _chr, _i64, _i64, _i64, _vp, _vp, _i64, _vp, _i64, _vp, _vp, _i64, _i32,
                           _vp, _i32, _vp]
_lib.oz2_ozaki1_dgemm.argtypes = [_vp, _i64, _i64, _i64, _vp, _i64, _vp, _i64, _vp, _i64, _i32]
_lib.oz2_precision_bits.argtypes = [_i64, _i32, C.POINTER(_i32)]
_lib.oz2_precision_bits_complex.argtypes = [_i64, _i32, C.POINTER(_i32)]
_lib.oz2_moduli_for_bits.argtypes = [_i64, _i32, C.POINTER(_i32)]
_lib.oz2_set_workspace_limit.argtypes = [_vp, _sz]
_lib.oz2_set_resident_hint.argtypes = [_vp, _sz]
_lib.oz2_release_workspace.argtypes = [_vp]
_lib.oz2_set_profiling.argtypes = [_vp, _i32]
_lib.oz2_stage_times.argtypes = [_vp, C.POINTER(_dbl)]
_lib.oz2_last_tiling.argtypes = [_vp, C.POINTER(_i64)]
_lib.oz2_set_tuning.argtypes = [_vp, _i32, _i32, _i32]
_lib.oz2_check_device_error.argtypes = [_vp]
_lib.oz2_set_failure_test.argtypes = [_i64, _i32]
_lib.oz2_set_split_kernel.argtypes = [_i32]
_lib.oz2_set_crt_kernel.argtypes = [_i32]
_lib.oz2_set_scale_fusion.argtypes = [_i32]
_lib.oz2_set_crt_fusion.argtypes = [_i32]


class DgemmProblem(C.Structure):
    """oz2_dgemm_problem of include/oz2/oz2.h"""
    _fields_ = [("ta", _chr), ("tb", _chr), ("num_moduli", _i32), ("m", _i64), ("n", _i64), ("k", _i64),
                ("alpha", _dbl), ("beta", _dbl), ("A", _vp), ("lda", _i64), ("B", _vp), ("ldb", _i64), ("C", _vp),
                ("ldc", _i64)]


_lib.oz2_dgemm_grouped.argtypes = [_vp, _i32, C.POINTER(DgemmProblem), _vp, _i32, _vp]
_lib.oz2_set_graph_mode.argtypes = [_vp, _i32]
_lib.oz2_kernel_launches.argtypes = [_vp, C.POINTER(_i64)]
_lib.oz2_accuracy.argtypes = [_vp, _i64, _i64, _vp, _i64, _vp, _vp, C.POINTER(_dbl), C.POINTER(_i64)]
_lib.oz2_set_gemm_config.argtypes = [_vp, _i32, _i32, _i32]
_lib.oz2_get_gemm_config.argtypes = [_vp, C.POINTER(_i32)]
_lib.oz2_autotune_grouped.argtypes = [_vp, _i32, C.POINTER(DgemmProblem), C.POINTER(_i32)]
_lib.oz2_dgemm_adaptive.argtypes = [_vp, _i32, C.POINTER(DgemmProblem), _i32, _i32, C.POINTER(_i64)]
_lib.oz2_set_adaptive_options.argtypes = [_vp, _i32, C.c_float]
_lib.oz2_adaptive_stage_times.argtypes = [_vp, C.POINTER(_dbl)]
_lib.oz2_adaptive_gemm_bytes.argtypes = [_vp, C.POINTER(_i64)]
_lib.oz2_set_probe_kind.argtypes = [_vp, _i32]
_lib.oz2_mlp_info.argtypes = [C.POINTER(_i32)]
_lib.oz2_mlp_set_weights.argtypes = [_vp, _vp, _i32]
_lib.oz2_mlp_train.argtypes = [_vp, _i32, _vp, _vp, _i32, C.c_float, C.c_uint, _vp, _vp]
_lib.oz2_mlp_infer.argtypes = [_vp, _vp, _i32, _vp, C.c_float, _vp, _vp]
_lib.oz2_tile_features.argtypes = [_vp, _i32, C.POINTER(DgemmProblem), _i32, _vp, _vp, C.POINTER(_i64)]
_lib.oz2_dd_reference.argtypes = [_vp, _i64, _i64, _i64, _vp, _i64, _vp, _i64, _vp, _vp, _vp]
_lib.oz2_error_ratio.argtypes = [_vp, _i64, _i64, _i64, _vp, _i64, _vp, _vp, _vp, _i32, C.POINTER(C.c_float)]
_lib.oz2_last_error.argtypes = [_vp]
_lib.oz2_last_error.restype = C.c_char_p
_lib.oz2_status_string.argtypes = [_i32]
_lib.oz2_status_string.restype = C.c_char_p


def lib():
    """The loaded ctypes library (for callers that bind further entry points)."""
    return _lib


def set_failure_test(wait_limit_ns=0, stall_mma=False):
    """Failure-path test of the INT8 GEMM's bounded waits (process-wide): wait_limit_ns bounds
    every wait (0 = the 2 s default); with stall_mma the MMA issuer issues nothing, so the waits
    run out and check_device_error raises TimeoutError. set_failure_test() restores normal runs."""
    _raise(_lib.oz2_set_failure_test(int(wait_limit_ns), 1 if stall_mma else 0))


S_ADAPTIVE = -1  # num_moduli of a grouped problem that takes the adaptive s per tile

SPLIT_DP4A = 0
SPLIT_TENSOR_CORE = 1


SPLIT_DEFAULT = SPLIT_DP4A


def set_split_kernel(kind):
    """Kernel of the real split (process-wide): SPLIT_DP4A (default, integer pipe) or
    SPLIT_TENSOR_CORE (the residues' byte dot products as one tcgen05 u8 x u8 MMA per 512
    elements; measured slower). Both write identical planes."""
    _raise(_lib.oz2_set_split_kernel(int(kind)))


CRT_DP2A = 0
CRT_TENSOR_CORE = 1
CRT_AUTO = 2


CRT_DEFAULT = CRT_AUTO


def set_crt_kernel(kind):
    """Kernel of the real CRT (process-wide): CRT_AUTO (default; the tensor-core CRT for 7- and
    8-limb plans, s = 26..32, dp2a below), CRT_TENSOR_CORE (limb sums as one tcgen05 u8 x u8 MMA per 128
    entries) or CRT_DP2A. All produce identical C."""
    _raise(_lib.oz2_set_crt_kernel(int(kind)))


def set_scale_fusion(on):
    """Scale pass fused into the split for real operands with k <= 2048 (1024 when the plane rows
    are contiguous), process-wide, default off (measured no faster). Results are identical."""
    _raise(_lib.oz2_set_scale_fusion(1 if on else 0))


def set_crt_fusion(on):
    """CRT in the GEMM's epilogue for real problems with s <= 8 and k <= 65408 (process-wide,
    default off: measured slower): the residues stay in tensor memory and the GEMM writes C.
    Results are identical."""
    _raise(_lib.oz2_set_crt_fusion(1 if on else 0))


def mlp_info():
    out = (_i32 * 4)()
    _raise(_lib.oz2_mlp_info(out))
    return {"params": out[0], "features": out[1], "classes": out[2], "hidden": out[3]}


def _raise(status, handle=None):
    if status == OK:
        return
    msg = (_lib.oz2_last_error(handle) or b"").decode() or _lib.oz2_status_string(status).decode()
    if status == EINVAL:
        raise ValueError(msg)
    if status == EOVERFLOW:
        raise OverflowError(msg)
    if status == ENOMEM:
        raise MemoryError(msg)
    if status == ETIMEOUT:
        raise TimeoutError(msg)
    raise RuntimeError(msg)


def _addr(x):
    if x is None:
        return None
    if isinstance(x, int):
        return x
    return x.data_ptr()


def _op(t):
    t = t.value if isinstance(t, Trans) else t
    return t.encode() if isinstance(t, str) else t


class Trans:
    """op(X): N, T or C (conjugate transpose; equals T for gemm)."""

    def __init__(self, value):
        self.value = value


Trans.N, Trans.T, Trans.C = Trans("N"), Trans("T"), Trans("C")


@dataclass
class StageTimes:
    scale_ms: float = 0.0
    split_ms: float = 0.0
    gemm_ms: float = 0.0
    crt_ms: float = 0.0

    def total_ms(self):
        return self.scale_ms + self.split_ms + self.gemm_ms + self.crt_ms


@dataclass
class TileInfo:
    mb: int = 0
    nb: int = 0
    pm: int = 0
    pn: int = 0
    k_chunks: int = 0
    workspace_bytes: int = 0


@dataclass
class Tuning:
    batched_gemm: bool = True
    pad_lda: bool = True
    pow2_tiles: bool = True


class Ozaki2:
    """Binds to a CUDA stream (a torch.cuda.Stream, a raw cudaStream_t int, or None for the
    current torch stream / the legacy default stream). Not thread-safe: one object per stream."""

    def __init__(self, stream=None, profiling=False):
        self._h = _vp()
        _raise(_lib.oz2_create(self._stream_ptr(stream), C.byref(self._h)))
        self._tuning = Tuning()
        if profiling:
            self.set_profiling(True)

    @staticmethod
    def _stream_ptr(stream):
        if stream is None:
            try:
                import torch
                if torch.cuda.is_available():
                    return torch.cuda.current_stream().cuda_stream
            except ImportError:
                pass
            return None
        if isinstance(stream, int):
            return stream
        return stream.cuda_stream

    def close(self):
        if self._h:
            _lib.oz2_destroy(self._h)
            self._h = _vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h.value

    def set_stream(self, stream):
        _raise(_lib.oz2_set_stream(self._h, self._stream_ptr(stream)), self._h)

    # ---- static planning (ref src/ozaki2_gpu.hpp:689-700, :762)
    @staticmethod
    def precision_bits(k, num_moduli):
        out = _i32()
        _raise(_lib.oz2_precision_bits(k, num_moduli, C.byref(out)))
        return out.value

    @staticmethod
    def precision_bits_complex(k, num_moduli):
        out = _i32()
        _raise(_lib.oz2_precision_bits_complex(k, num_moduli, C.byref(out)))
        return out.value

    @staticmethod
    def moduli_for_bits(k, bits):
        out = _i32()
        _raise(_lib.oz2_moduli_for_bits(k, bits, C.byref(out)))
        return out.value

    # ---- workspace and tuning (ref :702-714)
    def set_workspace_limit(self, nbytes):
        _raise(_lib.oz2_set_workspace_limit(self._h, nbytes), self._h)

    def set_resident_hint(self, nbytes):
        _raise(_lib.oz2_set_resident_hint(self._h, nbytes), self._h)

    def release_workspace(self):
        _raise(_lib.oz2_release_workspace(self._h), self._h)

    def set_tuning(self, t):
        self._tuning = t
        _raise(_lib.oz2_set_tuning(self._h, int(t.batched_gemm), int(t.pad_lda), int(t.pow2_tiles)), self._h)

    def tuning(self):
        return self._tuning

    def set_profiling(self, on):
        _raise(_lib.oz2_set_profiling(self._h, int(bool(on))), self._h)

    def stage_times(self):
        out = (_dbl * 4)()
        _raise(_lib.oz2_stage_times(self._h, out), self._h)
        return StageTimes(*list(out))

    def last_tiling(self):
        out = (_i64 * 6)()
        _raise(_lib.oz2_last_tiling(self._h, out), self._h)
        return TileInfo(*list(out))

    def check_device_error(self):
        _raise(_lib.oz2_check_device_error(self._h), self._h)

    # ---- grouped calls (no counterpart in the reference)
    @staticmethod
    def _problems(problems):
        arr = (DgemmProblem * len(problems))()
        for i, p in enumerate(problems):
            ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C_, ldc, s = p
            arr[i] = DgemmProblem(_op(ta), _op(tb), s, m, n, k, float(alpha), float(beta), _addr(A), lda, _addr(B),
                                  ldb, _addr(C_), ldc)
        return arr

    def gemm_grouped(self, problems, deps=None, done=None):
        """problems: sequence of (ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, num_moduli),
        the arguments of gemm() per problem; all run in one set of launches. num_moduli = S_ADAPTIVE
        (-1) gives that problem the adaptive s per tile (gemm_adaptive, mode 0, 53-bit target)."""
        arr = self._problems(problems)
        ev, nev = self._events(deps)
        d = done.cuda_event if hasattr(done, "cuda_event") else done
        _raise(_lib.oz2_dgemm_grouped(self._h, len(problems), arr, ev, nev, d), self._h)

    def kernel_launches(self):
        """kernels launched through this handle so far (graph replays count their kernel nodes)"""
        out = _i64()
        _raise(_lib.oz2_kernel_launches(self._h, C.byref(out)), self._h)
        return out.value

    def set_graph_mode(self, on):
        _raise(_lib.oz2_set_graph_mode(self._h, int(bool(on))), self._h)

    def set_gemm_config(self, bn=0, group_j=16, ctas=0):
        _raise(_lib.oz2_set_gemm_config(self._h, bn, group_j, ctas), self._h)

    def gemm_config(self):
        out = (_i32 * 3)()
        _raise(_lib.oz2_get_gemm_config(self._h, out), self._h)
        return {"bn": out[0], "group_j": out[1], "ctas": out[2]}

    def autotune_grouped(self, problems):
        out = (_i32 * 3)()
        _raise(_lib.oz2_autotune_grouped(self._h, len(problems), self._problems(problems), out), self._h)
        return {"bn": out[0], "group_j": out[1], "ctas": out[2]}

    # ---- adaptive number of moduli per tile (no counterpart in the reference)
    ADAPTIVE_MLP, ADAPTIVE_ANALYTIC_TILE, ADAPTIVE_ANALYTIC_PROBLEM, ADAPTIVE_FIXED = 0, 1, 2, 3
    ADAPTIVE_CERTIFIED_TILE, ADAPTIVE_CERTIFIED_PROBLEM = 4, 5

    def gemm_adaptive(self, problems, target_bits=53, mode=0):
        """problems as for gemm_grouped (num_moduli is used by mode 3 only). Returns the stats
        dict: tiles, sum_s (emulated tiles, reruns included), probed, rerun, rerun_sum_s,
        analytic_sum_s (the arbiter's s summed: the analytic s, or in modes 0, 4 and 5 the smaller of
        the analytic and certified s; 33 counts a native tile), mlp, int8_macs (sum of s m_t n_t k
        over emulated tiles), native_tiles, native_macs (tiles run as native FP64 GEMMs)."""
        arr = self._problems(problems)
        st = (_i64 * 10)()
        _raise(_lib.oz2_dgemm_adaptive(self._h, len(problems), arr, target_bits, mode, st), self._h)
        keys = ["tiles", "sum_s", "probed", "rerun", "rerun_sum_s", "analytic_sum_s", "mlp", "int8_macs",
                "native_tiles", "native_macs"]
        return dict(zip(keys, list(st)))

    def adaptive_stage_times(self):
        """with profiling on: {probe_ms, native_ms} of the last gemm_adaptive"""
        out = (_dbl * 2)()
        _raise(_lib.oz2_adaptive_stage_times(self._h, out), self._h)
        return {"probe_ms": out[0], "native_ms": out[1]}

    def adaptive_gemm_bytes(self):
        """{plane_bytes, residue_bytes, batches} of the last gemm_adaptive's INT8 GEMM launches"""
        out = (_i64 * 3)()
        _raise(_lib.oz2_adaptive_gemm_bytes(self._h, out), self._h)
        return {"plane_bytes": out[0], "residue_bytes": out[1], "batches": out[2]}

    PROBE_COLUMNS, PROBE_FREIVALDS, PROBE_BOTH, PROBE_NONE = 0, 1, 2, 3

    def set_probe_kind(self, kind):
        """mode 0's probe: PROBE_COLUMNS (8 columns entry by entry), PROBE_FREIVALDS (C x against
        alpha A (B x) in double-double, two random vectors), PROBE_BOTH, or PROBE_NONE (the MLP's s
        unchecked: for measuring what the probes catch)"""
        _raise(_lib.oz2_set_probe_kind(self._h, int(kind)), self._h)

    def set_adaptive_options(self, tile=512, threshold=0.9):
        _raise(_lib.oz2_set_adaptive_options(self._h, tile, threshold), self._h)
        self._tile = tile

    def set_mlp_weights(self, params):
        """params: sequence of floats (oz2_mlp_info()[0] of them), or None to unload"""
        if params is None:
            _raise(_lib.oz2_mlp_set_weights(self._h, None, 0), self._h)
            return
        buf = (C.c_float * len(params))(*params)
        _raise(_lib.oz2_mlp_set_weights(self._h, buf, len(params)), self._h)

    def load_model(self, path=None):
        """loads an MLP saved by oz2.adaptive.save_model (default: the model shipped with the package)"""
        from . import adaptive
        model = adaptive.load_model(path)
        self.set_mlp_weights(model["params"])
        self.set_adaptive_options(model.get("tile", 512), model.get("threshold", 0.9))
        return model

    def tile_features(self, problems, target_bits=53):
        """features (torch float32 [tiles, F]) and analytic s (torch int32 [tiles]) on the device"""
        import torch
        arr = self._problems(problems)
        T = getattr(self, "_tile", 512)
        ntiles = sum(((p[2] + T - 1) // T) * ((p[3] + T - 1) // T) for p in problems)
        F = mlp_info()["features"]
        feat = torch.zeros((max(ntiles, 1), F), dtype=torch.float32, device="cuda")
        sa = torch.zeros(max(ntiles, 1), dtype=torch.int32, device="cuda")
        n = _i64()
        _raise(_lib.oz2_tile_features(self._h, len(problems), arr, target_bits, feat.data_ptr(), sa.data_ptr(),
                                      C.byref(n)), self._h)
        return feat[: n.value], sa[: n.value]

    def dd_reference(self, m, n, k, A, lda, B, ldb, hi, lo, absab):
        _raise(_lib.oz2_dd_reference(self._h, m, n, k, _addr(A), lda, _addr(B), ldb, _addr(hi), _addr(lo),
                                     _addr(absab)), self._h)

    def accuracy(self, m, n, C_, ldc, hi, lo):
        """(max error in ulps of the correctly rounded value, entries correctly rounded) of C
        against the double-double product hi + lo"""
        u, c = _dbl(), _i64()
        _raise(_lib.oz2_accuracy(self._h, m, n, _addr(C_), ldc, _addr(hi), _addr(lo), C.byref(u), C.byref(c)),
               self._h)
        return u.value, c.value

    def error_ratio(self, m, n, k, C_, ldc, hi, lo, absab, target_bits=53):
        out = C.c_float()
        _raise(_lib.oz2_error_ratio(self._h, m, n, k, _addr(C_), ldc, _addr(hi), _addr(lo), _addr(absab),
                                    target_bits, C.byref(out)), self._h)
        return out.value

    def mlp_train(self, features, labels, params, epochs=300, lr=3e-3, seed=1):
        """trains in place: features torch float32 [N, F] and labels int32 [N] on the device,
        params a list of floats; returns (params, per-epoch losses)"""
        p = (C.c_float * len(params))(*params)
        loss = (C.c_float * epochs)()
        _raise(_lib.oz2_mlp_train(self._h, features.shape[0], features.data_ptr(), labels.data_ptr(), epochs, lr,
                                  seed, p, loss), self._h)
        return list(p), list(loss)

    def mlp_infer(self, params, features, threshold=0.9, probs=False):
        import torch
        p = (C.c_float * len(params))(*params)
        n = features.shape[0]
        s = torch.zeros(n, dtype=torch.int32, device="cuda")
        pr = torch.zeros((n, mlp_info()["classes"]), dtype=torch.float32, device="cuda") if probs else None
        _raise(_lib.oz2_mlp_infer(self._h, p, n, features.data_ptr(), threshold, s.data_ptr(),
                                  pr.data_ptr() if probs else None), self._h)
        return (s, pr) if probs else s

    # ---- the products (ref :739-786)
    @staticmethod
    def _events(deps):
        if not deps:
            return None, 0
        arr = (_vp * len(deps))(*[d.cuda_event if hasattr(d, "cuda_event") else d for d in deps])
        return arr, len(deps)

    def gemm(self, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C_, ldc, num_moduli, deps=None, done=None):
        ev, nev = self._events(deps)
        d = done.cuda_event if hasattr(done, "cuda_event") else done
        _raise(_lib.oz2_dgemm(self._h, _op(ta), _op(tb), m, n, k, float(alpha), _addr(A), lda, _addr(B), ldb,
                              float(beta), _addr(C_), ldc, num_moduli, ev, nev, d), self._h)

    def ozaki1(self, m, n, k, A, lda, B, ldb, C_, ldc, L):
        """C = A B by Ozaki Scheme I with L 7-bit digits (7 L - 2 bits per element), the
        reference's comparison baseline oz1::Ozaki1::gemm (benchmarks/ozaki1_gpu.hpp:85-147):
        column-major, untransposed, no alpha / beta"""
        _raise(_lib.oz2_ozaki1_dgemm(self._h, m, n, k, _addr(A), lda, _addr(B), ldb, _addr(C_), ldc, L), self._h)

    def zgemm(self, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C_, ldc, num_moduli, deps=None, done=None):
        alpha, beta = complex(alpha), complex(beta)
        al = (_dbl * 2)(alpha.real, alpha.imag)
        be = (_dbl * 2)(beta.real, beta.imag)
        ev, nev = self._events(deps)
        d = done.cuda_event if hasattr(done, "cuda_event") else done
        _raise(_lib.oz2_zgemm(self._h, _op(ta), _op(tb), m, n, k, al, _addr(A), lda, _addr(B), ldb, be, _addr(C_),
                              ldc, num_moduli, ev, nev, d), self._h)
