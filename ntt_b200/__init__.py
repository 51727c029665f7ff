"""ntt_b200 -- RNS negacyclic NTT / INTT on NVIDIA B200 (sm_100a).

Python host side over the C ABI of ``libntt_b200.so`` (include/ntt_b200.h).
It mirrors the reference's interface for this path (vnny27/NTT):

* ``ModulusConfig``, ``PhaseConfig``, ``TransformConfig`` -- src/ntt_config.h:6-29
* ``default_moduli()``, ``default_transform(logN)`` -- src/ntt_config.h:62-94
* ``modulus_runtime(logN, cfg)`` -- make_modulus_runtime, src/v04_montgomery.cu:681-718
* ``twiddle_table(logN, q, root)`` -- make_twiddle_table, v04:720-727
* ``launch_ntt(...)`` / ``launch_intt(...)`` -- launch_ntt<LC> / launch_intt<LC>,
  v04:603-658 (same arguments: caller-owned device buffers and the reference's
  Montgomery-form tables)

plus the native ``Plan`` (device-resident Shoup tables, fused cluster
kernels), the batch / multiply / serving layers and the autotuner.

Device buffers can be passed as torch CUDA tensors (int32 or uint32) or raw
integer device addresses; streams as ``torch.cuda.Stream``, raw handles or
None (legacy default stream).  There is no CPU fallback: every call goes
through the compiled library, and importing fails loudly if it is missing.
"""
from __future__ import annotations

import ctypes
import os
from typing import Iterable, List, Optional, Sequence

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libntt_b200.so")

if not os.path.exists(LIB_PATH):
    raise ImportError(
        f"ntt_b200: compiled library {LIB_PATH} is missing; build it with "
        "`make -C ntt_b200` (or __graft_entry__.build())")

_lib = ctypes.CDLL(LIB_PATH)

# ---------------------------------------------------------------------------
# C types
# ---------------------------------------------------------------------------


class ModulusConfig(ctypes.Structure):
    """src/ntt_config.h:6-9"""
    _fields_ = [("qi", ctypes.c_uint32), ("primitive_root", ctypes.c_uint32)]

    def __iter__(self):
        yield self.qi
        yield self.primitive_root

    def __repr__(self):
        return f"ModulusConfig({self.qi}, {self.primitive_root})"


class PhaseConfig(ctypes.Structure):
    """src/ntt_config.h:12-16"""
    _fields_ = [("radix_stages", ctypes.c_int), ("stage_merging", ctypes.c_int),
                ("warp_batching", ctypes.c_int)]

    def as_tuple(self):
        return (self.radix_stages, self.stage_merging, self.warp_batching)

    def __repr__(self):
        return f"PhaseConfig{self.as_tuple()}"


class TransformConfig(ctypes.Structure):
    """src/ntt_config.h:18-23"""
    _fields_ = [("ntt_phase1", PhaseConfig), ("ntt_phase2", PhaseConfig),
                ("intt_phase1", PhaseConfig), ("intt_phase2", PhaseConfig)]


class ModulusRuntime(ctypes.Structure):
    """src/v04_montgomery.cu:17-26"""
    _fields_ = [(n, ctypes.c_uint32) for n in (
        "qi", "primitive_root", "q_inv", "r2", "psi", "psi_inv", "omega", "degree_inv")]


class PlanInfo(ctypes.Structure):
    _fields_ = [("logN", ctypes.c_int), ("limbs", ctypes.c_int), ("cluster_ctas", ctypes.c_int),
                ("threads_per_cta", ctypes.c_int), ("smem_bytes", ctypes.c_uint32),
                ("effective", TransformConfig), ("device_bytes", ctypes.c_size_t),
                ("tuned", ctypes.c_int), ("fwd_config", ctypes.c_int), ("inv_config", ctypes.c_int),
                ("twiddle_entries", ctypes.c_int)]


class KernelConfig(ctypes.Structure):
    _fields_ = [("logN", ctypes.c_int), ("cluster_ctas", ctypes.c_int), ("r1", ctypes.c_int),
                ("words_log2", ctypes.c_int), ("k1a", ctypes.c_int), ("k2a", ctypes.c_int),
                ("threads", ctypes.c_int), ("smem_bytes", ctypes.c_uint32),
                ("polys_per_job", ctypes.c_int), ("exchange", ctypes.c_int),
                ("k2b", ctypes.c_int)]


class TuneResult(ctypes.Structure):
    _fields_ = [("fwd_index", ctypes.c_int), ("inv_index", ctypes.c_int),
                ("fwd_us", ctypes.c_double), ("inv_us", ctypes.c_double),
                ("candidates", ctypes.c_int)]


NTT_OK = 0
PLAN_COMPRESSED_TWIDDLES = 1  # include/ntt_b200.h: NTT_PLAN_COMPRESSED_TWIDDLES
SMALL_WARP, SMALL_SHARED = 0, 1  # include/ntt_b200_tune.h: NTT_SMALL_*
MULTIPLY_ONE_LAUNCH, MULTIPLY_THREE_LAUNCHES = 0, 1  # NTT_MULTIPLY_*
STATUS_NAMES = {
    0: "NTT_OK", 1: "NTT_ERR_INVALID_ARGUMENT", 2: "NTT_ERR_MODULUS", 3: "NTT_ERR_ROOT",
    4: "NTT_ERR_MODULUS_RANGE", 5: "NTT_ERR_UNSUPPORTED", 6: "NTT_ERR_MISALIGNED",
    7: "NTT_ERR_CUDA", 8: "NTT_ERR_OUT_OF_MEMORY", 9: "NTT_ERR_BUDGET", 10: "NTT_ERR_TIMEOUT",
    11: "NTT_ERR_CANCELLED", 12: "NTT_ERR_NOT_READY", 13: "NTT_ERR_SHUTDOWN",
}


class NttError(RuntimeError):
    """A non-OK ntt_status_t.  ``status`` is the numeric code, ``name`` its
    enumerator name."""

    def __init__(self, status: int, where: str):
        self.status = int(status)
        self.name = STATUS_NAMES.get(self.status, str(status))
        detail = _lib.ntt_last_error().decode(errors="replace")
        super().__init__(f"{where}: {self.name}: {detail}")


_u32p = ctypes.POINTER(ctypes.c_uint32)
_vp = ctypes.c_void_p
_st = ctypes.c_int


def _sig(name, res, *args):
    f = getattr(_lib, name)
    f.restype = res
    f.argtypes = list(args)
    return f


_sig("ntt_version", ctypes.c_int)
_sig("ntt_status_string", ctypes.c_char_p, _st)
_sig("ntt_last_error", ctypes.c_char_p)
_sig("ntt_modulus_runtime", _st, ctypes.c_int, ModulusConfig, ctypes.POINTER(ModulusRuntime))
_sig("ntt_twiddle_table_host", _st, ctypes.c_int, ctypes.c_uint32, ctypes.c_uint32, _vp)
_sig("ntt_default_moduli", ctypes.c_int, ctypes.POINTER(ModulusConfig), ctypes.c_int)
_sig("ntt_default_transform", _st, ctypes.c_int, ctypes.POINTER(TransformConfig))
_sig("ntt_find_moduli", _st, ctypes.c_int, ctypes.c_int, ctypes.c_uint32,
     ctypes.POINTER(ModulusConfig))
_sig("ntt_plan_create", _st, ctypes.c_int, ctypes.POINTER(ModulusConfig), ctypes.c_int,
     ctypes.POINTER(TransformConfig), ctypes.POINTER(_vp))
_sig("ntt_plan_create_ex", _st, ctypes.c_int, ctypes.POINTER(ModulusConfig), ctypes.c_int,
     ctypes.POINTER(TransformConfig), ctypes.c_uint32, ctypes.POINTER(_vp))
_sig("ntt_plan_destroy", _st, _vp)
_sig("ntt_plan_get_info", _st, _vp, ctypes.POINTER(PlanInfo))
_sig("ntt_plan_tables", _st, _vp, ctypes.POINTER(_vp), ctypes.POINTER(_vp), ctypes.POINTER(_vp))
_sig("ntt_forward", _st, _vp, _vp, _vp)
_sig("ntt_inverse", _st, _vp, _vp, _vp)
_sig("ntt_forward_many", _st, _vp, _vp, ctypes.c_size_t, ctypes.c_size_t, _vp)
_sig("ntt_inverse_many", _st, _vp, _vp, ctypes.c_size_t, ctypes.c_size_t, _vp)
_sig("ntt_pointwise_mul", _st, _vp, _vp, _vp, _vp, ctypes.c_size_t, ctypes.c_size_t, _vp)
_sig("ntt_multiply_many", _st, _vp, _vp, _vp, ctypes.c_size_t, ctypes.c_size_t, _vp)
_sig("ntt_multiply_spectrum_many", _st, _vp, _vp, _vp, ctypes.c_size_t, ctypes.c_size_t, _vp)
_sig("ntt_measure_int_peak", _st, ctypes.POINTER(ctypes.c_double))
_sig("ntt_launch_ntt", _st, _vp, _vp, _vp, _vp, _vp, ctypes.c_size_t, ctypes.c_int,
     ctypes.POINTER(PhaseConfig), ctypes.POINTER(PhaseConfig))
_sig("ntt_launch_intt", _st, _vp, _vp, _vp, _vp, _vp, ctypes.c_size_t, ctypes.c_int,
     ctypes.POINTER(PhaseConfig), ctypes.POINTER(PhaseConfig))
_sig("ntt_shim_cache_clear", None)
_sig("ntt_shim_check", _st)
_sig("ntt_config_count", ctypes.c_int)
_sig("ntt_config_get", _st, ctypes.c_int, ctypes.POINTER(KernelConfig))
_sig("ntt_autotune", _st, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
     ctypes.POINTER(TuneResult))
_sig("ntt_autotune_forget", None)
_sig("ntt_plan_force_config", _st, _vp, ctypes.c_int, ctypes.c_int)
_sig("ntt_plan_set_schedule", _st, _vp, ctypes.c_int)
_sig("ntt_plan_set_small_kernel", _st, _vp, ctypes.c_int)
_sig("ntt_plan_set_multiply_form", _st, _vp, ctypes.c_int)
_sig("ntt_plan_check", _st, _vp, ctypes.POINTER(ctypes.c_uint32))
_sig("ntt_config_resident_clusters", ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int)
SCHEDULE_DIRECT = 0
SCHEDULE_STAGED = 1
_sig("ntt_autotune_reload", None)
_sig("ntt_selftest_wait_expiry", _st, _vp, ctypes.c_uint32, _vp)
_sig("ntt_forward_scaled", _st, _vp, _vp, ctypes.c_size_t, ctypes.c_size_t, _vp, _vp)
_sig("ntt_inverse_scaled", _st, _vp, _vp, ctypes.c_size_t, ctypes.c_size_t, _vp, _vp)
_sig("ntt_forward_skip", _st, _vp, _vp, ctypes.c_size_t, ctypes.c_size_t, ctypes.c_int,
     ctypes.c_int, _vp)
_sig("ntt_forward_sub_scale", _st, _vp, _vp, ctypes.c_size_t, ctypes.c_size_t, _vp,
     ctypes.c_size_t, ctypes.c_int, ctypes.c_int, _vp, _vp, _vp)
_sig("ntt_inverse_scaled_range", _st, _vp, _vp, ctypes.c_size_t, ctypes.c_size_t, ctypes.c_int,
     ctypes.c_int, _vp, _vp)


def _check(st: int, where: str):
    if st != NTT_OK:
        raise NttError(st, where)


def _ptr(x) -> Optional[int]:
    """Device address of a torch tensor / raw int / None."""
    if x is None:
        return None
    if isinstance(x, int):
        return x
    if hasattr(x, "data_ptr"):
        if hasattr(x, "is_cuda") and not x.is_cuda:
            raise ValueError("expected a CUDA tensor")
        return int(x.data_ptr())
    raise TypeError(f"cannot take a device pointer of {type(x)!r}")


def _stream(s) -> Optional[int]:
    if s is None:
        return None
    if isinstance(s, int):
        return s
    if hasattr(s, "cuda_stream"):
        return int(s.cuda_stream)
    raise TypeError(f"cannot take a CUDA stream handle of {type(s)!r}")


def version() -> int:
    return _lib.ntt_version()


# ---------------------------------------------------------------------------
# host precompute (reference mirrors)
# ---------------------------------------------------------------------------


def _moduli_array(moduli: Iterable) -> "ctypes.Array":
    ms = [m if isinstance(m, ModulusConfig) else ModulusConfig(int(m[0]), int(m[1]))
          for m in moduli]
    arr = (ModulusConfig * max(1, len(ms)))(*ms)
    return arr, len(ms)


def default_moduli() -> List[ModulusConfig]:
    """default_moduli() -- src/ntt_config.h:75-94."""
    n = _lib.ntt_default_moduli(None, 0)
    arr = (ModulusConfig * n)()
    _lib.ntt_default_moduli(arr, n)
    return list(arr)


def default_transform(logN: int) -> TransformConfig:
    """DefaultNTTLaunchConfig<LogN>::runtime_transform() -- src/ntt_config.h:62-73."""
    t = TransformConfig()
    _check(_lib.ntt_default_transform(logN, ctypes.byref(t)), "default_transform")
    return t


def modulus_runtime(logN: int, cfg) -> ModulusRuntime:
    """make_modulus_runtime -- raises NttError(NTT_ERR_MODULUS / NTT_ERR_ROOT)
    where the reference calls std::exit."""
    out = ModulusRuntime()
    m = cfg if isinstance(cfg, ModulusConfig) else ModulusConfig(int(cfg[0]), int(cfg[1]))
    _check(_lib.ntt_modulus_runtime(logN, m, ctypes.byref(out)), "modulus_runtime")
    return out


def twiddle_table(logN: int, q: int, root: int):
    """make_twiddle_table: root^bitrev(i) mod q (host, numpy uint32)."""
    import numpy as np
    out = np.empty(1 << logN, dtype=np.uint32)
    _check(_lib.ntt_twiddle_table_host(logN, q, root, out.ctypes.data), "twiddle_table")
    return out


def find_moduli(logN: int, count: int, lower_bound: int) -> List[ModulusConfig]:
    """First `count` primes >= lower_bound with q == 1 (mod 2N), ascending,
    with their smallest primitive roots."""
    arr = (ModulusConfig * max(1, count))()
    _check(_lib.ntt_find_moduli(logN, count, lower_bound, arr), "find_moduli")
    return list(arr)[:count]


# ---------------------------------------------------------------------------
# plans
# ---------------------------------------------------------------------------


class Plan:
    """Validated moduli + device-resident twiddle tables for one (logN,
    modulus chain).  Immutable after creation apart from the tuning setters
    (set_schedule, set_small_kernel, set_multiply_form, force_config: call
    them before sharing the plan); usable from several host
    threads on different streams."""

    def __init__(self, logN: int, moduli: Sequence, transform: Optional[TransformConfig] = None,
                 compressed_twiddles: bool = False):
        arr, n = _moduli_array(moduli)
        h = _vp()
        flags = PLAN_COMPRESSED_TWIDDLES if compressed_twiddles else 0
        _check(_lib.ntt_plan_create_ex(logN, arr, n,
                                       ctypes.byref(transform) if transform is not None else None,
                                       flags, ctypes.byref(h)), "ntt_plan_create_ex")
        self._h = h
        self.logN = logN
        self.N = 1 << logN
        self.limbs = n
        self.moduli = [(m.qi, m.primitive_root) for m in arr[:n]]

    @property
    def handle(self) -> int:
        return self._h.value

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            _lib.ntt_plan_destroy(self._h)
            self._h = _vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def info(self) -> PlanInfo:
        i = PlanInfo()
        _check(_lib.ntt_plan_get_info(self._h, ctypes.byref(i)), "ntt_plan_get_info")
        return i

    def force_config(self, fwd_index: int = -1, inv_index: int = -1):
        """Pin the plan to compiled configurations (see kernel_configs())."""
        _check(_lib.ntt_plan_force_config(self._h, fwd_index, inv_index), "ntt_plan_force_config")

    def set_multiply_form(self, form: int = MULTIPLY_ONE_LAUNCH):
        """Split plans: multiply_many in one launch (MULTIPLY_ONE_LAUNCH) or
        as split forward, cluster forward with the product, split inverse
        (MULTIPLY_THREE_LAUNCHES)."""
        _check(_lib.ntt_plan_set_multiply_form(self._h, form), "ntt_plan_set_multiply_form")

    def set_small_kernel(self, kind: int = SMALL_WARP):
        """logN 6..9: SMALL_WARP (a warp per limb, shuffles) or SMALL_SHARED
        (a CTA per limb, a shared-memory round per stage)."""
        _check(_lib.ntt_plan_set_small_kernel(self._h, kind), "ntt_plan_set_small_kernel")

    def set_schedule(self, schedule: int = SCHEDULE_DIRECT):
        """SCHEDULE_DIRECT: one limb per cluster, input from global memory;
        SCHEDULE_STAGED: resident clusters with the next input slab
        bulk-copied ahead.  Results do not depend on it."""
        _check(_lib.ntt_plan_set_schedule(self._h, schedule), "ntt_plan_set_schedule")

    def check(self) -> int:
        """Synchronize, read and clear the plan's device status word; raises
        NttError(NTT_ERR_TIMEOUT) if a bounded wait expired."""
        st = ctypes.c_uint32()
        _check(_lib.ntt_plan_check(self._h, ctypes.byref(st)), "ntt_plan_check")
        return st.value

    def selftest_wait_expiry(self, limit: int = 256, stream=None):
        """Run the kernels' bounded mbarrier wait on a barrier nothing
        completes (gives up after `limit` tries); the next check() raises
        NttError(NTT_ERR_TIMEOUT)."""
        _check(_lib.ntt_selftest_wait_expiry(self._h, limit, _stream(stream)),
               "ntt_selftest_wait_expiry")

    def tables(self):
        """(forward pairs, inverse pairs, moduli) device addresses."""
        f, i, q = _vp(), _vp(), _vp()
        _check(_lib.ntt_plan_tables(self._h, ctypes.byref(f), ctypes.byref(i), ctypes.byref(q)),
               "ntt_plan_tables")
        return f.value, i.value, q.value

    def forward(self, a, stream=None):
        _check(_lib.ntt_forward(self._h, _ptr(a), _stream(stream)), "ntt_forward")

    def inverse(self, a, stream=None):
        _check(_lib.ntt_inverse(self._h, _ptr(a), _stream(stream)), "ntt_inverse")

    def forward_many(self, a, polys: int, poly_stride: int = 0, stream=None):
        _check(_lib.ntt_forward_many(self._h, _ptr(a), polys, poly_stride, _stream(stream)),
               "ntt_forward_many")

    def inverse_many(self, a, polys: int, poly_stride: int = 0, stream=None):
        _check(_lib.ntt_inverse_many(self._h, _ptr(a), polys, poly_stride, _stream(stream)),
               "ntt_inverse_many")

    def forward_scaled(self, a, scale, polys: int = 1, poly_stride: int = 0, stream=None):
        """a <- NTT(c_l * a) per limb l; `scale`: device array of one uint32
        constant per limb (normal domain)."""
        _check(_lib.ntt_forward_scaled(self._h, _ptr(a), polys, poly_stride, _ptr(scale),
                                       _stream(stream)), "ntt_forward_scaled")

    def inverse_scaled(self, a, scale, polys: int = 1, poly_stride: int = 0, stream=None):
        """a <- c_l * INTT(a) per limb l (see forward_scaled)."""
        _check(_lib.ntt_inverse_scaled(self._h, _ptr(a), polys, poly_stride, _ptr(scale),
                                       _stream(stream)), "ntt_inverse_scaled")

    def forward_skip(self, a, skip_begin: int, skip_end: int, polys: int = 1,
                     poly_stride: int = 0, stream=None):
        """ModUp's forward: every limb except [skip_begin, skip_end)."""
        _check(_lib.ntt_forward_skip(self._h, _ptr(a), polys, poly_stride, skip_begin, skip_end,
                                     _stream(stream)), "ntt_forward_skip")

    def forward_sub_scale(self, a, sub, sub_begin: int, sub_end: int, scale=None, sub_mul=None,
                          polys: int = 1, poly_stride: int = 0, sub_stride: int = 0,
                          stream=None):
        """ModDown's forward: a_l <- (NTT(a_l) - d_k s_l) c_l per limb l, s_l
        the limb k = l - sub_begin of `sub` for l in [sub_begin, sub_end)
        (0 elsewhere); `scale` (c) and `sub_mul` (d): optional device arrays of
        normal-domain constants, per plan limb and per sub limb."""
        _check(_lib.ntt_forward_sub_scale(self._h, _ptr(a), polys, poly_stride, _ptr(sub),
                                          sub_stride, sub_begin, sub_end, _ptr(scale),
                                          _ptr(sub_mul), _stream(stream)),
               "ntt_forward_sub_scale")

    def inverse_scaled_range(self, a, limb_begin: int, limb_end: int, scale=None,
                             polys: int = 1, poly_stride: int = 0, stream=None):
        """a_l <- c_k INTT(a_l) for limbs l in [limb_begin, limb_end) only,
        c_k = scale[l - limb_begin] (None: 1)."""
        _check(_lib.ntt_inverse_scaled_range(self._h, _ptr(a), polys, poly_stride, limb_begin,
                                             limb_end, _ptr(scale), _stream(stream)),
               "ntt_inverse_scaled_range")

    def pointwise_mul(self, c, a, b, polys: int = 1, poly_stride: int = 0, stream=None):
        """c = a (.) b: Montgomery product of two forward outputs per limb."""
        _check(_lib.ntt_pointwise_mul(self._h, _ptr(c), _ptr(a), _ptr(b), polys, poly_stride,
                                      _stream(stream)), "ntt_pointwise_mul")

    def multiply_spectrum_many(self, a_spec, b, polys: int = 1, poly_stride: int = 0,
                               stream=None):
        """b <- INTT(NTT(b) (.) a_spec): the product with an operand whose
        spectrum (this plan's forward output) is already resident."""
        _check(_lib.ntt_multiply_spectrum_many(self._h, _ptr(a_spec), _ptr(b), polys, poly_stride,
                                               _stream(stream)), "ntt_multiply_spectrum_many")

    def multiply_many(self, a, b, polys: int = 1, poly_stride: int = 0, stream=None):
        """b <- a * b negacyclic per limb (normal domain), a read only: three
        launches, the pointwise product folded into the forward of a."""
        _check(_lib.ntt_multiply_many(self._h, _ptr(a), _ptr(b), polys, poly_stride,
                                      _stream(stream)), "ntt_multiply_many")


# ---------------------------------------------------------------------------
# drop-in launchers (v04:603-658)
# ---------------------------------------------------------------------------


def _phase(p):
    if p is None:
        return None
    if isinstance(p, PhaseConfig):
        return ctypes.byref(p)
    return ctypes.byref(PhaseConfig(*p))


def launch_ntt(A_dev, twiddle_dev, moduli_dev, q_inv_dev, r2_dev, limb_count: int, logN: int,
               phase1=None, phase2=None):
    """launch_ntt<LC>(A, tw, moduli, q_inv, r2, limb_count) with LC's logN and
    NTT phase triples (None: DefaultNTTLaunchConfig<logN>)."""
    _check(_lib.ntt_launch_ntt(_ptr(A_dev), _ptr(twiddle_dev), _ptr(moduli_dev), _ptr(q_inv_dev),
                               _ptr(r2_dev), limb_count, logN, _phase(phase1), _phase(phase2)),
           "ntt_launch_ntt")


def launch_intt(A_dev, inv_twiddle_dev, moduli_dev, q_inv_dev, degree_inv_dev, limb_count: int,
                logN: int, phase1=None, phase2=None):
    """launch_intt<LC>(A, inv_tw, moduli, q_inv, degree_inv, limb_count)."""
    _check(_lib.ntt_launch_intt(_ptr(A_dev), _ptr(inv_twiddle_dev), _ptr(moduli_dev),
                                _ptr(q_inv_dev), _ptr(degree_inv_dev), limb_count, logN,
                                _phase(phase1), _phase(phase2)), "ntt_launch_intt")


def shim_cache_clear():
    _lib.ntt_shim_cache_clear()


def shim_check():
    """Raises NTT_ERR_MODULUS_RANGE if a drop-in call since the last check
    named a modulus that is even or not below 2^31 (synchronises)."""
    _check(_lib.ntt_shim_check(), "ntt_shim_check")


def measure_int_peak() -> float:
    """32-bit multiplies per second of the current device on the Shoup mix."""
    v = ctypes.c_double()
    _check(_lib.ntt_measure_int_peak(ctypes.byref(v)), "ntt_measure_int_peak")
    return v.value


# ---------------------------------------------------------------------------
# configuration catalogue and autotuner
# ---------------------------------------------------------------------------


def kernel_configs() -> List[KernelConfig]:
    out = []
    for i in range(_lib.ntt_config_count()):
        c = KernelConfig()
        _check(_lib.ntt_config_get(i, ctypes.byref(c)), "ntt_config_get")
        out.append(c)
    return out


def resident_clusters(index: int, forward: bool = True, schedule: int = SCHEDULE_DIRECT) -> int:
    """Clusters of compiled configuration `index` resident at once on the
    current device under `schedule`."""
    return _lib.ntt_config_resident_clusters(index, 1 if forward else 0, schedule)


def autotune(logN: int, limbs: int, polys: int = 8, iters: int = 5) -> TuneResult:
    r = TuneResult()
    _check(_lib.ntt_autotune(logN, limbs, polys, iters, ctypes.byref(r)), "ntt_autotune")
    return r


def autotune_forget():
    _lib.ntt_autotune_forget()


def autotune_reload():
    _lib.ntt_autotune_reload()


# ---------------------------------------------------------------------------
# ragged batches (include/ntt_b200_batch.h)
# ---------------------------------------------------------------------------

OP_FORWARD = 0
OP_INVERSE = 1
OP_MULTIPLY = 2
OP_MULTIPLY_SPECTRUM = 3
BATCH_MIN_LOGN = 12
BATCH_MAX_LOGN = 17


class Job(ctypes.Structure):
    _fields_ = [("op", ctypes.c_int), ("logN", ctypes.c_int), ("limbs", ctypes.c_int),
                ("moduli", ctypes.POINTER(ModulusConfig)), ("data", _vp), ("operand", _vp)]


class BatchOptions(ctypes.Structure):
    _fields_ = [("cluster_ctas", ctypes.c_int), ("use_graph", ctypes.c_int),
                ("max_clusters", ctypes.c_int)]


class BatchInfo(ctypes.Structure):
    _fields_ = [("jobs", ctypes.c_int), ("tiles", ctypes.c_int), ("groups", ctypes.c_int),
                ("cluster_ctas", ctypes.c_int), ("clusters", ctypes.c_int),
                ("multiply", ctypes.c_int), ("smem_bytes", ctypes.c_uint32),
                ("device_bytes", ctypes.c_size_t)]


_sig("ntt_batch_create", _st, ctypes.POINTER(Job), ctypes.c_int, ctypes.POINTER(BatchOptions),
     ctypes.POINTER(_vp))
_sig("ntt_batch_run", _st, _vp, _vp)
_sig("ntt_batch_get_info", _st, _vp, ctypes.POINTER(BatchInfo))
_sig("ntt_batch_destroy", _st, _vp)
_sig("ntt_batch_submit", _st, ctypes.POINTER(Job), ctypes.c_int, _vp)
_sig("ntt_tables_device_bytes", ctypes.c_size_t)
_sig("ntt_tables_trim", None)
_sig("ntt_tables_preload", _st, ctypes.c_int, ctypes.POINTER(ModulusConfig), ctypes.c_int)


def _job_array(jobs: Sequence) -> tuple:
    """jobs: sequence of (op, logN, moduli, data, operand-or-None)."""
    keep = []
    arr = (Job * max(1, len(jobs)))()
    for i, (op, logN, moduli, data, operand) in enumerate(jobs):
        m, n = _moduli_array(moduli)
        keep.append(m)
        arr[i] = Job(op, logN, n, ctypes.cast(m, ctypes.POINTER(ModulusConfig)), _ptr(data),
                     _ptr(operand))
    return arr, keep


class Batch:
    """A ragged set of jobs run by one persistent launch (CUDA-graph replay
    by default).  jobs: sequence of (op, logN, moduli, data, operand) with
    op in OP_FORWARD / OP_INVERSE / OP_MULTIPLY, data (and operand) device
    buffers of limbs * 2^logN uint32 words."""

    def __init__(self, jobs: Sequence, cluster_ctas: int = 0, use_graph: bool = True,
                 max_clusters: int = 0):
        arr, self._keep = _job_array(jobs)
        opts = BatchOptions(cluster_ctas, 1 if use_graph else 0, max_clusters)
        h = _vp()
        _check(_lib.ntt_batch_create(arr, len(jobs), ctypes.byref(opts), ctypes.byref(h)),
               "ntt_batch_create")
        self._h = h

    def run(self, stream=None):
        _check(_lib.ntt_batch_run(self._h, _stream(stream)), "ntt_batch_run")

    @property
    def info(self) -> BatchInfo:
        i = BatchInfo()
        _check(_lib.ntt_batch_get_info(self._h, ctypes.byref(i)), "ntt_batch_get_info")
        return i

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            _lib.ntt_batch_destroy(self._h)
            self._h = _vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def batch_submit(jobs: Sequence, stream=None):
    """Create, run, wait for and destroy a one-off batch."""
    arr, keep = _job_array(jobs)
    _check(_lib.ntt_batch_submit(arr, len(jobs), _stream(stream)), "ntt_batch_submit")


def tables_device_bytes() -> int:
    return _lib.ntt_tables_device_bytes()


def tables_trim():
    _lib.ntt_tables_trim()


def tables_preload(logN: int, moduli: Sequence):
    """Generate and keep the device tables of these moduli for logN."""
    m, n = _moduli_array(moduli)
    _check(_lib.ntt_tables_preload(logN, m, n), "ntt_tables_preload")


# ---------------------------------------------------------------------------
# serving loop (include/ntt_b200_serve.h)
# ---------------------------------------------------------------------------


class Request(ctypes.Structure):
    _fields_ = [("op", ctypes.c_int), ("logN", ctypes.c_int), ("limbs", ctypes.c_int),
                ("moduli", ctypes.POINTER(ModulusConfig)), ("input", _vp), ("operand", _vp),
                ("operand_handle", ctypes.c_uint64), ("output", _vp),
                ("device_buffers", ctypes.c_int)]


class ServerOptions(ctypes.Structure):
    _fields_ = [("hbm_budget_bytes", ctypes.c_size_t), ("streams", ctypes.c_int),
                ("max_round_tiles", ctypes.c_int), ("cluster_ctas", ctypes.c_int),
                ("max_round_requests", ctypes.c_int)]


class ServerStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_uint64), ("completed", ctypes.c_uint64),
                ("failed", ctypes.c_uint64), ("rounds", ctypes.c_uint64),
                ("mean_round_requests", ctypes.c_double), ("p50_ms", ctypes.c_double),
                ("p99_ms", ctypes.c_double), ("mean_ms", ctypes.c_double),
                ("max_ms", ctypes.c_double), ("elapsed_s", ctypes.c_double),
                ("limb_ntt_per_s", ctypes.c_double), ("budget_bytes", ctypes.c_size_t),
                ("arena_peak_bytes", ctypes.c_size_t), ("resident_bytes", ctypes.c_size_t),
                ("table_bytes", ctypes.c_size_t)]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


_sig("ntt_server_create", _st, ctypes.POINTER(ServerOptions), ctypes.POINTER(_vp))
_sig("ntt_server_submit", _st, _vp, ctypes.POINTER(Request), ctypes.POINTER(ctypes.c_uint64))
_sig("ntt_server_poll", _st, _vp, ctypes.c_uint64)
_sig("ntt_server_wait", _st, _vp, ctypes.c_uint64, ctypes.c_double)
_sig("ntt_server_latency_ms", ctypes.c_double, _vp, ctypes.c_uint64)
_sig("ntt_server_put", _st, _vp, _vp, ctypes.c_size_t, ctypes.POINTER(ctypes.c_uint64))
_sig("ntt_server_drop", _st, _vp, ctypes.c_uint64)
_sig("ntt_server_put_spectrum", _st, _vp, ctypes.c_int, ctypes.POINTER(ModulusConfig), ctypes.c_int,
     _vp, ctypes.POINTER(ctypes.c_uint64))
_sig("ntt_server_stats", _st, _vp, ctypes.c_int, ctypes.POINTER(ServerStats))
_sig("ntt_server_destroy", _st, _vp)


def _host_ptr(a) -> int:
    """Address of a C-contiguous host buffer (numpy array or CPU tensor)."""
    if hasattr(a, "ctypes"):
        if not a.flags["C_CONTIGUOUS"]:
            raise ValueError("host buffers must be C-contiguous")
        return a.ctypes.data
    if hasattr(a, "data_ptr"):
        if getattr(a, "is_cuda", False):
            raise ValueError("expected a host buffer")
        return int(a.data_ptr())
    if isinstance(a, int):
        return a
    raise TypeError(f"cannot take a host pointer of {type(a)!r}")


class Server:
    """Continuous-batching request loop.  Requests carry host buffers of
    limbs * 2^logN uint32 words (pinned memory keeps the copies
    asynchronous); results are written to `output` when the ticket
    completes.  The Python object keeps every buffer of a pending request
    alive until its ticket is waited on or polled complete."""

    def __init__(self, hbm_budget_bytes: int = 0, streams: int = 0, max_round_tiles: int = 0,
                 cluster_ctas: int = 0, max_round_requests: int = 0):
        o = ServerOptions(hbm_budget_bytes, streams, max_round_tiles, cluster_ctas,
                          max_round_requests)
        h = _vp()
        _check(_lib.ntt_server_create(ctypes.byref(o), ctypes.byref(h)), "ntt_server_create")
        self._h = h
        self._live = {}

    def request(self, op: int, logN: int, moduli: Sequence, input, output, operand=None,
                operand_handle: int = 0, device: bool = False):
        """A prepared request (for submit_prepared): device=True takes device
        tensors that are transformed in place (input copied into output
        first when they differ)."""
        m, n = _moduli_array(moduli)
        p = _ptr if device else _host_ptr
        r = Request(op, logN, n, ctypes.cast(m, ctypes.POINTER(ModulusConfig)), p(input),
                    p(operand) if operand is not None else None, operand_handle, p(output),
                    1 if device else 0)
        return r, (m, input, output, operand)

    def submit_prepared(self, prepared) -> int:
        r, keep = prepared
        t = ctypes.c_uint64()
        _check(_lib.ntt_server_submit(self._h, ctypes.byref(r), ctypes.byref(t)),
               "ntt_server_submit")
        self._live[t.value] = keep
        return t.value

    def submit(self, op: int, logN: int, moduli: Sequence, input, output, operand=None,
               operand_handle: int = 0, device: bool = False) -> int:
        return self.submit_prepared(self.request(op, logN, moduli, input, output, operand,
                                                 operand_handle, device))

    def poll(self, ticket: int) -> bool:
        st = _lib.ntt_server_poll(self._h, ticket)
        if st == 12:  # NTT_ERR_NOT_READY
            return False
        self._live.pop(ticket, None)
        _check(st, "ntt_server_poll")
        return True

    def wait(self, ticket: int, timeout: float = -1.0):
        st = _lib.ntt_server_wait(self._h, ticket, timeout)
        if st != 10:  # NTT_ERR_TIMEOUT keeps the buffers alive
            self._live.pop(ticket, None)
        _check(st, "ntt_server_wait")

    def latency_ms(self, ticket: int) -> float:
        return _lib.ntt_server_latency_ms(self._h, ticket)

    def put(self, host) -> int:
        h = ctypes.c_uint64()
        words = int(host.size) if hasattr(host, "size") and not callable(host.size) else host.numel()
        _check(_lib.ntt_server_put(self._h, _host_ptr(host), words, ctypes.byref(h)),
               "ntt_server_put")
        return h.value

    def put_spectrum(self, logN: int, moduli: Sequence, host) -> int:
        """Resident operand stored as its spectrum (for OP_MULTIPLY_SPECTRUM)."""
        m, n = _moduli_array(moduli)
        h = ctypes.c_uint64()
        _check(_lib.ntt_server_put_spectrum(self._h, logN, m, n, _host_ptr(host), ctypes.byref(h)),
               "ntt_server_put_spectrum")
        return h.value

    def drop(self, handle: int):
        _check(_lib.ntt_server_drop(self._h, handle), "ntt_server_drop")

    def stats(self, reset: bool = False) -> dict:
        s = ServerStats()
        _check(_lib.ntt_server_stats(self._h, 1 if reset else 0, ctypes.byref(s)),
               "ntt_server_stats")
        return s.as_dict()

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            _lib.ntt_server_destroy(self._h)
            self._h = _vp()
            self._live.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


# ---------------------------------------------------------------------------
# 64-bit words (include/ntt_b200_u64.h)
# ---------------------------------------------------------------------------


class ModulusConfig64(ctypes.Structure):
    _fields_ = [("qi", ctypes.c_uint64), ("primitive_root", ctypes.c_uint64)]

    def __iter__(self):
        return iter((self.qi, self.primitive_root))


_sig("ntt64_find_moduli", _st, ctypes.c_int, ctypes.c_int, ctypes.c_uint64,
     ctypes.POINTER(ModulusConfig64))
_sig("ntt64_plan_create", _st, ctypes.c_int, ctypes.POINTER(ModulusConfig64), ctypes.c_int,
     ctypes.POINTER(_vp))
_sig("ntt64_plan_destroy", _st, _vp)
_sig("ntt64_forward_many", _st, _vp, _vp, ctypes.c_size_t, ctypes.c_size_t, _vp)
_sig("ntt64_inverse_many", _st, _vp, _vp, ctypes.c_size_t, ctypes.c_size_t, _vp)


def find_moduli64(logN: int, count: int, lower_bound: int) -> List[ModulusConfig64]:
    """First `count` primes >= lower_bound with q == 1 (mod 2N), q < 2^62,
    ascending, each with its smallest quadratic non-residue as root."""
    arr = (ModulusConfig64 * max(1, count))()
    _check(_lib.ntt64_find_moduli(logN, count, lower_bound, arr), "ntt64_find_moduli")
    return list(arr)[:count]


class Plan64:
    """64-bit word plan: limbs * 2^logN uint64 words per polynomial (torch
    int64 / uint64 CUDA tensors), the 32-bit plans' domain contract with
    R = 2^64."""

    def __init__(self, logN: int, moduli: Sequence):
        m = (ModulusConfig64 * len(moduli))(*[ModulusConfig64(int(q), int(g)) for q, g in moduli])
        h = _vp()
        _check(_lib.ntt64_plan_create(logN, m, len(moduli), ctypes.byref(h)), "ntt64_plan_create")
        self._h, self.logN, self.limbs = h, logN, len(moduli)

    def forward_many(self, a, polys: int = 1, poly_stride: int = 0, stream=None):
        _check(_lib.ntt64_forward_many(self._h, _ptr(a), polys, poly_stride, _stream(stream)),
               "ntt64_forward_many")

    def inverse_many(self, a, polys: int = 1, poly_stride: int = 0, stream=None):
        _check(_lib.ntt64_inverse_many(self._h, _ptr(a), polys, poly_stride, _stream(stream)),
               "ntt64_inverse_many")

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            _lib.ntt64_plan_destroy(self._h)
            self._h = _vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
