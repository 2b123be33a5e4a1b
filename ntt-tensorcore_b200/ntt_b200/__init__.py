"""Python binding of libntt_b200.so (the C ABI in include/ntt_b200.h).

The library is the product: every call here goes through the C ABI to the
sm_100a kernels.  There is no CPU fallback -- if the shared library is missing
or no GPU is present, the calls raise.

Device buffers are passed as torch tensors (their data_ptr) or raw integer
addresses; torch is used only for device memory and streams.
"""
import ctypes
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
# NTT_B200_LIB=dbg selects the NTT_DEBUG_BOUNDS build (range-checked kernels),
# NTT_B200_LIB=phase the NTT_PHASE_PROFILE build (the INT8 kernel's phase counters)
LIB_PATH = os.path.join(HERE, {"dbg": "libntt_b200_dbg.so", "phase": "libntt_b200_phase.so"}.get(
    os.environ.get("NTT_B200_LIB", ""), "libntt_b200.so"))
HEADER = os.path.join(os.path.dirname(os.path.dirname(HERE)), "include", "ntt_b200.h")

OK = 0
ENGINE_AUTO, ENGINE_SCALAR, ENGINE_DMMA, ENGINE_INT8, ENGINE_TILES = 0, 1, 2, 3, 4
ENGINES = {"auto": ENGINE_AUTO, "scalar": ENGINE_SCALAR, "dmma": ENGINE_DMMA, "int8": ENGINE_INT8,
           "tiles": ENGINE_TILES}
NEGACYCLIC = 1
ERR_INVALID_ARG, ERR_UNSUPPORTED, ERR_CUDA, ERR_NO_MEMORY, ERR_TIMEOUT, ERR_BUDGET = 1, 2, 3, 4, 5, 6

_u64 = ctypes.c_uint64
_u32 = ctypes.c_uint32
_vp = ctypes.c_void_p
_int = ctypes.c_int


class NTTError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__("ntt_b200 status %d: %s" % (status, msg))
        self.status = status


class _Params(ctypes.Structure):
    _fields_ = [(n, _u64) for n in ("q", "q_twice", "barrett_k", "barrett_m", "omega", "omega_inv", "n_inv")]


class _PlanInfo(ctypes.Structure):
    _fields_ = [("n", _u64), ("log_n", _u64), ("q", _u64), ("mu", _u64),
                ("d_twiddles", _vp), ("d_twiddles_inv", _vp), ("params", _Params)]


class BatchJob(ctypes.Structure):
    """nttb_batch_job."""
    _fields_ = [("data", _vp), ("log_n", _u32), ("n_limbs", _u32), ("first_modulus", _u32), ("flags", _u32),
                ("pointwise", _vp)]


class BatchConfig(ctypes.Structure):
    """nttb_batch_config: tile_elems, threads, split, lag, ctas_per_sm, group, tensor."""
    _fields_ = [("tile_elems", _u32), ("threads", _u32), ("split", _u32), ("lag", _u32), ("ctas_per_sm", _u32),
                ("group", _u32), ("tensor", _u32)]

    def as_dict(self):
        return {f: int(getattr(self, f)) for f, _ in self._fields_}


class ServerConfig(ctypes.Structure):
    """nttb_server_config."""
    _fields_ = [("hbm_budget_bytes", _u64), ("max_log_n", _u32), ("slots", _u32), ("max_batch_requests", _u32),
                ("negacyclic", _u32), ("max_batch_residues", _u64), ("batch", BatchConfig)]


class ServerStats(ctypes.Structure):
    """nttb_server_stats_t."""
    _fields_ = [(f, _u64) for f in ("submitted", "completed", "queued", "batches", "batched_requests",
                                    "bytes_in_use", "peak_bytes_in_use", "region_bytes", "resident_bytes")]


BATCH_INVERSE = 2
BATCH_POLYMUL = 4

_lib = None


def header_symbols():
    """Function names declared in include/ntt_b200.h."""
    with open(HEADER) as f:
        text = f.read()
    return sorted(set(re.findall(r"NTTB_API\s+(?:const\s+char\s*\*|int)\s+(nttb_\w+)\s*\(", text)))


def lib():
    """Loads libntt_b200.so (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError("libntt_b200.so missing: run `python ntt-tensorcore_b200/build.py`")
    L = ctypes.CDLL(LIB_PATH)
    sig = {
        "nttb_version": (ctypes.c_char_p, []),
        "nttb_status_string": (ctypes.c_char_p, [_int]),
        "nttb_last_error": (ctypes.c_char_p, []),
        "nttb_create_params": (_int, [_u64, _u64, ctypes.POINTER(_Params)]),
        "nttb_find_primitive_root": (_int, [_u64, _u64, ctypes.POINTER(_u64)]),
        "nttb_find_psi": (_int, [_u64, _u64, ctypes.POINTER(_u64)]),
        "nttb_host_ntt": (_int, [_vp, _u64, ctypes.POINTER(_Params), _int]),
        "nttb_generate_primes": (_int, [_u32, _u32, _u32, _vp]),
        "nttb_plan_create": (_int, [_u64, _u64, ctypes.POINTER(_vp)]),
        "nttb_plan_destroy": (_int, [_vp]),
        "nttb_plan_get_info": (_int, [_vp, ctypes.POINTER(_PlanInfo)]),
        "nttb_u64_transform": (_int, [_vp, _vp, _u64, _int, _int, _vp]),
        "nttb_u64_four_step": (_int, [_vp, _vp, _int, _vp]),
        "nttb_u64_rowmaj_forward": (_int, [_vp, _vp, _vp]),
        "nttb_u64_pretransposed_transform": (_int, [_vp, _vp, _u64, _int, _vp]),
        "nttb_u64_transpose": (_int, [_vp, _vp, _u64, _u64, _vp]),
        "nttb_u64_pointwise_mul": (_int, [_vp, _vp, _vp, _vp, _vp]),
        "nttb_u64_bit_reverse": (_int, [_vp, _u64, _vp]),
        "nttb_rns_plan_create": (_int, [_u32, _vp, _u32, _u32, ctypes.POINTER(_vp)]),
        "nttb_rns_plan_destroy": (_int, [_vp]),
        "nttb_rns_transform": (_int, [_vp, _vp, _vp, _u32, _int, _int, _vp]),
        "nttb_rns_pointwise_mul": (_int, [_vp, _vp, _vp, _vp, _u32, _vp]),
        "nttb_rns_transform_noalloc": (_int, [_vp, _vp, _u32, _int, _vp]),
        "nttb_rns_forward_inverse": (_int, [_vp, _vp, _u32, _int, _vp]),
        "nttb_rns_stream_host": (_int, [_vp, _vp, _vp, _u32, _u32, _int, _int, _vp]),
        "nttb_wide_plan_create": (_int, [_u32, _vp, _u32, _u32, ctypes.POINTER(_vp)]),
        "nttb_wide_plan_destroy": (_int, [_vp]),
        "nttb_wide_transform": (_int, [_vp, _vp, _vp, _u32, _int, _vp]),
        "nttb_wide_transform_engine": (_int, [_vp, _vp, _vp, _u32, _int, _int, _vp]),
        "nttb_klimb_forward": (_int, [_u32, _vp, _vp, _u64, _u32, _vp, _u32, _vp]),
        "nttb_server_default_config": (_int, [ctypes.POINTER(ServerConfig)]),
        "nttb_server_create": (_int, [_vp, _u32, ctypes.POINTER(ServerConfig), ctypes.POINTER(_vp)]),
        "nttb_server_submit": (_int, [_vp, _vp, _vp, _vp, _u32, _u32, _u32, ctypes.POINTER(_u64)]),
        "nttb_server_submit_ntt": (_int, [_vp, _vp, _vp, _u32, _u32, _u32, _int, ctypes.POINTER(_u64)]),
        "nttb_server_submit_device": (_int, [_vp, _int, _vp, _vp, _vp, _u32, _u32, _u32, ctypes.POINTER(_u64)]),
        "nttb_server_wait": (_int, [_vp, _u64, ctypes.c_double, ctypes.POINTER(ctypes.c_double)]),
        "nttb_server_drain": (_int, [_vp, ctypes.c_double]),
        "nttb_server_stats": (_int, [_vp, ctypes.POINTER(ServerStats)]),
        "nttb_server_latencies": (_int, [_vp, _vp, _u64, ctypes.POINTER(_u64), _int]),
        "nttb_server_destroy": (_int, [_vp]),
        "nttb_batch_plan_create": (_int, [_vp, _u32, _u32, _u32, ctypes.POINTER(_vp)]),
        "nttb_batch_plan_destroy": (_int, [_vp]),
        "nttb_batch_default_config": (_int, [ctypes.POINTER(BatchConfig)]),
        "nttb_batch_ctas": (_int, [_vp, ctypes.POINTER(_u32)]),
        "nttb_batch_test_stall": (_int, [_vp, _u32]),
        "nttb_batch_autotune": (_int, [_vp, _vp, _u32, _vp, ctypes.POINTER(BatchConfig)]),
        "nttb_batch_create": (_int, [_vp, _vp, _u32, ctypes.POINTER(BatchConfig), ctypes.POINTER(_vp)]),
        "nttb_batch_destroy": (_int, [_vp]),
        "nttb_batch_launch": (_int, [_vp, _vp]),
        "nttb_batch_graph_launch": (_int, [_vp, _vp]),
        "nttb_batch_info": (_int, [_vp, ctypes.POINTER(_u64), ctypes.POINTER(_u64), ctypes.POINTER(_u64),
                                   ctypes.POINTER(BatchConfig)]),
        "nttb_device_errors": (_int, [ctypes.POINTER(_u32), _int]),
        "nttb_bounds_errors": (_int, [ctypes.POINTER(_u32), ctypes.POINTER(_int), _int]),
        "nttb_phase_profile": (_int, [ctypes.POINTER(_u64), ctypes.POINTER(_int), _int]),
        "nttb_launch_count": (_int, [ctypes.POINTER(_u64)]),
        "nttb_profile_start": (_int, []),
        "nttb_profile_stop": (_int, [ctypes.POINTER(_u32)]),
        "nttb_profile_read": (_int, [_u32, ctypes.c_char_p, _u32, ctypes.POINTER(_u64),
                                     ctypes.POINTER(ctypes.c_double)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def _check(status):
    if status != OK:
        msg = lib().nttb_last_error().decode()
        raise NTTError(status, msg)


def _ptr(x):
    if x is None:
        return None
    if isinstance(x, int):
        return x
    if hasattr(x, "data_ptr"):
        return x.data_ptr()  # torch tensor
    return x.ctypes.data  # numpy array


def _stream(stream):
    if stream is None:
        return None
    if isinstance(stream, int):
        return stream
    return stream.cuda_stream  # torch.cuda.Stream


def _engine(e):
    return ENGINES[e] if isinstance(e, str) else int(e)


def version():
    return lib().nttb_version().decode()


# ------------------------------------------------------------ uneven batches
def _jobs(jobs):
    """Job tuples -> nttb_batch_job[].  A transform is (data, log_n, n_limbs,
    first_modulus, inverse, negacyclic); a product adds its second operand:
    (a, log_n, n_limbs, first_modulus, "mul", negacyclic, b)."""
    arr = (BatchJob * len(jobs))()
    for i, job in enumerate(jobs):
        data, log_n, n_limbs, first, kind, nega = job[:6]
        if kind == "mul":
            flags, other = BATCH_POLYMUL, _ptr(job[6])
        else:
            flags, other = (BATCH_INVERSE if kind else 0), None
        arr[i] = BatchJob(_ptr(data), log_n, n_limbs, first, flags | (NEGACYCLIC if nega else 0), other)
    return arr


class BatchPlan:
    """Twiddle tables for a set of 31-bit moduli up to 2^max_log_n residues;
    uneven job lists run on it in one persistent launch (nttb_batch_*)."""

    def __init__(self, moduli, max_log_n, negacyclic=False):
        import numpy as np
        m = np.ascontiguousarray(moduli, dtype=np.uint64)
        h = _vp()
        _check(lib().nttb_batch_plan_create(m.ctypes.data, m.size, max_log_n, NEGACYCLIC if negacyclic else 0,
                                            ctypes.byref(h)))
        self._h, self.moduli, self.max_log_n = h, [int(x) for x in m], max_log_n

    def autotune(self, jobs, stream=None):
        cfg = BatchConfig()
        arr = _jobs(jobs)
        _check(lib().nttb_batch_autotune(self._h, arr, len(jobs), _stream(stream), ctypes.byref(cfg)))
        return cfg.as_dict()

    def batch(self, jobs, config=None):
        """jobs: (data, log_n, n_limbs, first_modulus, inverse, negacyclic) tuples."""
        arr = _jobs(jobs)
        cfg = None
        if config is not None:
            cfg = BatchConfig()
            _check(lib().nttb_batch_default_config(ctypes.byref(cfg)))
            for k, v in config.items():
                setattr(cfg, k, int(v))
        h = _vp()
        _check(lib().nttb_batch_create(self._h, arr, len(jobs), ctypes.byref(cfg) if cfg else None, ctypes.byref(h)))
        return Batch(h, self)

    def close(self):
        if getattr(self, "_h", None):
            lib().nttb_batch_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    def __init__(self, h, plan):
        self._h, self._plan = h, plan

    def launch(self, stream=None):
        _check(lib().nttb_batch_launch(self._h, _stream(stream)))

    def graph_launch(self, stream=None):
        _check(lib().nttb_batch_graph_launch(self._h, _stream(stream)))

    def test_stall(self, unit):
        """Failure-path test hook (nttb_batch_test_stall)."""
        _check(lib().nttb_batch_test_stall(self._h, unit))

    def info(self):
        u, t, w, cfg = _u64(), _u64(), _u64(), BatchConfig()
        _check(lib().nttb_batch_info(self._h, ctypes.byref(u), ctypes.byref(t), ctypes.byref(w), ctypes.byref(cfg)))
        g = _u32()
        _check(lib().nttb_batch_ctas(self._h, ctypes.byref(g)))
        return {"units": int(u.value), "tiles": int(t.value), "ws_bytes": int(w.value), "config": cfg.as_dict(),
                "ctas": int(g.value)}

    def close(self):
        if getattr(self, "_h", None):
            lib().nttb_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------- serving
class Server:
    """Polynomial-product and NTT server (nttb_server_*): requests are host
    arrays (numpy, or pinned torch CPU tensors) of n_limbs x 2^log_n residues."""

    def __init__(self, moduli, **config):
        import numpy as np
        cfg = ServerConfig()
        _check(lib().nttb_server_default_config(ctypes.byref(cfg)))
        for k, v in config.items():
            if k == "batch":
                for bk, bv in v.items():
                    setattr(cfg.batch, bk, int(bv))
            else:
                setattr(cfg, k, int(v))
        m = np.ascontiguousarray(moduli, dtype=np.uint64)
        h = _vp()
        _check(lib().nttb_server_create(m.ctypes.data, m.size, ctypes.byref(cfg), ctypes.byref(h)))
        self._h, self._keep, self.moduli = h, {}, [int(x) for x in m]

    @staticmethod
    def _addr(x):
        if hasattr(x, "data_ptr"):
            return x.data_ptr()
        return x.ctypes.data

    def submit(self, a, b, out, log_n, n_limbs, first_modulus=0):
        i = _u64()
        _check(lib().nttb_server_submit(self._h, self._addr(a), self._addr(b), self._addr(out), log_n, n_limbs,
                                        first_modulus, ctypes.byref(i)))
        self._keep[int(i.value)] = (a, b, out)
        return int(i.value)

    def submit_ntt(self, x, out, log_n, n_limbs, first_modulus=0, inverse=False):
        """Queues the forward (or inverse) transform of x per limb; result in out."""
        i = _u64()
        _check(lib().nttb_server_submit_ntt(self._h, self._addr(x), self._addr(out), log_n, n_limbs, first_modulus,
                                            int(inverse), ctypes.byref(i)))
        self._keep[int(i.value)] = (x, out)
        return int(i.value)

    def submit_device(self, kind, a, b, out, log_n, n_limbs, first_modulus=0):
        """Queues a request whose operands and result are CUDA tensors on the
        server's device: kind "mul" (out = a * b), "forward" or "inverse"
        (out = the transform of a; b unused)."""
        k = {"mul": 0, "forward": 1, "inverse": 2}[kind]
        i = _u64()
        _check(lib().nttb_server_submit_device(self._h, k, a.data_ptr(), b.data_ptr() if b is not None else None,
                                               out.data_ptr(), log_n, n_limbs, first_modulus, ctypes.byref(i)))
        self._keep[int(i.value)] = (a, b, out)
        return int(i.value)

    def wait(self, rid, timeout=60.0):
        lat = ctypes.c_double()
        try:
            _check(lib().nttb_server_wait(self._h, rid, timeout, ctypes.byref(lat)))
        finally:
            self._keep.pop(rid, None)
        return lat.value

    def drain(self, timeout=600.0):
        _check(lib().nttb_server_drain(self._h, timeout))

    def stats(self):
        st = ServerStats()
        _check(lib().nttb_server_stats(self._h, ctypes.byref(st)))
        return {f: int(getattr(st, f)) for f, _ in st._fields_}

    def latencies(self, reset=False):
        import numpy as np
        n = _u64()
        _check(lib().nttb_server_latencies(self._h, None, 0, ctypes.byref(n), 0))
        out = np.zeros(max(1, n.value), dtype=np.float64)
        _check(lib().nttb_server_latencies(self._h, out.ctypes.data, out.size, ctypes.byref(n), int(reset)))
        return out[:n.value]

    def close(self):
        if getattr(self, "_h", None):
            lib().nttb_server_destroy(self._h)
            self._h = None
            self._keep.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ------------------------------------------------------------ K-limb path
def klimb_forward(K, d_data, d_tw, log_n, prime_limbs, np_, stream=None):
    """nttb_klimb_forward: in-place forward NTT of 2^log_n K-limb Montgomery
    residues (K uint32 words of 24-bit limbs each) with twiddle table d_tw."""
    p = (ctypes.c_uint32 * K)(*[int(v) for v in prime_limbs])
    _check(lib().nttb_klimb_forward(K, _ptr(d_data), _ptr(d_tw), 1 << log_n, log_n, p, np_, _stream(stream)))


def klimb_neg_inv24(p0):
    """-p^-1 mod 2^24 from the lowest limb (the np argument)."""
    return (-pow(int(p0), -1, 1 << 24)) % (1 << 24)


# ------------------------------------------------------------- accounting
def launch_count():
    """Kernel launches issued by the library so far."""
    c = _u64()
    _check(lib().nttb_launch_count(ctypes.byref(c)))
    return int(c.value)


def device_errors(clear=True):
    """Error bits raised by bounded device waits (0 = none)."""
    f = _u32()
    _check(lib().nttb_device_errors(ctypes.byref(f), int(clear)))
    return int(f.value)


def bounds_errors(clear=True):
    """(enabled, flags) of the NTT_DEBUG_BOUNDS build's range checks
    (nttb_bounds_errors); enabled is False in the release build."""
    f, e = _u32(), _int()
    _check(lib().nttb_bounds_errors(ctypes.byref(f), ctypes.byref(e), int(clear)))
    return bool(e.value), int(f.value)


PHASES = ["mma_wait", "tmem_load", "gate", "part_sync_send", "level2_mma", "stage_end_sync", "stages",
          "cta_lifetime", "cta_startup", "ctas"]


def phase_profile(clear=True):
    """(enabled, {phase: cycles}) of the INT8 cluster kernel's phase counters
    (nttb_phase_profile; the NTT_PHASE_PROFILE build, NTT_B200_LIB=phase)."""
    v, e = (_u64 * 16)(), _int()
    _check(lib().nttb_phase_profile(v, ctypes.byref(e), int(clear)))
    return bool(e.value), {name: int(v[i]) for i, name in enumerate(PHASES)}


def profile_start():
    _check(lib().nttb_profile_start())


def profile_stop():
    """Stops per-launch event timing; returns {kernel: (launches, total_ms)}."""
    n = _u32()
    _check(lib().nttb_profile_stop(ctypes.byref(n)))
    out = {}
    buf = ctypes.create_string_buffer(128)
    for i in range(n.value):
        la, ms = _u64(), ctypes.c_double()
        _check(lib().nttb_profile_read(i, buf, 128, ctypes.byref(la), ctypes.byref(ms)))
        out[buf.value.decode()] = (int(la.value), float(ms.value))
    return out


# ----------------------------------------------------------------- host math
def create_params(q, n):
    p = _Params()
    _check(lib().nttb_create_params(q, n, ctypes.byref(p)))
    return {k: int(getattr(p, k)) for k, _ in _Params._fields_}


def find_primitive_root(q, n):
    w = _u64()
    _check(lib().nttb_find_primitive_root(q, n, ctypes.byref(w)))
    return int(w.value)


def find_psi(q, n):
    w = _u64()
    _check(lib().nttb_find_psi(q, n, ctypes.byref(w)))
    return int(w.value)


def host_ntt(data_np, q, inverse=False):
    """ntt_host equivalent on a numpy uint64 array (in place, returns it)."""
    import numpy as np
    assert data_np.dtype == np.uint64 and data_np.flags.c_contiguous
    p = _Params()
    _check(lib().nttb_create_params(q, data_np.size, ctypes.byref(p)))
    _check(lib().nttb_host_ntt(data_np.ctypes.data, data_np.size, ctypes.byref(p), int(inverse)))
    return data_np


def generate_primes(bits, two_adicity, count):
    import numpy as np
    out = np.zeros(count, dtype=np.uint64)
    _check(lib().nttb_generate_primes(bits, two_adicity, count, out.ctypes.data))
    return [int(x) for x in out]


# ------------------------------------------------------------------- plans
class Plan:
    """Single-modulus plan over uint64 words (backs the drop-in NTTConfig)."""

    def __init__(self, n, q):
        h = _vp()
        _check(lib().nttb_plan_create(n, q, ctypes.byref(h)))
        self._h = h
        self.n, self.q = n, q

    def info(self):
        i = _PlanInfo()
        _check(lib().nttb_plan_get_info(self._h, ctypes.byref(i)))
        return i

    def transform(self, data, batch=1, inverse=False, engine="auto", stream=None):
        _check(lib().nttb_u64_transform(self._h, _ptr(data), batch, int(inverse), _engine(engine), _stream(stream)))

    def four_step(self, data, inverse=False, stream=None):
        _check(lib().nttb_u64_four_step(self._h, _ptr(data), int(inverse), _stream(stream)))

    def rowmaj_forward(self, data, stream=None):
        _check(lib().nttb_u64_rowmaj_forward(self._h, _ptr(data), _stream(stream)))

    def pretransposed_transform(self, data, n1, inverse=False, stream=None):
        """Transform in the RowMaj pre-transposed layout pre[b*n1 + a] = x[a*n2 + b], in place."""
        _check(lib().nttb_u64_pretransposed_transform(self._h, _ptr(data), n1, int(inverse), _stream(stream)))

    def pointwise_mul(self, out, a, b, stream=None):
        _check(lib().nttb_u64_pointwise_mul(self._h, _ptr(out), _ptr(a), _ptr(b), _stream(stream)))

    def close(self):
        if getattr(self, "_h", None):
            lib().nttb_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def transpose_u64(dst, src, rows, cols, stream=None):
    _check(lib().nttb_u64_transpose(_ptr(dst), _ptr(src), rows, cols, _stream(stream)))


def bit_reverse_u64(data, n, stream=None):
    _check(lib().nttb_u64_bit_reverse(_ptr(data), n, _stream(stream)))


class RnsPlan:
    """Batched RNS plan over uint32 residues, layout [poly][limb][n]."""

    def __init__(self, log_n, moduli, negacyclic=False):
        import numpy as np
        m = np.ascontiguousarray(moduli, dtype=np.uint64)
        h = _vp()
        _check(lib().nttb_rns_plan_create(log_n, m.ctypes.data, m.size, NEGACYCLIC if negacyclic else 0,
                                          ctypes.byref(h)))
        self._h = h
        self.log_n, self.n, self.moduli, self.negacyclic = log_n, 1 << log_n, [int(x) for x in m], negacyclic

    def transform(self, dst, src, n_polys, inverse=False, engine="auto", stream=None):
        _check(lib().nttb_rns_transform(self._h, _ptr(dst), _ptr(src), n_polys, int(inverse), _engine(engine),
                                        _stream(stream)))

    def pointwise_mul(self, out, a, b, n_polys, stream=None):
        _check(lib().nttb_rns_pointwise_mul(self._h, _ptr(out), _ptr(a), _ptr(b), n_polys, _stream(stream)))

    def forward_inverse(self, data, n_polys, engine="auto", stream=None):
        """Forward then inverse in place (one persistent launch on the INT8 engine)."""
        _check(lib().nttb_rns_forward_inverse(self._h, _ptr(data), n_polys, _engine(engine), _stream(stream)))

    def stream_host(self, h_src, h_dst, n_polys, n_batches, mode="forward_inverse", engine="auto", stream=None):
        """Host-resident batches through the GPU (nttb_rns_stream_host): h_src,
        h_dst are pinned CPU tensors or numpy arrays of n_batches * n_polys *
        n_limbs * n words; mode "forward", "inverse" or "forward_inverse".
        Asynchronous on `stream`."""
        m = {"forward": 0, "inverse": 1, "forward_inverse": 2}[mode]
        _check(lib().nttb_rns_stream_host(self._h, _ptr(h_src), _ptr(h_dst), n_polys, n_batches, m, _engine(engine),
                                          _stream(stream)))

    def transform_noalloc(self, data, n_polys, inverse=False, stream=None):
        """In-place transform that allocates no device memory (static scratch;
        see nttb_rns_transform_noalloc in include/ntt_b200.h)."""
        _check(lib().nttb_rns_transform_noalloc(self._h, _ptr(data), n_polys, int(inverse), _stream(stream)))

    def close(self):
        if getattr(self, "_h", None):
            lib().nttb_rns_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class WidePlan:
    """Plan for moduli below 2^62, residues stored as uint64."""

    def __init__(self, log_n, moduli, negacyclic=False):
        import numpy as np
        m = np.ascontiguousarray(moduli, dtype=np.uint64)
        h = _vp()
        _check(lib().nttb_wide_plan_create(log_n, m.ctypes.data, m.size, NEGACYCLIC if negacyclic else 0,
                                           ctypes.byref(h)))
        self._h = h
        self.log_n, self.n, self.moduli = log_n, 1 << log_n, [int(x) for x in m]

    def transform(self, dst, src, n_polys, inverse=False, engine="auto", stream=None):
        """engine "auto" (the INT8 byte-plane engine where it serves the plan),
        "int8" or "scalar" (nttb_wide_transform_engine)."""
        _check(lib().nttb_wide_transform_engine(self._h, _ptr(dst), _ptr(src), n_polys, int(inverse), _engine(engine),
                                                _stream(stream)))

    def close(self):
        if getattr(self, "_h", None):
            lib().nttb_wide_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
