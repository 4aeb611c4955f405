"""bitz_b200: a B200-native BitZ SHA-256 prover.

Python mirror of the reference's prover-side interfaces over the C ABI of
libbitz_b200.so. Field elements are numpy uint64 arrays of shape (..., 2)
holding (lo, hi) in the reference's GF(2^128) basis.

- ``build_prover`` / ``ProverState``: crates/transcript/src/domain.rs:13,
  crates/transcript/src/prover.rs:10-84.
- ``post_gkr_prove``: crates/post_gkr/src/lib.rs:85 (post_gkr::prove).
- ``gkr_prove``: crates/gkr/src/lib.rs:24,785 (grand_product + gpgkr_prove).
- ``CircuitProofSystem``: tooling/cli/src/end_to_end.rs:150-336.
- ``batch_prove`` / ``ProveServer``: many proofs at once on prover lanes (no
  reference counterpart; the reference proves one statement per call).
"""
import ctypes

import numpy as np

from . import _lib


def _tuning():
    """The batched prover's tuned lane count and host-thread cap
    (bitz_b200/tuning.json, written by ``python -m bitz_b200.autotune``), or {}."""
    import json
    import os
    try:
        with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "tuning.json")) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


TUNING = _tuning()
if TUNING.get("lane_threads") and "BITZ_LANE_THREADS" not in __import__("os").environ:
    # read by the library when its first batch starts
    __import__("os").environ["BITZ_LANE_THREADS"] = str(int(TUNING["lane_threads"]))

__all__ = ["BitzError", "ProverState", "build_prover", "post_gkr_prove", "gkr_prove",
           "gkr_outputs", "device_count", "CircuitProofSystem", "Witness", "CommittedWitness",
           "wire_decode", "batch_prove", "ProveServer", "probe_kernel", "probe_read", "probe_kernels", "gf_peak",
           "l2_flush"]

_ERRORS = {
    1: "ArgumentError", 2: "ClaimDoesNotHold", 3: "Unsatisfied", 4: "Configuration",
    5: "CudaError", 6: "Internal", 7: "Scratch", 8: "VerifyError", 9: "MalformedProof",
    10: "NoDevice", 11: "Pending",
}
PENDING = 11


class BitzError(RuntimeError):
    """A non-zero status from the C ABI; ``code`` names the reference error variant."""

    def __init__(self, status, message):
        self.status = status
        self.code = _ERRORS.get(status, f"status{status}")
        super().__init__(f"{self.code}: {message}")


def _check(status):
    if status != 0:
        msg = _lib.load().bitz_last_error()
        raise BitzError(status, msg.decode() if msg else "")


def _u64(a):
    a = np.ascontiguousarray(a, dtype=np.uint64)
    return a, a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))


def device_count():
    return _lib.load().bitz_device_count()


def set_device(device: int):
    _check(_lib.load().bitz_set_device(device))


def launch_count() -> int:
    return int(_lib.load().bitz_launch_count())


def round_wait_stats():
    """(seconds the host has waited for round results on the default lane,
    number of waits) since the process started."""
    out = (ctypes.c_ulonglong * 2)()
    _check(_lib.load().bitz_round_wait_stats(out))
    return out[0] * 1e-9, int(out[1])


def gate_stats():
    """The device gate since the process started: lanes whose kernels may wait
    for their host thread hold it as resident stretches; device and pinned
    allocations wait until none is held. Returns a dict of the allocation and
    resident stretch counts and the seconds each kind waited."""
    out = (ctypes.c_ulonglong * 4)()
    _check(_lib.load().bitz_gate_stats(out))
    return {"allocs": int(out[0]), "alloc_wait_s": out[1] * 1e-9,
            "residents": int(out[2]), "resident_wait_s": out[3] * 1e-9}


class ProverState:
    """The prover transcript (crates/transcript/src/prover.rs:10)."""

    def __init__(self, session: bytes, instance: bytes):
        lib = _lib.load()
        self._lib = lib
        self._h = lib.bitz_transcript_new(session, len(session), instance, len(instance))
        if not self._h:
            raise BitzError(6, "transcript allocation failed")

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            self._lib.bitz_transcript_free(h)
            self._h = None

    @property
    def handle(self):
        return self._h

    def public_message(self, data: bytes):
        _check(self._lib.bitz_transcript_public(self._h, data, len(data)))

    def prover_message(self, data: bytes):
        _check(self._lib.bitz_transcript_prover(self._h, data, len(data)))

    def hint(self, data: bytes):
        _check(self._lib.bitz_transcript_hint(self._h, data, len(data)))

    def verifier_message_f128(self):
        out = np.zeros(2, dtype=np.uint64)
        _check(self._lib.bitz_transcript_challenge_f128(
            self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))))
        return out

    def grind(self, label: bytes, bits: int):
        _check(self._lib.bitz_transcript_grind(self._h, label, bits))

    def squeeze_prime(self, bits: int) -> int:
        buf = (ctypes.c_uint8 * 16)()
        _check(self._lib.bitz_transcript_prime(self._h, bits, buf))
        return int.from_bytes(bytes(buf), "little")

    def narg(self) -> bytes:
        n = self._lib.bitz_transcript_narg(self._h, None, 0)
        buf = (ctypes.c_uint8 * max(n, 1))()
        self._lib.bitz_transcript_narg(self._h, buf, n)
        return bytes(buf)[:n]

    def hints(self) -> bytes:
        n = self._lib.bitz_transcript_hints(self._h, None, 0)
        buf = (ctypes.c_uint8 * max(n, 1))()
        self._lib.bitz_transcript_hints(self._h, buf, n)
        return bytes(buf)[:n]


def build_prover(session: bytes, instance: bytes) -> ProverState:
    return ProverState(session, instance)


def post_gkr_prove(rows, cols, target, packed, security_bits, transcript: ProverState):
    """Runs the post-GKR sumcheck on the GPU; returns (point, value)."""
    rows, rp = _u64(rows)
    cols, cp = _u64(cols)
    packed, pp = _u64(packed)
    tgt, tp = _u64(target)
    log_rows = int(rows.shape[0]).bit_length() - 1
    log_cols = int(cols.shape[0]).bit_length() - 1
    point = np.zeros((log_rows + log_cols, 2), dtype=np.uint64)
    value = np.zeros(2, dtype=np.uint64)
    _check(_lib.load().bitz_post_gkr_prove(
        rp, log_rows, cp, log_cols, tp, pp, security_bits, transcript.handle,
        point.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)),
        value.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))))
    return point, value


def gkr_prove(row_images, columns, zeta, security_bits, transcript: ProverState):
    """Builds the product tree and runs the seven layer sumchecks; returns (point, claim)."""
    img, ip = _u64(row_images)
    cols, cp = _u64(columns)
    z, zp = _u64(zeta)
    log_cols = int(cols.shape[0]).bit_length() - 1
    point = np.zeros((log_cols + 7, 2), dtype=np.uint64)
    claim = np.zeros(2, dtype=np.uint64)
    _check(_lib.load().bitz_gkr_prove(
        ip, cp, log_cols, zp, security_bits, transcript.handle,
        point.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)),
        claim.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))))
    return point, claim


CIRCUITS = {"sha256-compression": 0, "sha256-chain": 1, "sha256-block-aligned": 2, "sha256-2kb": 3}


class CircuitProofSystem:
    """A prepared SHA-256 statement (tooling/cli/src/end_to_end.rs:150-336).

    ``inputs`` and ``outputs`` are 0/1 sequences in the statement's bit order
    (tooling/cli/src/circuits.rs:58-160); ``security_bits`` is 100 or 128.
    """

    def __init__(self, circuit: str, inputs, outputs, security_bits: int = 100):
        lib = _lib.load()
        self._lib = lib
        self._h = None
        inp = np.ascontiguousarray(inputs, dtype=np.uint8)
        out = np.ascontiguousarray(outputs, dtype=np.uint8)
        h = ctypes.c_void_p()
        _check(lib.bitz_system_new(CIRCUITS[circuit], inp.ctypes.data, inp.size, out.ctypes.data,
                                   security_bits, ctypes.byref(h)))
        self._h = h

    def __del__(self):
        if getattr(self, "_h", None):
            self._lib.bitz_system_free(self._h)
            self._h = None

    def stats(self):
        out = np.zeros(8, dtype=np.uint64)
        _check(self._lib.bitz_system_stats(self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))))
        keys = ["constraints", "assignment_bits", "committed_bits", "padded_committed_bits",
                "prime_bits", "pcs_security", "claim_log_cols", "compressions"]
        return dict(zip(keys, (int(x) for x in out)))

    def prove(self, witness=None, commitment=None, restage: bool = True):
        """Returns (proof bytes, times in ms).

        Without arguments: witness + commit + prove in one call (restage=False
        reuses the statement staged on the device at creation). With a
        Witness and its CommittedWitness (from ``witness`` and ``commit``):
        the prove stage alone, consuming both (end_to_end.rs:260); the times
        are then empty."""
        p = ctypes.POINTER(ctypes.c_uint8)()
        n = ctypes.c_size_t(0)
        if witness is not None or commitment is not None:
            if witness is None or commitment is None:
                raise BitzError(1, "prove takes both the witness and its commitment")
            wh, ch = witness._take(), commitment._take()
            _check(self._lib.bitz_prove(self._h, wh, ch, ctypes.byref(p), ctypes.byref(n)))
            data = ctypes.string_at(p, n.value)
            self._lib.bitz_free(p)
            return data, {}
        times = (ctypes.c_double * 4)()
        _check(self._lib.bitz_system_prove_ex(self._h, int(restage), ctypes.byref(p),
                                              ctypes.byref(n), times))
        data = ctypes.string_at(p, n.value)
        self._lib.bitz_free(p)
        return data, {"witness_ms": times[0], "commit_ms": times[1], "prove_ms": times[2],
                      "device_ms": times[3]}

    def witness(self, inputs):
        """CircuitProofSystem::witness (end_to_end.rs:215): the witness of
        ``inputs`` (0/1 per input bit), kept on the device."""
        inp = np.ascontiguousarray(inputs, dtype=np.uint8)
        h = ctypes.c_void_p()
        _check(self._lib.bitz_witness(self._h, inp.ctypes.data, inp.size, ctypes.byref(h)))
        return Witness(self._lib, h)

    def commit(self, witness):
        """CircuitProofSystem::commit (end_to_end.rs:248): commits the witness."""
        h = ctypes.c_void_p()
        _check(self._lib.bitz_commit(self._h, witness._handle(), ctypes.byref(h)))
        return CommittedWitness(self._lib, h)

    def verify(self, proof: bytes):
        """CircuitProofSystem::verify (end_to_end.rs:339-377) by this library's
        verifier; raises BitzError (MalformedProof or VerifyError, naming the
        failed check) unless the proof is accepted."""
        buf = (ctypes.c_uint8 * max(len(proof), 1)).from_buffer_copy(proof or b"\0")
        _check(self._lib.bitz_verify(self._h, buf, len(proof)))

    def witness_parts(self, f_words: int, h_words: int, rows: int):
        f = np.zeros(f_words, dtype=np.uint32)
        h = np.zeros(h_words, dtype=np.uint32)
        pr = np.zeros(3 * rows, dtype=np.int64)
        _check(self._lib.bitz_system_witness(self._h, f.ctypes.data, f.size, h.ctypes.data, h.size,
                                             pr.ctypes.data, pr.size))
        return f, h, pr


class _StagedHandle:
    """A witness or commitment held on the device between the staged calls."""

    _free = None

    def __init__(self, lib, h):
        self._lib = lib
        self._h = h

    def _handle(self):
        if not self._h:
            raise BitzError(1, "the handle was already consumed")
        return self._h

    def _take(self):
        h = self._handle()
        self._h = None
        return h

    def __del__(self):
        if getattr(self, "_h", None):
            getattr(self._lib, self._free)(self._h)
            self._h = None


class Witness(_StagedHandle):
    """CircuitProofSystem::witness's result (end_to_end.rs:215-243)."""
    _free = "bitz_witness_free"


class CommittedWitness(_StagedHandle):
    """CircuitProofSystem::commit's result (end_to_end.rs:248-255)."""
    _free = "bitz_committed_witness_free"


def wire_decode(data: bytes):
    """WireProof::from_bytes (crates/host/src/wire_proof.rs:109-140): returns
    (narg bytes, hint bytes); raises BitzError (MalformedProof) naming the
    reference's decoding error."""
    out = np.zeros(4, dtype=np.uint64)
    buf = (ctypes.c_uint8 * max(len(data), 1)).from_buffer_copy(data or b"\0")
    _check(_lib.load().bitz_wire_decode(buf, len(data),
                                        out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))))
    a, n, b, h = (int(x) for x in out)
    return data[a:a + n], data[b:b + h]


def gkr_outputs(row_images, columns):
    img, ip = _u64(row_images)
    cols, cp = _u64(columns)
    log_cols = int(cols.shape[0]).bit_length() - 1
    out = np.zeros((1 << log_cols, 2), dtype=np.uint64)
    _check(_lib.load().bitz_gkr_outputs(ip, cp, log_cols,
                                        out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))))
    return out


def batch_prove(systems, lanes=None):
    """Proves every CircuitProofSystem in ``systems`` on ``lanes`` concurrent
    prover lanes (the tuned count of bitz_b200/tuning.json when None, else
    16); returns (proofs, each proof's duration in ms)."""
    if lanes is None:
        lanes = int(TUNING.get("lanes", 16))
    lib = _lib.load()
    n = len(systems)
    hs = (ctypes.c_void_p * max(n, 1))(*[s._h.value for s in systems])
    ptrs = (ctypes.c_void_p * max(n, 1))()
    lens = (ctypes.c_size_t * max(n, 1))()
    lat = (ctypes.c_double * max(n, 1))()
    status = lib.bitz_batch_prove(hs, n, lanes, ptrs, lens, lat)
    proofs = []
    for i in range(n):
        if ptrs[i]:
            proofs.append(ctypes.string_at(ptrs[i], lens[i]))
            lib.bitz_free(ptrs[i])
        else:
            proofs.append(None)
    _check(status)
    return proofs, list(lat[:n])


class ProveServer:
    """Continuous-batching prove server over ``lanes`` prover lanes, admitting
    requests by padded-witness device footprint within ``hbm_budget`` bytes."""

    def __init__(self, lanes: int = 8, hbm_budget: int = 64 << 30, security_bits: int = 100):
        self._lib = _lib.load()
        h = ctypes.c_void_p()
        _check(self._lib.bitz_server_start(lanes, hbm_budget, security_bits, ctypes.byref(h)))
        self._h = h

    def submit(self, circuit: str, inputs, outputs) -> int:
        inp = np.ascontiguousarray(inputs, dtype=np.uint8)
        out = np.ascontiguousarray(outputs, dtype=np.uint8)
        t = ctypes.c_uint64(0)
        _check(self._lib.bitz_server_submit(self._h, CIRCUITS[circuit], inp.ctypes.data, inp.size,
                                            out.ctypes.data, ctypes.byref(t)))
        return t.value

    def poll(self, ticket: int, wait_ms: int = 0):
        """(proof bytes, latency ms) once done, else None; raises on failure."""
        p = ctypes.POINTER(ctypes.c_uint8)()
        n = ctypes.c_size_t(0)
        lat = ctypes.c_double(0)
        st = self._lib.bitz_server_poll(self._h, ticket, wait_ms, ctypes.byref(p), ctypes.byref(n),
                                        ctypes.byref(lat))
        if st == PENDING:
            return None
        _check(st)
        data = ctypes.string_at(p, n.value)
        self._lib.bitz_free(p)
        return data, lat.value

    def stats(self):
        out = np.zeros(6, dtype=np.uint64)
        _check(self._lib.bitz_server_stats(self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))))
        keys = ["submitted", "finished", "in_flight", "queued", "in_flight_bytes", "peak_in_flight"]
        return dict(zip(keys, (int(x) for x in out)))

    def stop(self):
        if getattr(self, "_h", None):
            _check(self._lib.bitz_server_stop(self._h))
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.stop()

    def __del__(self):
        try:
            self.stop()
        except Exception:
            pass


def probe_kernel(spec):
    """Times every launch of the probed kernels with CUDA events: None turns
    the probe off, "*" probes every instrumented kernel, else a
    comma-separated list of names. While on, every round is its own launch."""
    _check(_lib.load().bitz_probe_kernel(spec.encode() if spec else None))


def probe_read(kernel):
    """One probed kernel's totals: ms, algorithmic bytes, GF(2^128) products
    (gmuls reduced, wides unreduced, tables by the round challenge through its
    window table) and launches."""
    out = (ctypes.c_double * 5)()
    n = ctypes.c_ulonglong(0)
    _check(_lib.load().bitz_probe_read(kernel.encode(), out, ctypes.byref(n)))
    return {"ms": out[0], "bytes": out[1], "gmuls": out[2], "wides": out[3], "tables": out[4],
            "launches": n.value}


def probe_kernels():
    """Names of the probed kernels that launched since the probe was enabled."""
    lib = _lib.load()
    n = lib.bitz_probe_kernels(None, 0)
    buf = ctypes.create_string_buffer(n + 1)
    lib.bitz_probe_kernels(buf, n + 1)
    return [x for x in buf.value.decode().split(",") if x]


def gf_peak(kind: int) -> float:
    """Measured GF(2^128) products per second on this GPU: kind 0 reduced, 1
    unreduced (wide), 2 through a window table."""
    v = ctypes.c_double(0)
    _check(_lib.load().bitz_diag_gf_peak(kind, ctypes.byref(v)))
    return v.value


def l2_flush():
    """Evicts the L2 cache by overwriting a 256 MiB device buffer."""
    _check(_lib.load().bitz_l2_flush())
