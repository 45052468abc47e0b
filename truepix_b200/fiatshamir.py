"""Drop-in for the reference prover's Fiat-Shamir transcript
(TruePix-main/libTruePix/fiatshamir.py, class FiatShamir), backed by the
library's transcript (tp_fs_*, include/native_fp2.h).

Same constructor and methods (put / take with the io and trans queues,
hash_update, hash_append, rand_scalar, rand_ext, to_string / from_string,
proof_size, unpack_proof), same bytes absorbed and the same challenges for
q = 2^61 - 1 with the binary encoding (fiatshamir.py:101-138). put() also takes
a 1-D numpy integer array, absorbed as the list of its values (the circuit
outputs of truepix_b200.frame.circuit_outputs, copied to the host). In addition the
running state is a 120-byte buffer (`state()` / `set_state()`): a transcript
begun here can continue on the device, one state per frame, where the batched
rounds put their claims and draw their challenges (tp_fs_*_dev,
tp_vole_round_dev, truepix_b200.frame.BatchFrameProver), and come back.
"""
from __future__ import annotations

import array
import bz2
import ctypes
import pickle
import struct
from collections import deque

import numpy as np

from . import native

P61 = (1 << 61) - 1
_M64 = (1 << 64) - 1


def _is_fp2(x) -> bool:
    return hasattr(x, "real") and hasattr(x, "imag") and not isinstance(x, (int, float, complex))


def _flatten(vals):
    """util.flatten_iter: lists and tuples (and the native Fp2 buffers) recursively"""
    for v in vals:
        if isinstance(v, (list, tuple)) or type(v).__name__ == "Fp2Buf":
            yield from _flatten(v)
        else:
            yield v


class FiatShamir:
    VERSION = 4
    VERSION_FP2 = 5
    ndb = None
    rvstart = None
    rvend = None
    wDiv = None
    protocol = "truepix"

    def __init__(self, q, protocol="truepix", fp2_type=None):
        """q must be 2^61 - 1 (the only field TruePix uses; the library's draws
        take 61-bit values). fp2_type builds rand_ext's result from (real, imag,
        q): the reference's Fp2 when libTruePix is importable, else a pair."""
        if q != P61:
            raise ValueError("the library transcript serves q = 2^61 - 1 only")
        self.q = q
        self.protocol = protocol
        self.lib = native.gkr(require_device=False)
        self._st = ctypes.create_string_buffer(self.lib.tp_fs_state_bytes())
        native.check(self.lib, self.lib.tp_fs_init(self._st, str(protocol).encode("utf-8")), "tp_fs_init")
        self.io = deque()
        self.trans = deque()
        self.can_put = True
        if fp2_type is None:
            try:
                from libTruePix.extfield import Fp2 as fp2_type
            except ImportError:
                fp2_type = None
        self._fp2 = fp2_type

    @property
    def rnum(self) -> int:
        """rand_scalar's counter (in the state after the SHA-256 words, the
        pending block and the byte count)"""
        return struct.unpack_from("<Q", self._st.raw, 104)[0]

    # ---- the state, for the device ----
    def state(self) -> bytes:
        """The running transcript state (tp_fs_state_bytes() bytes)."""
        return self._st.raw

    def set_state(self, raw: bytes) -> None:
        if len(raw) != len(self._st.raw):
            raise ValueError("transcript state of %d bytes expected" % len(self._st.raw))
        ctypes.memmove(self._st, raw, len(raw))

    # ---- absorbing ----
    def _absorb(self, b: bytes) -> None:
        if b:
            native.check(self.lib, self.lib.tp_fs_absorb(self._st, b, len(b)), "tp_fs_absorb")

    def hash_update(self, vals):
        if isinstance(vals, np.ndarray):
            self._hash_array(vals)
            return
        if isinstance(vals, list) and vals and type(vals[0]) is int:
            try:
                a = array.array("Q", vals)
            except (TypeError, OverflowError):
                a = None
            if a is not None:
                self._absorb(b"\x01" + struct.pack("<I", len(a)) + a.tobytes())
                return
        buf = bytearray()
        for elm in _flatten(vals):
            if type(elm) is int:
                buf += b"\x02" + struct.pack("<Q", elm & _M64)
            elif _is_fp2(elm):
                buf += b"\x03" + struct.pack("<QQ", int(elm.real) & _M64, int(elm.imag) & _M64)
            elif isinstance(elm, str):
                b = elm.encode("utf-8")
                buf += b"\x04" + struct.pack("<I", len(b)) + b
            elif elm is None:
                buf += b"\x05"
            else:
                raise TypeError("unsupported FS element: %r" % (type(elm),))
        self._absorb(bytes(buf))

    def _hash_array(self, a: np.ndarray) -> None:
        """A 1-D integer array absorbs as the list of its values would
        (a frame's circuit outputs, 2^23 values at 1080p, without a Python list)."""
        if a.ndim != 1 or a.dtype.kind not in "iu":
            raise TypeError("unsupported FS array: %r %r" % (a.dtype, a.shape))
        if a.size == 0:
            return
        if a.dtype.kind == "i" and (a < 0).any():
            self.hash_update(a.tolist())
            return
        a = np.ascontiguousarray(a.astype(np.uint64, copy=False))
        native.check(self.lib, self.lib.tp_fs_put_u64s(self._st, a.ctypes.data, a.size), "tp_fs_put_u64s")

    def hash_append(self, elm):
        self.hash_update([elm])

    def put(self, vals, is_io=False):
        if not self.can_put:
            raise AssertionError("Cannot put values into an input FS transcript")
        call_items = isinstance(vals, dict)
        if not call_items and not isinstance(vals, (list, np.ndarray)):
            vals = [vals]
        (self.io if is_io else self.trans).append(vals)
        self.hash_update(list(vals.items()) if call_items else vals)

    def take(self, take_io=False):
        if self.can_put:
            raise AssertionError("Cannot take values from an output FS transcript")
        vals = self.io.popleft() if take_io else self.trans.popleft()
        self.hash_update(list(vals.items()) if isinstance(vals, dict) else vals)
        return vals

    # ---- drawing ----
    def rand_scalar(self) -> int:
        out = ctypes.c_uint64()
        native.check(self.lib, self.lib.tp_fs_rand_scalar(self._st, ctypes.byref(out)), "tp_fs_rand_scalar")
        return out.value

    def rand_ext(self, label="chal"):
        re, im = ctypes.c_uint64(), ctypes.c_uint64()
        native.check(self.lib, self.lib.tp_fs_rand_ext(self._st, str(label).encode("utf-8"), ctypes.byref(re),
                                                       ctypes.byref(im)), "tp_fs_rand_ext")
        if self._fp2 is not None:
            return self._fp2(re.value, im.value, self.q)
        return (re.value, im.value)

    def digest(self) -> bytes:
        """hash.digest() of the running state"""
        d = ctypes.create_string_buffer(32)
        native.check(self.lib, self.lib.tp_fs_digest(self._st, d), "tp_fs_digest")
        return d.raw

    def hexdigest(self) -> str:
        return self.digest().hex()

    # ---- the proof container (fiatshamir.py:164-237) ----
    @classmethod
    def from_string(cls, string, protocol="truepix"):
        (q, iovals, tvals, ndb, rvstart, rvend, wDiv) = cls.unpack_proof(string)
        ret = cls(q, protocol=protocol)
        ret.can_put = False
        ret.io.extend(iovals)
        ret.trans.extend(tvals)
        ret.ndb, ret.rvstart, ret.rvend, ret.wDiv = ndb, rvstart, rvend, wDiv
        return ret

    @classmethod
    def proof_size(cls, string):
        (_, _, tvals, _, _, _, _) = cls.unpack_proof(string)
        nelems = len(list(_flatten(tvals)))
        return nelems, len(bz2.compress(pickle.dumps(tvals, -1)))

    @classmethod
    def unpack_proof(cls, string):
        (q, iovals, tvals, ndb, rvstart, rvend, wDiv, version) = pickle.loads(string)
        assert version == cls.VERSION, "Version: expected %d, got %d" % (cls.VERSION, version)
        return q, iovals, tvals, ndb, rvstart, rvend, wDiv

    def to_string(self, full=True):
        if full:
            return pickle.dumps((self.q, list(self.io), list(self.trans), self.ndb, self.rvstart, self.rvend,
                                 self.wDiv, self.VERSION), -1)
        return pickle.dumps(list(self.trans), -1)
