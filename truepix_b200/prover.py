"""The reference prover's proof of a frame (TruePix-main/libTruePix/
circuitnizkvec_vole.py:265-500, CircuitProverNIZK.run, and the zero-knowledge
variant circuitnizkvec_vole_ZK.py:293-520, TruePix's default) for the one-layer
TruePix circuits, with every step after the transcript's IO prefix on the device:

  host    put(pid), put(muxbits = None, io), put(["private_input_omitted", n], io),
          put(outputs, io), put(commit_binding(manifest)), z1 / z2 = rand_ext(...)
          (:277-375; the 64 MiB output vector of a 1080p frame is absorbed by the
          library's host transcript with the x86 SHA extensions)
  device  the circuit's output vector (tp_circuit_outputs_pixels_dev), the gate
          weights eq(z1, g) and beta (native_fp2_compute_beta, tp_compute_beta_*),
          the VOLE-committed early rounds (BatchFrameProver.prove), the late rounds,
          line and closing proofs (BatchFrameProver.prove_late), each frame's
          transcript and VOLE state carried from round to round in device memory
  host    the proof container: the values the device put, in the reference's
          trans-queue order, and FiatShamir.to_string()

The inputs the reference reads from files are taken as arguments: the VOLE
correlations (read_vole_prover_file reads the reference's binary prover file,
ExtVOLEGen.py:25-50, 130-186) and the Orion commitment manifest
(commit_binding, fp2_link.py:487-504). One VOLE repetition (defs.py:14).
"""
from __future__ import annotations

import concurrent.futures
import ctypes
import json
import math
import os
import pickle
import struct

import numpy as np

from . import native
from .fiatshamir import FiatShamir, P61

PROTOCOL_ID = "truepix"
LAYOUT_ID = "copy-major-384-const128-pad512-v1"
MANIFEST_INT_FIELDS = ("copies", "padded_copies", "copy_size", "padded_copy_size", "const_idx", "const_val", "n",
                       "lg_n")


class Fp2Value:
    """An Fp2 proof value (real, imag) when the reference's Fp2 class is not importable."""
    __slots__ = ("real", "imag", "p")

    def __init__(self, real, imag, p=P61):
        self.real, self.imag, self.p = int(real) % p, int(imag) % p, p

    def __eq__(self, other):
        return (self.real, self.imag) == (int(other.real), int(other.imag))

    def __hash__(self):
        return hash((self.real, self.imag))

    def __repr__(self):
        return "Fp2(%d, %d)" % (self.real, self.imag)


def commit_binding(manifest: dict) -> list:
    """fp2_link.commit_binding: what the transcript absorbs of the Orion commitment"""
    return (["orion-commit", PROTOCOL_ID, LAYOUT_ID, 1 if manifest.get("zk", True) else 0]
            + [int(manifest[f]) for f in MANIFEST_INT_FIELDS]
            + [manifest["masked_root"], manifest.get("mask_root") or ""])


def commit_manifest(layout, masked_root: str, mask_root: str = "", zk: bool = True) -> dict:
    """The manifest the reference's commit phase writes (truepix_gkr.h:391-418,
    with the layout of make_layout :106-150) for a frame committed in `layout`
    (truepix_b200.frame.FrameLayout); roots as root_hex strings
    (FrameCommitter.root_hex)."""
    n = layout.padded_copies * layout.n_wires
    return dict(protocol=PROTOCOL_ID, layout=LAYOUT_ID, zk=bool(zk), copies=layout.copies,
                padded_copies=layout.padded_copies, copy_size=layout.copy_size, padded_copy_size=layout.n_wires,
                const_idx=layout.const_idx, const_val=layout.const_val, n=n, lg_n=n.bit_length() - 1,
                masked_root=masked_root, mask_root=mask_root if zk else (mask_root or ""))


def manifests_of(committer) -> list:
    """commit_manifest of every frame of a truepix_b200.orion.FrameCommitter whose
    commits have completed"""
    out = []
    for f, L in enumerate(committer.layouts):
        mask = committer.hex(committer.mask_root(f)) if committer.zk else ""
        out.append(commit_manifest(L, committer.root_hex(f), mask, committer.zk))
    return out


def write_point_file(path: str, point) -> tuple:
    """fp2_link.write_point_file: the input point for the Orion open phase, as JSON
    and as the plain-text companion the Orion binaries read ("<count>" then one
    "<real> <imag>" line per coordinate). point: Fp2 values or (real, imag) pairs.
    Returns (json path, text path)."""
    pairs = [[int(x.real), int(x.imag)] if hasattr(x, "real") else [int(x[0]), int(x[1])] for x in point]
    with open(path, "w") as fh:
        json.dump({"protocol": PROTOCOL_ID, "field": "fp2-mersenne61", "layout": LAYOUT_ID, "point": pairs}, fh,
                  indent=2)
    txt = path if path.endswith(".txt") else os.path.splitext(path)[0] + ".txt"
    with open(txt, "w") as fh:
        fh.write("%d\n" % len(pairs))
        for re, im in pairs:
            fh.write("%d %d\n" % (re, im))
    return path, txt


def read_vole_prover_file(path: str):
    """The reference's binary VOLE prover file ("EVOL", version 1, role 1): the
    correlations u, v as uint64 [n, 2] (real, imag). One repetition."""
    head = struct.Struct("<4sIIIIQ")
    with open(path, "rb") as fh:
        raw = fh.read()
    if len(raw) < head.size:
        raise ValueError("%s: truncated VOLE file" % path)
    magic, version, role, reps, n, prime = head.unpack_from(raw, 0)
    if magic != b"EVOL" or version != 1 or role != 1:
        raise ValueError("%s: not a version-1 VOLE prover file" % path)
    if reps != 1 or prime != P61:
        raise ValueError("%s: one repetition over 2^61 - 1 expected (got %d, %d)" % (path, reps, prime))
    if len(raw) != head.size + 4 * 8 * n:
        raise ValueError("%s: truncated VOLE file" % path)
    a = np.frombuffer(raw, np.uint64, count=4 * n, offset=head.size).reshape(4, n)
    return np.stack([a[0], a[1]], axis=1).copy(), np.stack([a[2], a[3]], axis=1).copy()


class LayerTranscript:
    """One frame's transcript and proof container (the reference's FiatShamir with
    its io and trans queues)."""

    def __init__(self, pid: int, fp2_type=None):
        self.fs = FiatShamir(P61, protocol=PROTOCOL_ID, fp2_type=fp2_type)
        self.F = self.fs._fp2 or Fp2Value
        self.pid = int(pid)
        self.final_input_point = None
        self.final_input_tag = None

    def _f(self, pair):
        return self.F(int(pair[0]), int(pair[1]), P61)

    def io_prefix(self, outvals: np.ndarray, n_inputs: int, binding: list, n_out_bits: int, n_copy_bits: int):
        """circuitnizkvec_vole.py:277-375: the puts before the GKR point and the
        point's draws; returns (z1, z2) as (real, imag) pairs"""
        fs = self.fs
        fs.put(self.pid)
        fs.put(None, True)
        fs.put(["private_input_omitted", int(n_inputs)], True)
        fs.put(outvals, True)
        fs.put(binding)
        pair = lambda x: (int(x.real), int(x.imag)) if hasattr(x, "real") else (int(x[0]), int(x[1]))
        z1 = [pair(fs.rand_ext("z1-%d" % i)) for i in range(n_out_bits)]
        z2 = [pair(fs.rand_ext("z2-%d" % i)) for i in range(n_copy_bits)]
        return z1, z2

    def record(self, early, late, closing, point, tag, zk: bool = False) -> None:
        """Append the values the device put to the trans queue in the reference's
        order (early: [rounds][5] = four d, the equality value; late: [rounds][4];
        closing: the closing values, n + 10, or n + 15 for the zero-knowledge
        prover; point, tag: the input point and tag)."""
        t = self.fs.trans
        F = self.F
        tl = lambda a: a.tolist() if hasattr(a, "tolist") else [[int(v) for v in x] for x in a]
        for rnd in list(early) + list(late):
            for a, b in tl(rnd):          # plain ints first: far cheaper than numpy scalars one by one
                t.append([F(a, b, P61)])
        n = len(closing) - (15 if zk else 10)
        cl = [F(a, b, P61) for a, b in tl(closing)]
        t.append([(cl[0], cl[1])])
        for k in range(n):
            t.append([cl[2 + k]])
        t.append([(cl[n + 2], cl[n + 3])])
        k = n + 4
        if zk:       # circuitnizkvec_vole_ZK.py:224-240: the masks' commitments, then both product proofs
            t.append([(cl[k], cl[k + 1], cl[k + 2])])
            k += 3
        t.append([(cl[k], cl[k + 1])])
        k += 2
        if zk:
            t.append([(cl[k], cl[k + 1])])
            k += 2
        t.append([cl[k]])
        t.append([(cl[k + 1], cl[k + 2])])
        t.append(["gkr_input_point", [[int(a), int(b)] for a, b in point]])
        t.append([cl[k + 3]])
        self.final_input_point = [self._f(x) for x in point]
        self.final_input_tag = self._f(tag)

    def proof_bytes(self) -> bytes:
        """FiatShamir.to_string() as the reference writes it (io arrays as lists)"""
        fs = self.fs
        io = [v.tolist() if isinstance(v, np.ndarray) else v for v in fs.io]
        return pickle.dumps((fs.q, io, list(fs.trans), fs.ndb, fs.rvstart, fs.rvend, fs.wDiv, fs.VERSION), -1)


def gate_weights(lib, z1, n_gates: int) -> np.ndarray:
    """eq(z1, g) for g < n_gates (LSB first), uint64 [2, n_gates], computed on the device"""
    k = len(z1)
    zr = np.ascontiguousarray([a for a, _ in z1], np.uint64)
    zi = np.ascontiguousarray([b for _, b in z1], np.uint64)
    out_r = np.zeros(1 << k, np.uint64)
    out_i = np.zeros(1 << k, np.uint64)
    P = ctypes.POINTER(ctypes.c_uint64)
    lib.native_fp2_compute_beta(zr.ctypes.data_as(P), zi.ctypes.data_as(P), k, 1, 0, out_r.ctypes.data_as(P),
                                out_i.ctypes.data_as(P))
    native.check(lib, None, "native_fp2_compute_beta")
    return np.stack([out_r[:n_gates], out_i[:n_gates]])


def prove_frames(frames, layout, gate_type, in0, in1, pids, correlations, manifests, fp2_type=None,
                 stream=None, zk: bool = True, io_threads: int = 0):
    """Proofs of a batch of frames of one size and circuit.

    frames: uint8 device tensors (layout.copies * layout.copy_size bytes each);
    layout: truepix_b200.frame.FrameLayout; gate tables of the circuit; pids,
    correlations [(u, v) uint64 [count, 2]] (the same count for every frame) and
    commitment manifests per frame. zk: the zero-knowledge prover
    (circuitnizkvec_vole_ZK.py, TruePix's default), else circuitnizkvec_vole.py.
    io_threads: host threads absorbing the frames' output vectors (0: one per
    CPU). Returns one LayerTranscript per frame (proof_bytes() is the
    reference's proof)."""
    import torch
    from .frame import BatchFrameProver, circuit_outputs, pack_fp2
    lib = native.gkr()
    B = len(frames)
    dev = frames[0].device
    gt, i0, i1 = (np.ascontiguousarray(a, np.int32) for a in (gate_type, in0, in1))
    G = gt.size
    n_out_bits = (G - 1).bit_length()      # util.clog2 of the gate count
    nb = layout.n_copy_bits
    counts = {len(u) for u, _ in correlations}
    if len(counts) != 1:
        raise ValueError("every frame needs the same number of VOLE correlations")
    count = counts.pop()
    n_inputs = layout.padded_copies * layout.n_wires
    # IO prefix: circuit outputs on the device, absorbed on the host
    bufs = [circuit_outputs(f, layout, gt, i0, i1, stream=stream) for f in frames]
    if stream is not None:
        stream.synchronize()
    # each frame's output vector (64 MiB at 1080p) is one sequential SHA-256
    # chain; the frames' chains run on host threads (the library's transcript
    # calls release the interpreter lock)
    outs = [b.cpu().numpy().view(np.uint64) for b in bufs]
    tr = [LayerTranscript(pids[f], fp2_type) for f in range(B)]

    def prefix(f):
        return tr[f].io_prefix(outs[f], n_inputs, commit_binding(manifests[f]), n_out_bits, nb)

    workers = max(1, min(B, io_threads or os.cpu_count() or 1))
    if workers > 1:
        with concurrent.futures.ThreadPoolExecutor(workers) as pool:
            points = list(pool.map(prefix, range(B)))
    else:
        points = [prefix(f) for f in range(B)]
    z1s = [gate_weights(lib, z1, G) for z1, _ in points]
    z2s = [z2 for _, z2 in points]
    z2 = np.array(z2s, np.uint64).reshape(B, nb, 2)
    d_z2 = torch.from_numpy(pack_fp2(z2[..., 0].reshape(-1), z2[..., 1].reshape(-1))).to(dev)
    d_pt = torch.zeros(B * (nb + int(math.log2(layout.n_wires))) * 2, dtype=torch.int64, device=dev)
    states = torch.from_numpy(np.frombuffer(b"".join(t.fs.state() for t in tr), np.uint8).copy()).to(dev)
    vs = b""
    for _ in range(B):
        s = ctypes.create_string_buffer(lib.tp_vole_state_bytes())
        native.check(lib, lib.tp_vole_state_init(s, 0, None), "tp_vole_state_init")
        vs += s.raw
    u = np.stack([np.asarray(a, np.uint64) for a, _ in correlations])
    v = np.stack([np.asarray(b, np.uint64) for _, b in correlations])
    vole = dict(states=torch.from_numpy(np.frombuffer(vs, np.uint8).copy()).to(dev),
                u=torch.from_numpy(u.view(np.int64).reshape(-1).copy()).to(dev),
                v=torch.from_numpy(v.view(np.int64).reshape(-1).copy()).to(dev), count=count)
    bp = BatchFrameProver([layout] * B, gt, i0, i1, device=dev.index or 0, stream=stream)
    bp.prove(frames, z1s, d_z2, d_pt, None, transcripts=states, vole=vole)
    bp.prove_late(z1s, transcripts=states, vole=vole, zk=zk)
    if stream is not None:
        stream.synchronize()
    torch.cuda.synchronize(dev)
    nst, nvs = lib.tp_fs_state_bytes(), lib.tp_vole_state_bytes()
    raw_st = states.cpu().numpy().tobytes()
    raw_vs = vole["states"].cpu().numpy().tobytes()
    n = int(math.log2(layout.n_wires))
    early = bp.device_proof.cpu().numpy().view(np.uint64).reshape(nb, B, 5, 2)
    late = bp.late_proof.cpu().numpy().view(np.uint64).reshape(B, 2 * n, 4, 2)
    closing = bp.closing.cpu().numpy().view(np.uint64).reshape(B, n + (15 if zk else 10), 2)
    point = bp.input_point.cpu().numpy().view(np.uint64).reshape(B, n + nb, 2)
    tag = bp.input_tag.cpu().numpy().view(np.uint64).reshape(B, 2)
    for f in range(B):
        if struct.unpack_from("<I", raw_vs, f * nvs + 12)[0]:
            raise IndexError("frame %d: VOLE correlations ran out (%d given)" % (f, count))
        tr[f].record(early[:, f], late[f], closing[f], point[f], tag[f], zk=zk)
        tr[f].fs.set_state(raw_st[f * nst:(f + 1) * nst])
    return tr
