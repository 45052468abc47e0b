"""Generate the golden fixtures for the Orion side of the path from the reference.

Runs the reference's own Orion sources, compiled by `make -C oracle ref` into
oracle/_ref/liborion_ref.so (TruePix-main/Orion/Orion_nonzk sources + the C
harness oracle/orion_ref_harness.cpp), on seeded inputs (tests/orionlib.py
`elements`, splitmix64-based) and stores the outputs in
tests/golden/orion_golden.npz:

  commit_<case>   32-byte Merkle roots of the Orion commit (linearPC.cpp:97-197),
                  incl. one 1080p frame in TruePix's layout (frameroot_1080)
  encode_<n>      SHA-256 digest of the expander codeword of one column
                  (linear_code_encode.h:17-72); full codeword for n = 64
  fft_<m>_<o>     digest of P(w^i), i < o, for m seeded coefficients
                  (RS_polynomial.cpp:46-130)
  ifft_<m>_<o>    digest of the m coefficients from o seeded evaluations
                  (RS_polynomial.cpp:132-206)
  rs_<L>          Merkle root and codeword digest of the rate-2^-5 RS commit
                  of 2^L elements (poly_commit.h:42-96, fri.cpp:36-123)
  fri*_<log M>    one FRI commit-phase step (fri::commit_phase_step, fri.cpp:316-420)
                  on a seeded interleaved witness of 2^log M x 64 elements: digest of
                  the next interleaved witness and its Merkle root
  virgo*_<p>_<n>_<bit>  one Virgo sumcheck update (zk_prover::sumcheck_phase<p>_update,
                  prover.cpp:576-644, 935-1006) of three seeded linear_poly
                  tables: digests of the folded tables and the round polynomial
  combine*_<N>    the tensor-product opening passes (linearPC.cpp:480-531,
                  569-571) run with the reference's primitives on its retained
                  codeword: combined codeword digest, its Merkle root, answer

and, from the zero-knowledge tree (TruePix-main/Orion/Orion_zk, built into
oracle/_ref/liborion_zk_ref.so with oracle/orion_zk_ref_harness.cpp), in
tests/golden/orion_zk_golden.npz:

and, in tests/golden/virgo_init_golden.npz (from oracle/_ref/liborion_ref.so):

  vinit*_<p>_<seed>  zk_prover::sumcheck_phase<p>_init (prover.cpp:246-570,
                  645-930) of a seeded layer (tests/orionlib.py virgo_layer: every
                  gate type, 2^length_g gates over 2^length_u values): digests
                  of V_mult_add, addV_array, add_mult_sum

  zk*_<case>      the commit phase of linearPC_multi_commit_zk on a seeded frame
                  (examples/multivariate_PC_test_commit.cpp:280-340): masked and
                  mask Merkle roots of commit_pair (linearPC.cpp:253-460) and the
                  digest of the mask polynomial (truepix_gkr.h:286-384)

Every reference call runs in a fresh spawned process: the reference keeps
global scratch state sized by its first call.

Run here (needs the reference checkout and `make -C oracle ref`):
    python tests/golden/gen_orion_golden.py          # both files
    python tests/golden/gen_orion_golden.py zk       # the ZK file only
    python tests/golden/gen_orion_golden.py vinit    # the Virgo init file only
"""
from __future__ import annotations

import ctypes
import multiprocessing as mp
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
from orionlib import (ORION_REF_LIB, ORION_ZK_REF_LIB, digest, virgo_layer, elements, frame_bytes, frame_elements,  # noqa: E402
                      virgo_inputs)

V = ctypes.c_void_p

COMMIT_CASES = [  # (name, N, seed, kind)
    ("r13", 1 << 13, 1, "random"), ("zero13", 1 << 13, 0, "zero"), ("max13", 1 << 13, 0, "max"),
    ("small14", 1 << 14, 7, "small"), ("r14", 1 << 14, 2, "random"), ("r15", 1 << 15, 3, "random"),
    ("r16", 1 << 16, 4, "random"), ("r18", 1 << 18, 5, "random"), ("r20", 1 << 20, 6, "random"),
    ("c100", 128 * 100, 8, "random"), ("c13", 128 * 13, 9, "random"), ("c1", 128, 10, "random"),
    ("c1000", 128 * 1000, 11, "random"),
]
# one 1080p frame (TruePix layout: 16,200 copies of 384 bytes, gray constant 128
# at wire 384, 512 wires, padded to 16,384 copies -> N = 2^23)
FRAME = dict(copies=16200, cs=384, W=512, const_idx=384, const_val=128, padded=16384, seed=12)
ENCODE_CASES = [1, 13, 14, 64, 100, 1000, 8192, 65536]
FFT_CASES = [(1, 1), (1, 8), (2, 2), (8, 8), (4, 16), (16, 256), (1024, 1024), (256, 4096),
             (1 << 12, 1 << 17), (1 << 16, 1 << 16), (1 << 20, 1 << 20)]
RS_CASES = [6, 7, 10, 13, 16, 18]
COMBINE_CASES = [(1 << 14, 21), (128 * 100, 22), (1 << 18, 23)]   # (N, seed)
FRI_CASES = [(2, 41), (3, 42), (5, 43), (10, 44), (16, 45)]   # (log2 M, seed)
VIRGO_CASES = [(1, 2, 0, 31), (1, 2, 1, 32), (1, 16, 1, 33), (2, 16, 0, 34), (1, 1 << 10, 1, 35),
               (2, 1 << 14, 1, 36), (1, 1 << 18, 1, 37), (2, 1 << 18, 0, 38)]   # (phase, total_uv, bit, seed)

# (name, copies, copy_size, const_idx, const_val, padded copies, pixel seed, mask seed)
ZK_CASES = [
    ("gray40", 40, 384, 384, 128, 64, 3, 0x0123456789ABCDEF), ("crop33", 33, 385, -1, 0, 64, 4, 99),
    ("inv7", 7, 384, 384, 255, 8, 5, 1), ("one", 1, 384, 384, 128, 1, 6, 0),
    ("all512", 16, 512, -1, 0, 16, 7, 0xFFFFFFFFFFFFFFFF), ("gray1000", 1000, 384, 384, 128, 1024, 8, 42),
    ("zk1080", 16200, 384, 384, 128, 16384, 12, 0x5EED5EED5EED5EED),
]


def _ref():
    lib = ctypes.CDLL(ORION_REF_LIB)
    lib.ref_commit.argtypes = [V, ctypes.c_longlong, V, V]
    lib.ref_fft.argtypes = [V, ctypes.c_int, ctypes.c_int, V]
    lib.ref_ifft.argtypes = [V, ctypes.c_int, ctypes.c_int, V]
    lib.ref_rs_commit.argtypes = [V, ctypes.c_int, V, V]
    lib.ref_encode.argtypes = [V, ctypes.c_longlong, V]
    lib.ref_combine.argtypes = [V, ctypes.c_longlong, V, V, V, V, V]
    lib.ref_virgo_update.argtypes = [ctypes.c_int, V, V, V, ctypes.c_int, V, ctypes.c_int, V, V, V, V]
    lib.ref_fri_step.argtypes = [V, ctypes.c_int, V, V, V]
    lib.ref_encode_len.argtypes = [ctypes.c_longlong]
    lib.ref_encode_len.restype = ctypes.c_longlong
    return lib


def _commit(args):
    n, seed, kind = args
    src = elements(seed, n, kind)
    root = ctypes.create_string_buffer(32)
    hx = ctypes.create_string_buffer(80)
    _ref().ref_commit(V(src.ctypes.data), n, root, hx)
    return root.raw, hx.value


def _commit_frame(_):
    src = frame_elements(frame_bytes(FRAME["seed"], FRAME["copies"] * FRAME["cs"]), **{
        k: FRAME[k] for k in ("copies", "cs", "W", "const_idx", "const_val", "padded")})
    root = ctypes.create_string_buffer(32)
    hx = ctypes.create_string_buffer(80)
    _ref().ref_commit(V(src.ctypes.data), src.size // 2, root, hx)
    return root.raw


def _encode(n):
    lib = _ref()
    src = elements(100 + n, n)
    out = np.zeros(2 * lib.ref_encode_len(n), np.uint64)
    lib.ref_encode(V(src.ctypes.data), n, V(out.ctypes.data))
    return out


def _fft(args):
    m, o = args
    src = elements(200 + m + o, m)
    out = np.zeros(2 * o, np.uint64)
    _ref().ref_fft(V(src.ctypes.data), m, o, V(out.ctypes.data))
    return out


def _ifft(args):
    m, o = args
    src = elements(300 + m + o, o)
    out = np.zeros(2 * m, np.uint64)
    _ref().ref_ifft(V(src.ctypes.data), m, o, V(out.ctypes.data))
    return out


def _combine(args):
    n, seed = args
    lib = _ref()
    src = elements(seed, n)
    r0, r1 = elements(seed + 1000, 128), elements(seed + 2000, n // 128)
    comb = np.zeros(2 * lib.ref_encode_len(n // 128), np.uint64)
    root = ctypes.create_string_buffer(32)
    ans = np.zeros(2, np.uint64)
    lib.ref_combine(V(src.ctypes.data), n, V(r0.ctypes.data), V(r1.ctypes.data), V(comb.ctypes.data),
                    root, V(ans.ctypes.data))
    return digest(comb), root.raw, ans


def _virgo(args):
    phase, n, bit, seed = args
    vma, addv, ams, r = virgo_inputs(n, seed)
    outs = [np.zeros(2 * n, np.uint64) for _ in range(3)]
    ret = np.zeros(6, np.uint64)
    _ref().ref_virgo_update(phase, V(vma.ctypes.data), V(addv.ctypes.data), V(ams.ctypes.data), n,
                            V(r.ctypes.data), bit, *[V(o.ctypes.data) for o in outs], V(ret.ctypes.data))
    return [digest(o) for o in outs], ret


def _fri(args):
    lm, seed = args
    w, r = elements(seed, (1 << lm) * 64), elements(seed + 1, 1)
    nxt = np.zeros((1 << lm) * 64, np.uint64)
    root = ctypes.create_string_buffer(32)
    _ref().ref_fri_step(V(w.ctypes.data), lm, V(r.ctypes.data), V(nxt.ctypes.data), root)
    return digest(nxt), root.raw


def _rs(lg):
    src = elements(400 + lg, 1 << lg)
    root = ctypes.create_string_buffer(32)
    cw = np.zeros(2 << (lg + 5), np.uint64)
    _ref().ref_rs_commit(V(src.ctypes.data), lg, root, V(cw.ctypes.data))
    return root.raw, digest(cw)


def _zk(case):
    _, copies, cs, ci, cv, padded, pseed, mseed = case
    lib = ctypes.CDLL(ORION_ZK_REF_LIB)
    lib.ref_zk_commit.argtypes = [V, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_ulonglong,
                                  V, V, V, V, V]
    coefs = frame_elements(frame_bytes(pseed, copies * cs), copies, cs, 512, ci, cv, padded)
    ra, rb = ctypes.create_string_buffer(32), ctypes.create_string_buffer(32)
    ha, hb = ctypes.create_string_buffer(80), ctypes.create_string_buffer(80)
    mask = np.zeros(2 * padded * 512, np.uint64)
    lib.ref_zk_commit(V(coefs.ctypes.data), copies, cs, ci, cv, mseed, ra, rb, ha, hb, V(mask.ctypes.data))
    return ra.raw, rb.raw, ha.value, digest(mask)


# (phase, seed, length_g, length_u)
VINIT_CASES = [(1, 1, 1, 1), (2, 1, 1, 1), (1, 2, 4, 4), (2, 3, 4, 4), (1, 4, 8, 6), (2, 5, 8, 6), (1, 6, 6, 10),
               (2, 7, 6, 10), (1, 8, 12, 12), (2, 9, 12, 12), (1, 10, 16, 14), (2, 11, 16, 14)]


def _vinit(case):
    phase, seed, lg, lu = case
    L = virgo_layer(seed, lg, lu)
    lib = ctypes.CDLL(ORION_REF_LIB)
    lib.ref_virgo_init.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int] + [V] * 17
    outs = [np.zeros(4 << lu, np.uint64) for _ in range(3)]
    vp = lambda a: V(a.ctypes.data)
    lib.ref_virgo_init(phase, lg, lu, vp(L["ty"]), vp(L["u"]), vp(L["v"]), vp(L["comb_ptr"]), vp(L["comb_src"]),
                       vp(L["comb_w"]), vp(L["values"]), vp(L["r0"]), vp(L["r1"]), vp(L["alpha"]), vp(L["beta"]),
                       vp(L["vma0"]), vp(L["prev_r"]), vp(L["r_u"]), *[vp(o) for o in outs])
    return b"".join(digest(o) for o in outs)


def main_vinit():
    ctx = mp.get_context("spawn")
    out = {}
    with ctx.Pool(8, maxtasksperchild=1) as pool:
        for case, d in zip(VINIT_CASES, pool.map(_vinit, VINIT_CASES, chunksize=1)):
            key = "%d_%d" % (case[0], case[1])
            out["vinitcase_" + key] = np.array(case, np.int64)
            out["vinit_" + key] = np.frombuffer(d, np.uint8)
    np.savez_compressed(os.path.join(HERE, "virgo_init_golden.npz"), **out)
    print("wrote", len(out), "arrays")


def main_zk():
    ctx = mp.get_context("spawn")
    out = {}
    with ctx.Pool(8, maxtasksperchild=1) as pool:
        for case, (ra, rb, hx, md) in zip(ZK_CASES, pool.map(_zk, ZK_CASES, chunksize=1)):
            name = case[0]
            out["zkcase_" + name] = np.array(case[1:7], np.int64)
            out["zkseed_" + name] = np.array([case[7]], np.uint64)
            out["zkmasked_" + name] = np.frombuffer(ra, np.uint8)
            out["zkmask_" + name] = np.frombuffer(rb, np.uint8)
            out["zkmaskedhex_" + name] = np.frombuffer(hx, np.uint8)
            out["zkmaskdigest_" + name] = np.frombuffer(md, np.uint8)
    np.savez_compressed(os.path.join(HERE, "orion_zk_golden.npz"), **out)
    print("wrote", len(out), "arrays")


def main():
    ctx = mp.get_context("spawn")
    out = {}
    with ctx.Pool(8, maxtasksperchild=1) as pool:
        for (name, n, seed, kind), (root, hx) in zip(
                COMMIT_CASES, pool.map(_commit, [c[1:] for c in COMMIT_CASES], chunksize=1)):
            out["commit_" + name] = np.frombuffer(root, np.uint8)
            out["commithex_" + name] = np.frombuffer(hx, np.uint8)
            out["commitcase_" + name] = np.array([n, seed, ["random", "zero", "max", "small"].index(kind)])
        out["frameroot_1080"] = np.frombuffer(pool.apply(_commit_frame, (0,)), np.uint8)
        out["frame1080"] = np.array([FRAME[k] for k in ("copies", "cs", "W", "const_idx", "const_val",
                                                         "padded", "seed")])
        for n, cw in zip(ENCODE_CASES, pool.map(_encode, ENCODE_CASES, chunksize=1)):
            out["encode_%d" % n] = np.frombuffer(digest(cw), np.uint8)
            out["encodelen_%d" % n] = np.array([cw.size // 2])
            if n == 64:
                out["encodefull_64"] = cw
        for (m, o), r in zip(FFT_CASES, pool.map(_fft, FFT_CASES, chunksize=1)):
            out["fft_%d_%d" % (m, o)] = np.frombuffer(digest(r), np.uint8)
            out["ffthead_%d_%d" % (m, o)] = r[:16].copy()
        for (m, o), r in zip(FFT_CASES, pool.map(_ifft, FFT_CASES, chunksize=1)):
            out["ifft_%d_%d" % (m, o)] = np.frombuffer(digest(r), np.uint8)
        for lg, (root, d) in zip(RS_CASES, pool.map(_rs, RS_CASES, chunksize=1)):
            out["rs_%d" % lg] = np.frombuffer(root, np.uint8)
            out["rscw_%d" % lg] = np.frombuffer(d, np.uint8)
        for (n, seed), (d, root, ans) in zip(COMBINE_CASES, pool.map(_combine, COMBINE_CASES, chunksize=1)):
            out["combine_%d" % n] = np.frombuffer(d, np.uint8)
            out["combineroot_%d" % n] = np.frombuffer(root, np.uint8)
            out["combineanswer_%d" % n] = ans
            out["combinecase_%d" % n] = np.array([n, seed])
        for (phase, n, bit, seed), (ds, ret) in zip(VIRGO_CASES, pool.map(_virgo, VIRGO_CASES, chunksize=1)):
            key = "%d_%d_%d" % (phase, n, bit)
            out["virgocase_" + key] = np.array([phase, n, bit, seed])
            out["virgotables_" + key] = np.frombuffer(b"".join(ds), np.uint8)
            out["virgoret_" + key] = ret
        for (lm, seed), (d, root) in zip(FRI_CASES, pool.map(_fri, FRI_CASES, chunksize=1)):
            out["fricase_%d" % lm] = np.array([lm, seed])
            out["frinext_%d" % lm] = np.frombuffer(d, np.uint8)
            out["friroot_%d" % lm] = np.frombuffer(root, np.uint8)
    np.savez_compressed(os.path.join(HERE, "orion_golden.npz"), **out)
    print("wrote", len(out), "arrays")


if __name__ == "__main__":
    only = sys.argv[1:]
    if not only:
        main()
    if not only or only == ["zk"]:
        main_zk()
    if not only or only == ["vinit"]:
        main_vinit()
