"""truepix_b200.fiatshamir.FiatShamir, the drop-in for the reference prover's
transcript class (libTruePix/fiatshamir.py), against the vectors made by the
reference class itself (tests/golden/fs_golden.npz): the same challenges and
digests for put() of int lists, Fp2 values, strings, None, tuples, dicts and
mixed lists; the proof container round trip with take(); and a transcript
begun in the class, continued on the device by the batched entry points and
brought back, against the same script replayed on the host."""
import ctypes

import numpy as np
import pytest

from fslib import P61, golden, py_value, replay_python, scripts

pytestmark = pytest.mark.gpu


class F2:
    """the reference Fp2's constructor and attributes (extfield.py)"""

    def __init__(self, re, im, q=P61):
        self.real, self.imag, self.q = re, im, q

    def __eq__(self, o):
        return (self.real, self.imag) == (o.real, o.imag)


def replay_class(FS, protocol, ops):
    fs = FS(P61, protocol=protocol, fp2_type=F2)
    outs, digs, puts = [], b"", []
    for op in ops:
        if op[0] in ("u64s", "str", "put_py"):
            v = py_value(op[1], F2) if op[0] == "put_py" else op[1]
            fs.put(v)
            puts.append(v)
        elif op[0] == "fp2s":
            for re, im in op[1]:
                fs.put(F2(re, im))
                puts.append(F2(re, im))
        elif op[0] == "ext":
            e = fs.rand_ext(op[1])
            outs += [e.real, e.imag]
        elif op[0] == "scalar":
            outs.append(fs.rand_scalar())
        elif op[0] == "digest":
            digs += fs.digest()
    return fs, np.array(outs, np.uint64), digs, puts


def test_class_matches_reference_vectors():
    from truepix_b200.fiatshamir import FiatShamir
    g = golden()
    n = 0
    for name, protocol, ops in scripts(g):
        fs, outs, digs, _ = replay_class(FiatShamir, protocol, ops)
        np.testing.assert_array_equal(outs, g["fsout_" + name])
        assert digs == g["fsdigest_" + name].tobytes(), name
        assert fs.rnum == sum(2 if op[0] == "ext" else 1 for op in ops if op[0] in ("ext", "scalar"))
        n += 1
    assert n == 4


def test_proof_container_round_trip_replays_the_transcript():
    """to_string / from_string / take: the verifier side absorbs the same values
    in the same order and draws the same challenges (fiatshamir.py:188-237)"""
    from truepix_b200.fiatshamir import FiatShamir
    g = golden()
    for name, protocol, ops in scripts(g):
        fs, outs, _, puts = replay_class(FiatShamir, protocol, ops)
        s = fs.to_string()
        v = FiatShamir.from_string(s, protocol=protocol)
        v._fp2 = F2
        got = []
        for op in ops:
            if op[0] in ("u64s", "str", "put_py"):
                v.take()
            elif op[0] == "fp2s":
                for _ in op[1]:
                    v.take()
            elif op[0] == "ext":
                e = v.rand_ext(op[1])
                got += [e.real, e.imag]
            elif op[0] == "scalar":
                got.append(v.rand_scalar())
        np.testing.assert_array_equal(np.array(got, np.uint64), outs)
        assert v.digest() == fs.digest()
        nelems, size = FiatShamir.proof_size(s)
        assert nelems >= len(puts) and size > 0
        with pytest.raises(AssertionError):
            v.put([1])
        with pytest.raises(AssertionError):
            fs.take()


def test_class_rejects_other_fields_and_bad_elements():
    from truepix_b200.fiatshamir import FiatShamir
    with pytest.raises(ValueError):
        FiatShamir((1 << 127) - 1)
    fs = FiatShamir(P61)
    with pytest.raises(TypeError):
        fs.put([1.5, 2])
    with pytest.raises(ValueError):
        fs.set_state(b"\x00" * 7)
    # with no Fp2 type importable the draw is a pair
    fs._fp2 = None
    assert isinstance(fs.rand_ext("x"), tuple)


def test_state_continues_on_the_device_and_back():
    """A transcript begun in the class (prefix puts), moved to the device as one
    state of a batch, where each frame puts four Fp2 claims and draws
    rand_ext("sc-0-k") for three rounds, then brought back into the class and
    finished on the host: the challenges and final digest equal the whole
    script replayed by the hashlib restatement."""
    import torch
    from truepix_b200 import native
    from truepix_b200.fiatshamir import FiatShamir
    lib = native.gkr()
    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(7)
    B, R = 5, 3
    claims = rng.integers(0, P61, size=(R, B, 4, 2), dtype=np.uint64)
    prefix = [["put_py", ["private_input_omitted", 384]], ["u64s", [3, 1 << 40]], ["ext", "z2-0"]]
    tail = [["put_py", {"tuple": [None, 9]}], ["ext", "final"], ["digest"]]

    host = []
    for f in range(B):
        fs, _, _, _ = replay_class(FiatShamir, "truepix", prefix + [["u64s", [f]]])
        host.append(fs)
    d_states = torch.from_numpy(np.frombuffer(b"".join(fs.state() for fs in host), np.uint8).copy()).to(dev)
    d_out = torch.zeros((R, B, 2), dtype=torch.int64, device=dev)
    for k in range(R):
        d_cl = torch.from_numpy(claims[k].view(np.int64).copy()).to(dev)
        assert lib.tp_fs_put_fp2s_dev(d_states.data_ptr(), B, d_cl.data_ptr(), 4, None) == 0
        assert lib.tp_fs_rand_ext_dev(d_states.data_ptr(), B, ("sc-0-%d" % k).encode(), d_out[k].data_ptr(),
                                      None) == 0
    torch.cuda.synchronize()
    raw = d_states.cpu().numpy().tobytes()
    dev_ch = d_out.cpu().numpy().view(np.uint64)
    nst = lib.tp_fs_state_bytes()

    for f in range(B):
        fs = host[f]
        fs.set_state(raw[f * nst:(f + 1) * nst])
        fs.put((None, 9))
        e = fs.rand_ext("final")
        script = prefix + [["u64s", [f]]]
        for k in range(R):
            script += [["fp2s", [[int(a), int(b)] for a, b in claims[k, f]]], ["ext", "sc-0-%d" % k]]
        outs, digs = replay_python("truepix", script + tail)
        np.testing.assert_array_equal(dev_ch[:, f].reshape(-1), outs[2:2 + 2 * R])
        assert [e.real, e.imag] == [int(x) for x in outs[-2:]]
        assert fs.digest() == digs
        assert fs.rnum == 2 * (R + 2)
