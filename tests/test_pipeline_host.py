"""Host pieces of the pipelined prover (truepix_b200.pipeline) on the CPU: the
host eq table (tp_eq_table_host) against the oracle's compute_beta, the Merkle
node list of an opening (tp_orion_path_nodes) against the restatement of the
reference's collect_merkle_siblings, the VOLE correlation count of a frame's
proof against the reference chain's fixture, and the run loop's ordering (IO
hashed ahead, slots reused, batches handed out in order) with its stages stubbed."""
import ctypes

import numpy as np

from fp2lib import ORACLE_LIB, Fp2Lib, rand_fp


def _lib():
    from truepix_b200 import native
    return native.gkr(require_device=False)


def test_eq_table_matches_oracle_compute_beta():
    lib, orc = _lib(), Fp2Lib(ORACLE_LIB, "oracle_fp2_")
    rng = np.random.default_rng(3)
    for k in (0, 1, 2, 7, 12, 16):
        zr, zi = rand_fp(rng, k), rand_fp(rng, k)
        z = np.ascontiguousarray(np.stack([zr, zi], axis=1).reshape(-1))
        out = np.empty(2 << k, np.uint64)
        assert lib.tp_eq_table_host(z.ctypes.data, k, out.ctypes.data) == 0
        if k == 0:
            assert out.tolist() == [1, 0]
            continue
        wr, wi = orc.compute_beta(zr, zi, (1, 0))
        np.testing.assert_array_equal(out.reshape(-1, 2)[:, 0], wr)
        np.testing.assert_array_equal(out.reshape(-1, 2)[:, 1], wi)
    bad = np.array([(1 << 61) - 1, 0], np.uint64)
    assert lib.tp_eq_table_host(bad.ctypes.data, 1, np.empty(4, np.uint64).ctypes.data) == -1


def test_path_nodes_match_collect_merkle_siblings():
    from truepix_b200.opening import merkle_siblings
    lib = _lib()
    rng = np.random.default_rng(4)
    for leaves, count in ((2, 1), (16, 5), (1 << 12, 300), (1 << 17, 1222)):
        pos = rng.integers(0, leaves, size=count, dtype=np.int64)
        tree = np.zeros((2 * leaves, 32), np.uint8)
        want, _ = merkle_siblings(tree, leaves, pos)
        cap = count * int(np.log2(leaves))
        out = np.empty(cap, np.int32)
        n = lib.tp_orion_path_nodes(leaves, pos.ctypes.data, count, out.ctypes.data, cap)
        assert out[:n].tolist() == want
    pos = np.array([0, 5], np.int64)
    out = np.empty(2, np.int32)
    assert lib.tp_orion_path_nodes(8, pos.ctypes.data, 2, out.ctypes.data, 2) == -1     # over the cap
    assert lib.tp_orion_path_nodes(8, np.array([8], np.int64).ctypes.data, 1, out.ctypes.data, 8) == -1


def test_correlation_count_matches_reference_chain():
    """early rounds 4 each, late rounds 3 each, closing n + 2: what the reference
    prover's whole-layer chain consumed (tests/golden/layer_vole_golden.npz)"""
    from layervole import cases
    from truepix_b200.frame import FrameLayout
    from truepix_b200.pipeline import correlations_needed
    n = 0
    for c in cases():
        layout = FrameLayout(copies=1 << c["nb"], n_wires=1 << c["n_in_bits"], copy_size=1, const_idx=-1)
        assert layout.n_copy_bits == c["nb"] and layout.n_in_bits == c["n_in_bits"]
        assert correlations_needed(layout) == int(c["used_closed"][0]) - int(c["start"][0])
        n += 1
    assert n == 2


def test_run_order_lookahead_and_slot_reuse():
    """ProofPipeline._run with its stages stubbed (no device): every batch is
    hashed ahead (the first in pairs, the rest in io_group), started on the slots
    in turn, finished once, and handed out in input order; a slot is started again
    only after the batch that last held it was finished (its proofs' futures exist:
    the real _start waits on them)"""
    import concurrent.futures
    from truepix_b200.pipeline import ProofPipeline
    for n_slots, ahead, n_batches in ((3, 3, 7), (2, 1, 5), (3, 0, 1), (4, 2, 0)):
        pipe = object.__new__(ProofPipeline)
        pipe.io_ahead, pipe.io_group = ahead, 16
        pipe.slots = [dict(name=i, holds=None) for i in range(n_slots)]
        log, out = [], []

        def prehash(batch, group):
            log.append(("hash", batch, group))
            return batch

        def start(slot, batch):
            assert slot["holds"] is None or ("finish", slot["holds"]) in log, (slot, log)
            slot["holds"] = batch
            log.append(("start", batch))

        def finish(slot):
            log.append(("finish", slot["holds"]))
            fut = concurrent.futures.Future()
            fut.set_result(slot["holds"])
            return [fut]

        pipe._prehash, pipe._start, pipe._finish = prehash, start, finish
        for got in pipe._run(iter(range(n_batches))):
            out.extend(got)
        assert out == list(range(n_batches))
        hashes = [e for e in log if e[0] == "hash"]
        assert [e[1] for e in hashes] == list(range(n_batches))
        assert [e[2] for e in hashes] == [2] + [16] * (n_batches - 1) if n_batches else hashes == []
        starts = [e[1] for e in log if e[0] == "start"]
        assert starts == list(range(n_batches))
        assert sorted(e[1] for e in log if e[0] == "finish") == list(range(n_batches))
        for b in range(n_batches):     # hashing runs ahead of the commits by io_ahead + 1 batches at most
            assert log.index(("hash", b, 2 if b == 0 else 16)) < log.index(("start", b))
            if b > ahead + 1:
                assert log.index(("start", b - ahead - 2)) < log.index(("hash", b, 16))
