"""The benchmark's L2 policy: a step whose footprint is within 16 L2 sizes
gets a buffer of twice the L2 written before every timed step (so nothing
a step reads is still in L2 from the step before); larger steps are timed
back to back. Host logic only, on CPU tensors."""
import torch

import bench


def test_small_step_is_flushed():
    g = bench.L2Guard(136e6, torch.device("cpu"))
    assert g.active
    assert g.buf.numel() == 2 * bench.L2_BYTES
    assert "flushed" in g.text() and "136 MB" in g.text()
    g.flush(None)
    g.flush(None)
    assert g.n == 2 and int(g.buf[0]) == 2


def test_large_step_runs_back_to_back():
    g = bench.L2Guard(20.88e9, torch.device("cpu"))
    assert not g.active
    assert "larger than L2" in g.text() and "20.88 GB" in g.text()
    g.flush(None)  # no buffer, nothing written
    assert g.n == 0


def test_threshold():
    assert bench.L2Guard(16 * bench.L2_BYTES - 1, torch.device("cpu")).active
    assert not bench.L2Guard(16 * bench.L2_BYTES, torch.device("cpu")).active
