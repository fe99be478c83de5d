"""Scan uploads: ``ptx_stage_host_bytes`` (host bytes copied into the library's page-locked
ring, then read over the bus by a kernel) and ``_utils.upload_small``, through which the
operators move host scans.

Bit-exact: the staged bytes equal the host bytes for word-aligned and misaligned buffers
with ragged tails, for pageable and page-locked sources, across ring wrap-round and for the
large-input copy path.  An operator given a host scan matches the same scan already on the
device to 1e-6 (the gradient atomics may add in another order)."""

import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _lib():
    from ptychox_b200 import _abi

    _abi.load()
    assert torch.cuda.is_available()


def _stage(dst, src_ptr, nbytes):
    from ptychox_b200 import _abi
    from ptychox_b200._utils import stream_handle

    _abi.call("ptx_stage_host_bytes", dst.data_ptr(), src_ptr, nbytes, stream_handle(dst.device))


@pytest.mark.parametrize("nbytes,offset", [(8, 0), (14400, 0), (13, 0), (4099, 3), (1, 7), (200003, 0)])
def test_stage_pinned_bytes(nbytes, offset):
    rng = np.random.default_rng(nbytes + offset)
    host = torch.from_numpy(rng.integers(0, 256, nbytes + offset, dtype=np.uint8)).pin_memory()
    dst = torch.zeros(nbytes + 8, dtype=torch.uint8, device="cuda")
    _stage(dst[offset:], host.data_ptr() + offset, nbytes)
    torch.cuda.synchronize()
    got = dst.cpu().numpy()
    assert np.array_equal(got[offset:offset + nbytes], host.numpy()[offset:])
    assert not got[:offset].any() and not got[offset + nbytes:].any()


def test_stage_pageable_and_reuse_after_return():
    """Pageable memory is staged too, and the source may be overwritten as soon as the call
    returns (the bytes were copied into the library's ring at the call)."""
    buf = (ctypes.c_uint8 * 1000)(*range(256), *range(256), *range(256), *range(232))
    want = np.frombuffer(bytes(buf), dtype=np.uint8).copy()
    dst = torch.zeros(1000, dtype=torch.uint8, device="cuda")
    torch.cuda._sleep(20_000_000)  # keep the stream busy so the staging kernel runs after the overwrite
    _stage(dst, ctypes.addressof(buf), 1000)
    ctypes.memset(buf, 0xAB, 1000)
    torch.cuda.synchronize()
    assert np.array_equal(dst.cpu().numpy(), want)


def test_stage_many_spans_and_large_copy():
    """More staged bytes than the 1 MiB ring holds (spans wrap round and wait for their
    events), and a 1 MiB input above the ring's 256 KiB limit (cudaMemcpyAsync)."""
    rng = np.random.default_rng(5)
    outs, wants = [], []
    for i in range(40):
        n = int(rng.integers(1, 120_000))
        host = torch.from_numpy(rng.integers(0, 256, n, dtype=np.uint8))
        dst = torch.empty(n, dtype=torch.uint8, device="cuda")
        _stage(dst, host.data_ptr(), n)
        outs.append(dst)
        wants.append(host.numpy().copy())
    big = torch.from_numpy(rng.integers(0, 256, 1 << 20, dtype=np.uint8)).pin_memory()
    big_d = torch.empty(1 << 20, dtype=torch.uint8, device="cuda")
    _stage(big_d, big.data_ptr(), 1 << 20)
    torch.cuda.synchronize()
    for d, w in zip(outs, wants):
        assert np.array_equal(d.cpu().numpy(), w)
    assert torch.equal(big_d.cpu(), big)


def test_upload_small_paths():
    from ptychox_b200._utils import upload_small

    dev = torch.device("cuda")
    pos = torch.arange(1800, dtype=torch.int64).reshape(900, 2)
    for src in (pos.pin_memory(), pos, pos.to(torch.int32).pin_memory(), pos.t().contiguous().t(), pos.cuda()):
        out = upload_small(src, dev, torch.long)
        assert out.is_cuda and out.dtype == torch.long and out.is_contiguous()
        assert torch.equal(out.cpu(), pos)
    empty = upload_small(torch.empty(0, 2, dtype=torch.long).pin_memory(), dev, torch.long)
    assert empty.shape == (0, 2) and empty.is_cuda
    shifts = torch.randn(64, 2, dtype=torch.float64)
    out = upload_small(shifts, dev, torch.float32)
    assert torch.equal(out.cpu(), shifts.to(torch.float32))
    # the host tensor may be rewritten right after the call
    host = pos.clone()
    torch.cuda._sleep(20_000_000)
    first = upload_small(host, dev, torch.long)
    host.add_(1)
    second = upload_small(host, dev, torch.long)
    torch.cuda.synchronize()
    assert torch.equal(first.cpu(), pos) and torch.equal(second.cpu(), pos + 1)


def test_capture_rereads_host_buffer_on_replay():
    """Inside CUDA graph capture the staging is a copy node of the caller's page-locked
    buffer, so every replay reads its current contents."""
    from ptychox_b200._utils import upload_small

    host = torch.arange(64, dtype=torch.int64).pin_memory()
    dst = torch.zeros(64, dtype=torch.int64, device="cuda")
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    g = torch.cuda.CUDAGraph()
    with torch.cuda.stream(s):
        upload_small(host, dst.device, torch.long)  # warm-up outside the capture
        with torch.cuda.graph(g, stream=s):
            dst.copy_(upload_small(host, dst.device, torch.long))
    torch.cuda.synchronize()
    for k in (1, 5):
        host.copy_(torch.arange(64, dtype=torch.int64) * k)
        g.replay()
        torch.cuda.synchronize()
        assert torch.equal(dst.cpu(), torch.arange(64) * k)


def test_pinned_scan_matches_device_scan():
    from ptychox_b200 import ptychoX_base_loss, synth
    from oracle import ptycho_oracle as O

    rng = np.random.default_rng(11)
    obj = synth.random_object(256, 256, rng)
    probe = synth.gaussian_probe(64, 64, rng)
    pos = synth.raster_positions(5, 40, 4, 2, rng).astype(np.int64)
    amp, _, _ = O.base_forward(obj, probe, pos)
    meas, scale = synth.poisson_counts(amp**2, 1e4, rng)
    meas_d = torch.from_numpy(meas).cuda()
    res = []
    for scan in (torch.from_numpy(pos).pin_memory(), torch.from_numpy(pos).cuda()):
        s = torch.from_numpy(obj).cuda().requires_grad_(True)
        p = torch.from_numpy(probe).cuda().requires_grad_(True)
        loss = ptychoX_base_loss(s, p, scan, meas_d, scale)
        loss.backward()
        res.append((float(loss.detach()), s.grad.cpu(), p.grad.cpu()))
    # same inputs, same kernels; only the order of the gradient atomics differs between runs
    assert abs(res[0][0] - res[1][0]) <= 1e-12 * abs(res[1][0])
    for a, b in ((res[0][1], res[1][1]), (res[0][2], res[1][2])):
        assert float((a - b).norm() / b.norm()) < 1e-6
