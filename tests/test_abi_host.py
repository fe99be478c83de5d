"""CPU-only checks of the C ABI library and the host-side logic (no GPU calls)."""

import re
from pathlib import Path

import numpy as np
import pytest
import torch

from conftest import ROOT

HEADER = ROOT / "include" / "ptychox.h"


def declared_functions() -> list[str]:
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(ptx_[a-z0-9_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    from ptychox_b200 import _abi
    from ptychox_b200.build import build_library

    build_library()
    return _abi.load()


def test_library_exports_every_declared_symbol(lib):
    names = declared_functions()
    assert len(names) >= 10
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_python_signatures_cover_header():
    from ptychox_b200 import _abi

    assert sorted(_abi.SIGNATURES) == declared_functions()


def test_pure_host_entry_points(lib):
    assert lib.ptx_version() >= 100
    for n in (2, 3, 4, 5, 16, 96, 128, 160, 384, 512, 640, 768, 1000, 1024):
        assert lib.ptx_fft_supported(n) == 1, n
    for n in (0, 1, 7, 14, 2048, 1025):
        assert lib.ptx_fft_supported(n) == 0, n
    # which FFT engine serves each length: every smooth length 6..1000 that is not a power of
    # two has compiled mixed-radix kernels; only 2, 3, 4, 5 and 8 are left to the runtime plan
    smooth = [n for n in range(2, 1025) if lib.ptx_fft_supported(n)]
    engines = {n: lib.ptx_fft_engine(n) for n in smooth}
    assert [n for n, e in engines.items() if e == 1] == [16, 32, 64, 128, 256, 512, 1024]
    assert [n for n, e in engines.items() if e == 3] == [2, 3, 4, 5, 8]
    assert all(e == 2 for n, e in engines.items() if n >= 6 and n & (n - 1))
    assert lib.ptx_fft_engine(7) == 0 and lib.ptx_fft_engine(2048) == 0
    hdr = 256 + 65536 * 4  # error word + count-decode table
    ws = lib.ptx_base_workspace_bytes(512, 512, 900)
    frame = 512 * 512 * 8
    assert ws >= hdr + frame and (ws - hdr) % frame == 0
    assert lib.ptx_base_workspace_bytes(128, 128, 3) == hdr + 3 * 128 * 128 * 8
    assert lib.ptx_base_workspace_bytes(0, 16, 1) == 0
    # persistent-pass granularity knob: a host-side setting, negative values rejected
    assert lib.ptx_set_units_per_cta(4) == 0
    assert lib.ptx_set_units_per_cta(-1) != 0
    assert lib.ptx_set_units_per_cta(0) == 0


def test_thread_units_bound_stays_in_its_thread(lib):
    """A server thread's capture-time bound (ptx_set_thread_units_per_cta) never leaks into
    other threads or the process-wide setting, however the threads interleave."""
    import threading

    barrier = threading.Barrier(2)
    seen = {}

    def server(name, k):
        lib.ptx_set_thread_units_per_cta(k)
        barrier.wait()
        seen[name] = lib.ptx_get_units_per_cta()
        barrier.wait()
        lib.ptx_set_thread_units_per_cta(-1)
        seen[name + "_after"] = lib.ptx_get_units_per_cta()

    threads = [threading.Thread(target=server, args=(n, k)) for n, k in (("a", 8), ("b", 3))]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert seen == {"a": 8, "b": 3, "a_after": 0, "b_after": 0}
    assert lib.ptx_get_units_per_cta() == 0
    assert lib.ptx_set_units_per_cta(5) == 0
    lib.ptx_set_thread_units_per_cta(2)
    assert lib.ptx_get_units_per_cta() == 2
    lib.ptx_set_thread_units_per_cta(-1)
    assert lib.ptx_get_units_per_cta() == 5
    assert lib.ptx_set_units_per_cta(0) == 0


def test_new_entry_points_refuse_bad_arguments_on_the_host(lib):
    """Checks that run before any CUDA call: the small-frame sweep's size rule, the server's
    device and argument checks, the registration workspace query."""
    import ctypes as C

    from ptychox_b200 import _abi

    # ptx_base_sweep_small takes square 32 / 64 / 128 probes only
    assert lib.ptx_base_sweep_small(None, 256, 256, None, 64, 32, None, 1, None, 1.0, None, None, None, None, 0,
                                    None) == _abi.PTX_ERR_UNSUPPORTED_SIZE
    assert "square 32, 64 or 128" in _abi.last_error()
    # the server needs a CUDA device and positive slot counts
    h = C.c_void_p()
    assert lib.ptx_server_create(0, 0, 0, C.addressof(h)) == _abi.PTX_ERR_INVALID_ARGUMENT
    assert lib.ptx_server_create(-1, 0, 8, C.addressof(h)) == _abi.PTX_ERR_INVALID_ARGUMENT
    if not torch.cuda.is_available():
        assert lib.ptx_server_create(0, 0, 8, C.addressof(h)) == _abi.PTX_ERR_INVALID_ARGUMENT
    assert not h.value
    assert lib.ptx_server_create(0, 0, 8, None) == _abi.PTX_ERR_INVALID_ARGUMENT
    assert lib.ptx_server_destroy(None) == _abi.PTX_OK
    # registration workspace: none up to usfac 2, else FP64 patches of ceil(1.5 usfac)^2 and
    # n_out x rows per image
    assert lib.ptx_reg_workspace_bytes(3, 64, 64, 2) == 0
    assert lib.ptx_reg_workspace_bytes(2, 64, 80, 600) == 16 * 2 * 900 * (64 + 900)
    assert lib.ptx_stage_host_bytes(None, None, 0, None) == _abi.PTX_OK  # nothing to copy


def test_reference_input_checks_and_messages():
    from ptychox_b200._utils import check_complex_scan_inputs

    s = torch.zeros(8, 8, dtype=torch.complex64)
    p = torch.zeros(4, 4, dtype=torch.complex64)
    pos = torch.zeros(2, 2, dtype=torch.long)
    check_complex_scan_inputs(s, p, pos)
    with pytest.raises(ValueError, match="must be 2D complex tensors"):
        check_complex_scan_inputs(s[None], p, pos)
    with pytest.raises(TypeError, match="must be complex tensors"):
        check_complex_scan_inputs(s.real, p, pos)
    with pytest.raises(ValueError, match="same dtype"):
        check_complex_scan_inputs(s, p.to(torch.complex128), pos)
    with pytest.raises(ValueError, match=r"shape \[batch, 2\]"):
        check_complex_scan_inputs(s, p, torch.zeros(2, 3, dtype=torch.long))


def test_cpu_tensors_are_rejected_no_fallback():
    from ptychox_b200 import ptychoX_base

    s = torch.zeros(8, 8, dtype=torch.complex64)
    p = torch.zeros(4, 4, dtype=torch.complex64)
    with pytest.raises(ValueError, match="CUDA"):
        ptychoX_base(s, p, torch.zeros(1, 2, dtype=torch.long), use_cuda_kernels=True)


def test_positions_bounds_and_counts():
    from ptychox_b200._utils import as_u16, device_positions, matlab_positions_to_torch

    pos = torch.tensor([[0, 0], [4, 4]])
    out = device_positions(pos, torch.device("cpu"), (4, 4), (8, 8))
    assert out.dtype == torch.long
    with pytest.raises(ValueError, match="leaves"):
        device_positions(torch.tensor([[5, 0]]), torch.device("cpu"), (4, 4), (8, 8))
    with pytest.raises(ValueError, match="leaves"):
        device_positions(torch.tensor([[-1, 0]]), torch.device("cpu"), (4, 4), (8, 8))
    assert torch.equal(matlab_positions_to_torch(torch.tensor([[1, 2]])), torch.tensor([[0, 1]]))
    u = as_u16(torch.tensor([0, 65535], dtype=torch.int32), torch.device("cpu"))
    assert u.dtype == torch.uint16
    with pytest.raises(ValueError):
        as_u16(torch.tensor([70000]), torch.device("cpu"))
    with pytest.raises(TypeError):
        as_u16(torch.tensor([1.0]), torch.device("cpu"))


def test_synthetic_configs():
    from ptychox_b200 import synth

    rng = np.random.default_rng(0)
    o = synth.random_object(64, 64, rng)
    a = np.abs(o)
    assert o.dtype == np.complex64 and a.min() >= 0.8 - 1e-6 and a.max() <= 1.0 + 1e-6
    pos = synth.raster_positions(30, 48, 64, 3, rng)
    assert pos.shape == (900, 2) and pos.min() >= 61 and pos.max() + 512 <= 2048
    pos0 = synth.raster_positions(11, 32, 8, 2, rng)
    assert pos0.shape == (121, 2) and pos0.min() >= 6 and pos0.max() + 128 <= 512
    with pytest.raises(ValueError, match="saturate"):
        synth.poisson_counts(np.full((1, 2, 2), 1.0), 1e6, rng)
    counts, scale = synth.poisson_counts(np.full((3, 4, 4), 2.0), 160.0, rng)
    assert counts.dtype == np.uint16 and abs(scale - 32.0 / 160.0) < 1e-6
    dx = synth.fpm_dx_for_pupil(1024, 256, 0.1, 0.532, 0.3)
    assert abs(dx - 0.399) < 1e-3
    led = synth.fpm_led_windows(1024, 256, 15, 4.0, 90.0, 0.532, dx)
    assert led.shape == (225, 2) and led.min() >= 0 and led.max() <= 768
    t = synth.angular_spectrum_transfer(64, 1.85e-6, 0.5e-6, 2e-3)
    assert np.allclose(np.abs(t), 1.0, atol=1e-6)  # all propagating at 1.85 um pixels
    sh = synth.coded_shifts(64, 20.0, 1024, rng)
    assert sh.dtype == np.float32 and np.abs(sh).max() <= 20.0 / 1024
