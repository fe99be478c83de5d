"""Conventional ptychography: CUDA library (through the C ABI) vs the oracle and golden vectors.

Tolerance: relative L2 error ``||x - x_ref|| / ||x_ref||`` below 1e-5 for loss and
gradients against the FP64 oracle / FP64 reference fixtures, the bar of the FP32 path.
"""

import numpy as np
import pytest
import torch

from conftest import load_golden, rel_l2
from oracle import ptycho_oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-5


def cuda(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.fixture(scope="module", autouse=True)
def _lib():
    import ptychox_b200  # noqa: F401
    from ptychox_b200 import _abi

    _abi.load()
    assert torch.cuda.is_available()


def run_sweep(sample, probe, pos, meas, scale):
    from ptychox_b200.base import base_sweep

    loss, gs, gp = base_sweep(cuda(sample), cuda(probe), cuda(pos.astype(np.int64)), cuda(meas), scale)
    torch.cuda.synchronize()
    return float(loss.item()), gs.cpu().numpy(), gp.cpu().numpy()


def test_test_ops_case_forward_backward():
    """python/test_ops.py:30-49 case (4x5 probe: runtime-plan kernels)."""
    from ptychox_b200 import ptychoX_base

    g = load_golden("test_ops_base.npz")
    s = cuda(g["sample"]).requires_grad_(True)
    p = cuda(g["probe"]).requires_grad_(True)
    out = ptychoX_base(s, p, cuda(g["positions"]), use_cuda_kernels=True)
    (out * cuda(g["grad"])).sum().backward()
    assert rel_l2(out.detach().cpu().numpy(), g["out"]) < TOL
    assert rel_l2(s.grad.cpu().numpy(), g["grad_sample"]) < TOL
    assert rel_l2(p.grad.cpu().numpy(), g["grad_probe"]) < TOL


@pytest.mark.parametrize("name", ["sweep_base_fp64.npz", "sweep_base_odd_fp64.npz"])
def test_sweep_golden(name):
    g = load_golden(name)
    loss, gs, gp = run_sweep(g["sample"], g["probe"], g["positions"], g["measured"], float(g["scale"]))
    assert abs(loss - float(g["loss"])) <= TOL * abs(float(g["loss"]))
    assert rel_l2(gs, g["grad_sample"]) < TOL
    assert rel_l2(gp, g["grad_probe"]) < TOL


def small_problem(n_obj, p, grid, step, origin, jitter, photons, seed):
    from ptychox_b200 import synth

    rng = np.random.default_rng(seed)
    obj = synth.random_object(n_obj, n_obj, rng)
    probe = synth.gaussian_probe(p, p, rng)
    pos = synth.raster_positions(grid, step, origin, jitter, rng)
    amp, _, _ = O.base_forward(obj, probe, pos)
    meas, scale = synth.poisson_counts(amp**2, photons, rng)
    guess = (obj * (1 + 0.1 * rng.standard_normal(obj.shape))).astype(np.complex64)
    return guess, probe, pos, meas, scale


@pytest.mark.parametrize("p", [32, 64, 96, 128, 160])
def test_sweep_vs_oracle_sizes(p):
    """Power-of-two (32, 64, 128) and mixed-radix (96 = 8 x 12, 160 = 10 x 16) transform lengths."""
    obj, probe, pos, meas, scale = small_problem(4 * p, p, 4, p // 2, 3, 2, 1e4, seed=p)
    loss, gs, gp = run_sweep(obj, probe, pos, meas, scale)
    rl, rs, rp = O.base_sweep(obj, probe, pos, meas, scale)
    assert abs(loss - rl) <= TOL * abs(rl)
    assert rel_l2(gs, rs) < TOL
    assert rel_l2(gp, rp) < TOL


@pytest.mark.parametrize("ph,pw,n_pos", [(256, 256, 6), (1024, 1024, 3), (64, 128, 9), (128, 64, 9),
                                         (96, 160, 6), (512, 256, 4)])
def test_sweep_vs_oracle_large_and_rectangular(ph, pw, n_pos):
    """The largest compile-time frame (1024 points per line: 32 threads per row line, 256-thread
    column CTAs), 256-point frames, and rectangular probes whose rows and columns take
    different line plans (compile-time and runtime) against the FP64 oracle."""
    from ptychox_b200 import synth

    rng = np.random.default_rng(ph * 7 + pw)
    h, w = ph + 3 * 24 + 8, pw + 3 * 24 + 8
    obj = synth.random_object(h, w, rng)
    probe = synth.gaussian_probe(ph, pw, rng)
    pos = np.stack([rng.integers(0, w - pw + 1, n_pos), rng.integers(0, h - ph + 1, n_pos)], axis=1).astype(np.int64)
    amp, _, _ = O.base_forward(obj, probe, pos)
    meas, scale = synth.poisson_counts(amp**2, 1e4, rng)
    guess = (obj * (1 + 0.1 * rng.standard_normal(obj.shape))).astype(np.complex64)
    loss, gs, gp = run_sweep(guess, probe, pos, meas, scale)
    rl, rs, rp = O.base_sweep(guess, probe, pos, meas, scale)
    assert abs(loss - rl) <= TOL * abs(rl)
    assert rel_l2(gs, rs) < TOL
    assert rel_l2(gp, rp) < TOL


def test_config0_sweep_vs_oracle():
    """Config 0 shape: 512x512 object, 128x128 probe, 11x11 raster step 32 with U[-2,2] jitter."""
    obj, probe, pos, meas, scale = small_problem(512, 128, 11, 32, 8, 2, 1e4, seed=0)
    loss, gs, gp = run_sweep(obj, probe, pos, meas, scale)
    rl, rs, rp = O.base_sweep(obj, probe, pos, meas, scale)
    assert abs(loss - rl) <= TOL * abs(rl)
    assert rel_l2(gs, rs) < TOL
    assert rel_l2(gp, rp) < TOL


def test_operator_matches_oracle_and_fused():
    """autograd.Function forward/backward vs the oracle, and vs the fused sweep."""
    from ptychox_b200 import ptychoX_base, ptychoX_base_loss

    obj, probe, pos, meas, scale = small_problem(256, 64, 5, 40, 4, 2, 1e4, seed=3)
    rng = np.random.default_rng(5)
    gout = rng.standard_normal((len(pos), 64, 64)).astype(np.float32)
    s = cuda(obj).requires_grad_(True)
    p = cuda(probe).requires_grad_(True)
    amp = ptychoX_base(s, p, torch.from_numpy(pos))  # CPU positions are accepted
    (amp * cuda(gout)).sum().backward()
    ramp, far, patches = O.base_forward(obj, probe, pos)
    rgs, rgp = O.base_backward(gout, patches, probe.astype(np.complex128), far, pos, obj.shape)
    assert rel_l2(amp.detach().cpu().numpy(), ramp) < TOL
    assert rel_l2(s.grad.cpu().numpy(), rgs) < TOL
    assert rel_l2(p.grad.cpu().numpy(), rgp) < TOL

    s2 = cuda(obj).requires_grad_(True)
    p2 = cuda(probe).requires_grad_(True)
    amp2 = ptychoX_base(s2, p2, cuda(pos))
    observed = torch.sqrt(cuda(meas).to(torch.float32) * np.float32(scale))
    torch.nn.functional.mse_loss(amp2, observed).backward()
    s3 = cuda(obj).requires_grad_(True)
    p3 = cuda(probe).requires_grad_(True)
    ptychoX_base_loss(s3, p3, cuda(pos), cuda(meas), scale).backward()
    assert rel_l2(s3.grad.cpu().numpy(), s2.grad.cpu().numpy()) < TOL
    assert rel_l2(p3.grad.cpu().numpy(), p2.grad.cpu().numpy()) < TOL


def test_chunked_workspace_matches():
    """A workspace holding one frame (many launches) gives the same result as a full one."""
    from ptychox_b200 import _abi
    from ptychox_b200.base import base_sweep

    obj, probe, pos, meas, scale = small_problem(256, 64, 5, 40, 4, 2, 1e4, seed=4)
    full = base_sweep(cuda(obj), cuda(probe), cuda(pos), cuda(meas), scale)
    frame = 64 * 64 * 8
    hdr = 256 + 65536 * 4
    ws = torch.empty(hdr + frame, dtype=torch.uint8, device="cuda")
    one = base_sweep(cuda(obj), cuda(probe), cuda(pos), cuda(meas), scale, ws=ws)
    assert abs(float(full[0]) - float(one[0])) <= 1e-12 * abs(float(full[0]))
    assert rel_l2(one[1].cpu().numpy(), full[1].cpu().numpy()) < 1e-6
    with pytest.raises(RuntimeError):
        base_sweep(cuda(obj), cuda(probe), cuda(pos), cuda(meas), scale,
                   ws=torch.empty(frame // 2, dtype=torch.uint8, device="cuda"))
    assert _abi.query("ptx_fft_supported", 7) == 0


def test_synthesize_dataset_and_device_counts():
    """``synth.synthesize_dataset`` (the reference's chunked forward) equals one operator call
    over all positions bit for bit; device Poisson counts repeat for a seed and hold the
    requested photons per pattern on average (5 standard deviations)."""
    from ptychox_b200 import ptychoX_base, synth

    rng = np.random.default_rng(21)
    obj = cuda(synth.random_object(256, 256, rng))
    probe = cuda(synth.gaussian_probe(64, 64, rng))
    pos = cuda(synth.raster_positions(5, 40, 4, 2, rng))
    amp = synth.synthesize_dataset(obj, probe, pos, batch_size=7)
    assert torch.equal(amp, ptychoX_base(obj, probe, pos))
    c1, s1 = synth.poisson_counts_device(amp, 1e4, seed=3)
    c2, s2 = synth.poisson_counts_device(amp, 1e4, seed=3)
    assert c1.dtype == torch.uint16 and torch.equal(c1, c2) and s1 == s2
    total = float(c1.to(torch.float64).sum())
    expect = float((amp.double() ** 2).sum()) / s1
    assert abs(total - expect) < 5 * expect**0.5
    assert abs(total / amp.shape[0] - 1e4) < 0.01 * 1e4
    with pytest.raises(ValueError):
        synth.synthesize_dataset(obj, probe, pos, batch_size=0)


def test_errors_are_mapped():
    from ptychox_b200 import ptychoX_base

    s = torch.zeros(64, 64, dtype=torch.complex64, device="cuda")
    p = torch.zeros(14, 14, dtype=torch.complex64, device="cuda")  # 14 = 2*7: unsupported length
    with pytest.raises(ValueError):
        ptychoX_base(s, p, torch.zeros(1, 2, dtype=torch.long))
    p = torch.zeros(16, 16, dtype=torch.complex64, device="cuda")
    with pytest.raises(ValueError):
        ptychoX_base(s, p, torch.tensor([[60, 0]]))  # window leaves the sample
    with pytest.raises(TypeError):
        ptychoX_base(s.to(torch.complex128), p.to(torch.complex128), torch.zeros(1, 2, dtype=torch.long))
    out = ptychoX_base(s, p, torch.zeros(0, 2, dtype=torch.long))
    assert out.shape == (0, 16, 16)


def test_config1_subset_vs_oracle():
    """Config 1 frame size (2048^2 object, 512^2 probe) on a 48-position subset vs FP64 oracle."""
    from ptychox_b200 import synth

    rng = np.random.default_rng(1)
    obj = synth.random_object(2048, 2048, rng)
    probe = synth.gaussian_probe(512, 512, rng)
    pos = synth.raster_positions(30, 48, 64, 3, rng)
    sub = pos[rng.choice(len(pos), 48, replace=False)]
    amp, _, _ = O.base_forward(obj, probe, sub, fp64=False)
    meas, scale = synth.poisson_counts(amp.astype(np.float64) ** 2, 1e5, rng)
    guess = (obj * (1 + 0.1 * rng.standard_normal(obj.shape))).astype(np.complex64)
    loss, gs, gp = run_sweep(guess, probe, sub, meas, scale)
    rl, rs, rp = O.base_sweep(guess, probe, sub, meas, scale)
    assert abs(loss - rl) <= TOL * abs(rl)
    assert rel_l2(gs, rs) < TOL
    assert rel_l2(gp, rp) < TOL


def _fd_base(obj, probe, pos, meas, scale, obj_pix, probe_pix, delta=1e-5):
    """Central differences of the FP64 loss at single object / probe pixels.

    A pixel perturbation changes each affected exit wave at one point, so the far field
    changes by delta * value * (outer product of two DFT rows): the loss differences are
    evaluated exactly from the stored FP64 far fields, stably as
    (|F+D| - |F|)(|F+D| + |F| - 2Y) with |F+D| - |F| = (2 Re(conj(F) D) + |D|^2)/(|F+D| + |F|).
    Returns (dL/dRe, dL/dIm) per pixel.
    """
    p = probe.shape[0]
    obj = obj.astype(np.complex128)
    probe = probe.astype(np.complex128)
    _, far, _ = O.base_forward(obj, probe, pos)
    y = O.measured_amplitude(meas, scale).astype(np.float64)
    a = np.abs(far)
    numel = far.size
    k = np.arange(p) - p // 2

    def dloss(b, ly, lx, d):
        ey = np.exp(-2j * np.pi * k * ly / p)
        ex = np.exp(-2j * np.pi * k * lx / p)
        dF = d * np.outer(ey, ex)
        F = far[b]
        anew = np.abs(F + dF)
        diff = (2 * (np.conj(F) * dF).real + np.abs(dF) ** 2) / (anew + a[b] + 1e-300)
        return float(np.sum(diff * (anew + a[b] - 2 * y[b]))) / numel

    def central(terms):
        out = []
        for e in (1.0, 1j):
            plus = sum(dloss(b, ly, lx, delta * e * v) for b, ly, lx, v in terms)
            minus = sum(dloss(b, ly, lx, -delta * e * v) for b, ly, lx, v in terms)
            out.append((plus - minus) / (2 * delta))
        return out

    fd_obj, fd_probe = [], []
    for (yy, xx) in obj_pix:
        terms = [(b, yy - y0, xx - x0, probe[yy - y0, xx - x0]) for b, (x0, y0) in enumerate(pos.tolist())
                 if x0 <= xx < x0 + p and y0 <= yy < y0 + p]
        fd_obj.append(central(terms))
    for (ly, lx) in probe_pix:
        terms = [(b, ly, lx, obj[y0 + ly, x0 + lx]) for b, (x0, y0) in enumerate(pos.tolist())]
        fd_probe.append(central(terms))
    return np.array(fd_obj), np.array(fd_probe)


def test_config1_finite_differences():
    """Config 1 frames (2048^2 object, 512^2 probe, 48-position subset): the autograd.Function
    gradient of the fused loss vs FP64 central differences at 64 random object pixels and
    16 random probe pixels."""
    from ptychox_b200 import ptychoX_base_loss, synth

    rng = np.random.default_rng(31)
    obj = synth.random_object(2048, 2048, rng)
    probe = synth.gaussian_probe(512, 512, rng)
    pos = synth.raster_positions(30, 48, 64, 3, rng)
    sub = pos[rng.choice(len(pos), 48, replace=False)]
    amp, _, _ = O.base_forward(obj, probe, sub, fp64=False)
    meas, scale = synth.poisson_counts(amp.astype(np.float64) ** 2, 1e5, rng)
    guess = (obj * (1 + 0.1 * rng.standard_normal(obj.shape))).astype(np.complex64)
    s = cuda(guess).requires_grad_(True)
    p = cuda(probe).requires_grad_(True)
    ptychoX_base_loss(s, p, cuda(sub), cuda(meas), scale).backward()
    gs, gp = s.grad.cpu().numpy(), p.grad.cpu().numpy()
    covered = [(int(y0 + rng.integers(0, 512)), int(x0 + rng.integers(0, 512)))
               for x0, y0 in sub[rng.choice(len(sub), 64)].tolist()]
    ppix = [(int(a), int(b)) for a, b in rng.integers(150, 362, size=(16, 2))]  # inside the probe's support
    fd_o, fd_p = _fd_base(guess, probe, sub, meas, scale, covered, ppix)
    g_o = np.array([[gs[y, x].real, gs[y, x].imag] for y, x in covered])
    g_p = np.array([[gp[a, b].real, gp[a, b].imag] for a, b in ppix])
    assert rel_l2(g_o, fd_o) < TOL
    assert rel_l2(g_p, fd_p) < TOL


def test_device_window_check_without_host_copy():
    """Device-resident positions are checked by the kernels: the out-of-object window is
    reported through the workspace status word (ptx_workspace_status), deferred to the next
    call or check_errors() by default, at the call itself in "sync" mode."""
    import ptychox_b200
    from ptychox_b200 import _abi, ptychoX_base, ptychoX_base_loss

    s = torch.ones(64, 64, dtype=torch.complex64, device="cuda")
    p = torch.ones(16, 16, dtype=torch.complex64, device="cuda")
    bad = torch.tensor([[0, 0], [60, 3]], device="cuda")
    good = torch.tensor([[0, 0], [40, 3]], device="cuda")
    assert ptychox_b200.bounds_check_mode() == "deferred"
    out = ptychoX_base(s, p, bad)  # no exception at the call: no host copy, no sync
    assert out.shape == (2, 16, 16)
    with pytest.raises(ValueError, match="window leaves the object"):
        ptychox_b200.check_errors()
    ptychox_b200.check_errors()  # reported once
    ptychoX_base(s, p, good)
    ptychox_b200.check_errors()
    try:
        ptychox_b200.set_bounds_check("sync")
        with pytest.raises(ValueError, match="window leaves the object"):
            ptychoX_base_loss(s, p, bad, torch.zeros(2, 16, 16, dtype=torch.uint16, device="cuda"), 1.0)
        ptychox_b200.set_bounds_check("host")
        with pytest.raises(ValueError, match="window leaves"):
            ptychoX_base(s, p, bad)
    finally:
        ptychox_b200.set_bounds_check("deferred")
    # the C ABI directly: the word after a sweep over the bad scan, and the code it maps to
    from ptychox_b200._utils import workspace

    ws = workspace(_abi.query("ptx_base_workspace_bytes", 16, 16, 2), torch.device("cuda"))
    loss = torch.empty((), dtype=torch.float64, device="cuda")
    gs, gp = torch.empty_like(s), torch.empty_like(p)
    meas = torch.zeros(2, 16, 16, dtype=torch.uint16, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    word = torch.full((1,), 7, dtype=torch.int32, device="cuda")
    for scan, expect in ((bad, 1), (good, 0)):
        _abi.call("ptx_base_sweep", s.data_ptr(), 64, 64, p.data_ptr(), 16, 16, scan.data_ptr(), 2, meas.data_ptr(),
                  1.0, loss.data_ptr(), gs.data_ptr(), gp.data_ptr(), ws.data_ptr(), ws.numel(), stream)
        _abi.call("ptx_workspace_status", ws.data_ptr(), word.data_ptr(), stream)
        assert int(word.item()) == expect
        assert _abi.query("ptx_status_code", int(word.item())) == (_abi.PTX_ERR_OUT_OF_BOUNDS if expect else 0)
