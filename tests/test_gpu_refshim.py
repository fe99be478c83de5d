"""The reference's own autograd.Function classes running on libptychox.

The unmodified reference package (``baseline/_ref``) gets ``ptychox_b200.refshim`` as its
native extension (``refshim.install``); ``ptychoX_base`` / ``ptychoX_fourier`` /
``ptychoX_coded`` with ``use_cuda_kernels=True`` then run forward and backward through the C
ABI.  Their outputs and gradients must equal ``ptychox_b200``'s own operators and the FP64
oracle (relative L2 1e-5).
"""

import numpy as np
import pytest
import torch

from conftest import rel_l2
from oracle import ptycho_oracle as O
from refpkg import reference_package

pytestmark = pytest.mark.gpu

TOL = 1e-5


def cuda(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.fixture(scope="module")
def ref():
    pkg = reference_package()
    from ptychox_b200 import refshim

    refshim.install(pkg)
    yield pkg
    import ptychoX.base.ops as b
    import ptychoX.coded.ops as c
    import ptychoX.fpm.ops as f

    b._CUDA_EXT = f._CUDA_EXT = c._CUDA_EXT = None


def test_reference_base_function_on_libptychox(ref):
    from ptychox_b200 import ptychoX_base, synth

    rng = np.random.default_rng(41)
    obj = synth.random_object(160, 192, rng)
    probe = synth.gaussian_probe(64, 64, rng)
    pos = np.stack([rng.integers(0, 192 - 64 + 1, 9), rng.integers(0, 160 - 64 + 1, 9)], axis=1).astype(np.int64)
    gout = rng.standard_normal((9, 64, 64)).astype(np.float32)
    s = cuda(obj).requires_grad_(True)
    p = cuda(probe).requires_grad_(True)
    amp = ref.ptychoX_base(s, p, cuda(pos), use_cuda_kernels=True)
    (amp * cuda(gout)).sum().backward()
    s2 = cuda(obj).requires_grad_(True)
    p2 = cuda(probe).requires_grad_(True)
    amp2 = ptychoX_base(s2, p2, cuda(pos))
    (amp2 * cuda(gout)).sum().backward()
    ramp, far, patches = O.base_forward(obj, probe, pos)
    rgs, rgp = O.base_backward(gout, patches, probe.astype(np.complex128), far, pos, obj.shape)
    assert rel_l2(amp.detach().cpu().numpy(), ramp) < TOL
    assert rel_l2(s.grad.cpu().numpy(), rgs) < TOL
    assert rel_l2(p.grad.cpu().numpy(), rgp) < TOL
    assert torch.equal(amp, amp2)
    assert rel_l2(s.grad.cpu().numpy(), s2.grad.cpu().numpy()) < 1e-6
    ref.clear_cuda_plan_cache()


def test_reference_training_step_on_libptychox(ref):
    """The reference driver's step (train_ptychography.py:549-557) on the shim equals our fused loss."""
    from ptychox_b200 import ptychoX_base_loss, synth

    rng = np.random.default_rng(42)
    obj = synth.random_object(256, 256, rng)
    probe = synth.gaussian_probe(128, 128, rng)
    pos = synth.raster_positions(4, 40, 4, 2, rng)
    amp, _, _ = O.base_forward(obj, probe, pos)
    meas, scale = synth.poisson_counts(amp**2, 1e4, rng)
    s = cuda(obj).requires_grad_(True)
    p = cuda(probe).requires_grad_(True)
    observed = torch.sqrt(cuda(meas).to(torch.float32) * np.float32(scale))
    loss = torch.nn.functional.mse_loss(ref.ptychoX_base(s, p, cuda(pos), use_cuda_kernels=True), observed)
    loss.backward()
    s2 = cuda(obj).requires_grad_(True)
    p2 = cuda(probe).requires_grad_(True)
    loss2 = ptychoX_base_loss(s2, p2, cuda(pos), cuda(meas), scale)
    loss2.backward()
    assert abs(float(loss) - float(loss2)) <= TOL * abs(float(loss2))
    assert rel_l2(s.grad.cpu().numpy(), s2.grad.cpu().numpy()) < TOL
    assert rel_l2(p.grad.cpu().numpy(), p2.grad.cpu().numpy()) < TOL


def test_reference_fourier_function_on_libptychox(ref):
    from ptychox_b200 import synth

    rng = np.random.default_rng(43)
    obj = synth.random_object(128, 128, rng)
    pupil = synth.circular_pupil(32, 0.3)
    led = np.array([[x, y] for y in (40, 48, 56) for x in (44, 48, 52)], dtype=np.int64)
    gout = rng.standard_normal((len(led), 32, 32)).astype(np.float32)
    o = cuda(obj).requires_grad_(True)
    q = cuda(pupil).requires_grad_(True)
    amp = ref.ptychoX_fourier(o, q, cuda(led), use_cuda_kernels=True)
    (amp * cuda(gout)).sum().backward()
    ramp, image, sub = O.fpm_forward(obj, pupil, led)
    rgo, rgp = O.fpm_backward(gout, sub, pupil.astype(np.complex128), image, led, obj.shape)
    assert rel_l2(amp.detach().cpu().numpy(), ramp) < TOL
    assert rel_l2(o.grad.cpu().numpy(), rgo) < TOL
    assert rel_l2(q.grad.cpu().numpy(), rgp) < TOL


def test_reference_coded_function_on_libptychox(ref):
    from ptychox_b200 import synth

    rng = np.random.default_rng(44)
    n = 128
    obj = synth.random_object(n, n, rng)
    mask = synth.binary_mask(n, 0.5, rng)
    t1 = synth.angular_spectrum_transfer(n, 1.85e-6, 0.5e-6, 396.95e-6)
    t2 = synth.angular_spectrum_transfer(n, 1.85e-6, 0.5e-6, 2e-3)
    shifts = synth.coded_shifts(6, 5.0, n, rng).astype(np.float32)
    gout = rng.standard_normal((6, n // 2, n // 2)).astype(np.float32)
    o = cuda(obj).requires_grad_(True)
    m = cuda(mask).requires_grad_(True)
    amp = ref.ptychoX_coded(o, m, cuda(t1), cuda(t2), cuda(shifts), 2, use_cuda_kernels=True)
    (amp * cuda(gout)).sum().backward()
    _, xf, sensor, ramp = O.coded_forward(obj, mask, t1, t2, shifts, 2)
    rgo, rgm = O.coded_backward(gout, xf, sensor, ramp, mask, t1, t2, shifts, 2)
    assert rel_l2(amp.detach().cpu().numpy(), ramp) < TOL
    assert rel_l2(o.grad.cpu().numpy(), rgo) < TOL
    assert rel_l2(m.grad.cpu().numpy(), rgm) < TOL
