"""The numpy oracle against golden vectors produced by the reference's own PyTorch path.

This pins the oracle: every CUDA parity test compares against the oracle (and the same
fixtures), so the oracle must reproduce the reference on every case the fixtures hold.
"""

import numpy as np
import pytest

from conftest import load_golden, rel_l2
from oracle import ptycho_oracle as O

# complex64 reference vs FP64 oracle on the same inputs: FP32 rounding only
TOL_C64 = 2e-6
# FP64 reference vs FP64 oracle: different FFT libraries, same math
TOL_F64 = 1e-10


def test_test_ops_base():
    g = load_golden("test_ops_base.npz")
    amp, far, patches = O.base_forward(g["sample"], g["probe"], g["positions"])
    assert rel_l2(amp, g["out"]) < TOL_C64
    gs, gp = O.base_backward(g["grad"], patches, g["probe"].astype(np.complex128), far, g["positions"],
                             g["sample"].shape)
    assert rel_l2(gs, g["grad_sample"]) < TOL_C64
    assert rel_l2(gp, g["grad_probe"]) < TOL_C64


def test_test_ops_fpm():
    g = load_golden("test_ops_fpm.npz")
    amp, image, sub = O.fpm_forward(g["object"], g["pupil"], g["leds"])
    assert rel_l2(amp, g["out"]) < TOL_C64
    go, gp = O.fpm_backward(g["grad"], sub, g["pupil"].astype(np.complex128), image, g["leds"], g["object"].shape)
    assert rel_l2(go, g["grad_object"]) < TOL_C64
    assert rel_l2(gp, g["grad_pupil"]) < TOL_C64


def test_test_ops_coded():
    g = load_golden("test_ops_coded.npz")
    ds = int(g["downsample"])
    _, xf, sensor, amp = O.coded_forward(g["object"], g["mask"], g["transfer_1"], g["transfer_2"], g["shifts"], ds)
    assert rel_l2(amp, g["out"]) < TOL_C64
    go, gm = O.coded_backward(g["grad"], xf, sensor, amp, g["mask"], g["transfer_1"], g["transfer_2"], g["shifts"], ds)
    assert rel_l2(go, g["grad_object"]) < 5 * TOL_C64
    assert rel_l2(gm, g["grad_mask"]) < 5 * TOL_C64


@pytest.mark.parametrize("name", ["sweep_base_fp64.npz", "sweep_base_odd_fp64.npz"])
def test_sweep_base(name):
    g = load_golden(name)
    loss, gs, gp = O.base_sweep(g["sample"], g["probe"], g["positions"], g["measured"], float(g["scale"]))
    assert abs(loss - float(g["loss"])) <= TOL_F64 * abs(float(g["loss"]))
    assert rel_l2(gs, g["grad_sample"]) < TOL_F64
    assert rel_l2(gp, g["grad_probe"]) < TOL_F64


def test_sweep_fpm():
    g = load_golden("sweep_fpm_fp64.npz")
    loss, go, gp = O.fpm_sweep(g["object"], g["pupil"], g["leds"], g["measured"], float(g["scale"]))
    assert abs(loss - float(g["loss"])) <= TOL_F64 * abs(float(g["loss"]))
    assert rel_l2(go, g["grad_object"]) < TOL_F64
    assert rel_l2(gp, g["grad_pupil"]) < TOL_F64


@pytest.mark.parametrize("name", ["sweep_coded_fp64.npz", "sweep_nearfield_fp64.npz"])
def test_sweep_coded(name):
    g = load_golden(name)
    t1 = None if bool(g["nearfield"]) else g["transfer_1"]
    loss, go, gm = O.coded_sweep(g["object"], g["mask"], t1, g["transfer_2"], g["shifts"], int(g["downsample"]),
                                 g["measured"], float(g["scale"]))
    assert abs(loss - float(g["loss"])) <= TOL_F64 * abs(float(g["loss"]))
    assert rel_l2(go, g["grad_object"]) < TOL_F64
    assert rel_l2(gm, g["grad_mask"]) < TOL_F64


def test_nearfield_is_coded_with_unit_transfer():
    g = load_golden("sweep_nearfield_fp64.npz")
    ones = np.ones_like(g["transfer_2"])
    a = O.coded_sweep(g["object"], g["mask"], ones, g["transfer_2"], g["shifts"], int(g["downsample"]),
                      g["measured"], float(g["scale"]))
    b = O.nearfield_sweep(g["object"], g["mask"], g["transfer_2"], g["shifts"], int(g["downsample"]),
                          g["measured"], float(g["scale"]))
    assert abs(a[0] - b[0]) <= 1e-13 * abs(a[0])
    assert rel_l2(a[1], b[1]) < 1e-13 and rel_l2(a[2], b[2]) < 1e-13


@pytest.mark.parametrize("name,loss", [("sweep_coded_fd_iso_fp64.npz", "fd-isotropic"),
                                       ("sweep_coded_fd_aniso_fp64.npz", "fd-anisotropic")])
def test_sweep_coded_fd_loss(name, loss):
    """The fd_loss data term (train_coded.py:101-107) against the reference's own function."""
    g = load_golden(name)
    got, go, gm = O.coded_sweep(g["object"], g["mask"], g["transfer_1"], g["transfer_2"], g["shifts"],
                                int(g["downsample"]), g["measured"], float(g["scale"]), loss=loss)
    assert abs(got - float(g["loss"])) <= TOL_F64 * abs(float(g["loss"]))
    assert rel_l2(go, g["grad_object"]) < TOL_F64
    assert rel_l2(gm, g["grad_mask"]) < TOL_F64


def test_coded_shift_gradient():
    """dL/dshifts: the reference's torch formulation is differentiable in shifts_xy through
    shift_phase_ramp (coded/ops.py:157-171); the oracle's closed form matches its autograd."""
    g = load_golden("sweep_coded_shifts_fp64.npz")
    loss, go, gm, gs = O.coded_sweep(g["object"], g["mask"], g["transfer_1"], g["transfer_2"], g["shifts"],
                                     int(g["downsample"]), g["measured"], float(g["scale"]), with_shifts=True)
    assert abs(loss - float(g["loss"])) <= TOL_F64 * abs(float(g["loss"]))
    assert rel_l2(go, g["grad_object"]) < TOL_F64
    assert rel_l2(gm, g["grad_mask"]) < TOL_F64
    assert rel_l2(gs, g["grad_shifts"]) < TOL_F64


def test_sweep_base_subpixel():
    """Sub-pixel conventional sweep: the oracle against the fixture composed from the reference's
    own crop, shift_phase_ramp and ptychoX_base (rectangular 16 x 32 probe, real jitter)."""
    g = load_golden("sweep_base_subpix_fp64.npz")
    assert np.any(np.abs(g["positions"] - np.round(g["positions"])) > 0.1)
    loss, gs, gp = O.base_subpix_sweep(g["sample"], g["probe"], g["positions"], g["measured"], float(g["scale"]))
    assert abs(loss - float(g["loss"])) <= TOL_F64 * abs(float(g["loss"]))
    assert rel_l2(gs, g["grad_sample"]) < TOL_F64
    assert rel_l2(gp, g["grad_probe"]) < TOL_F64
    chunked = O.base_subpix_sweep(g["sample"], g["probe"], g["positions"], g["measured"], float(g["scale"]), chunk=5)
    assert abs(chunked[0] - loss) <= 1e-12 * abs(loss)
    assert rel_l2(chunked[1], gs) < 1e-12 and rel_l2(chunked[2], gp) < 1e-12


def test_subpixel_integer_positions_equal_base():
    """At integer positions the sub-pixel operator is the conventional one."""
    g = load_golden("sweep_base_fp64.npz")
    pos = g["positions"].astype(np.float64)
    a = O.base_sweep(g["sample"], g["probe"], g["positions"], g["measured"], float(g["scale"]))
    b = O.base_subpix_sweep(g["sample"], g["probe"], pos, g["measured"], float(g["scale"]))
    assert abs(a[0] - b[0]) <= 1e-12 * abs(a[0])
    assert rel_l2(b[1], a[1]) < 1e-12 and rel_l2(b[2], a[2]) < 1e-12
