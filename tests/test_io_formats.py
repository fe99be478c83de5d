"""Reconstruction files: the reference drivers' torch.save dictionaries, written and read."""

import numpy as np
import torch

from ptychox_b200 import io


def test_keys_match_the_reference_drivers():
    # train_ptychography.py:588-597, train_fpm.py:303-312, train_coded.py:284-293
    assert set(io.reconstruction_dict("conventional", np.zeros((4, 4), np.complex64), np.zeros((2, 2), np.complex64),
                                      np.zeros((3, 2), np.int64), np.zeros((3, 2, 2), np.float32))) == {
        "sample", "probe", "positions_xy", "observed_amplitude", "args"}
    assert set(io.reconstruction_dict("fourier", np.zeros((4, 4), np.complex64), np.zeros((2, 2), np.complex64),
                                      np.zeros((3, 2), np.int64), np.zeros((3, 2, 2), np.float32))) == {
        "object", "pupil", "led_indices_xy", "observed_amplitude", "args"}
    assert set(io.reconstruction_dict("coded", np.zeros((4, 4), np.complex64), np.zeros((4, 4), np.complex64),
                                      np.zeros((3, 2), np.float32), np.zeros((3, 2, 2), np.float32))) == {
        "object", "coded_surface", "shifts_xy_pixels", "observed_amplitude", "args"}
    assert io.FILE_NAMES == {"conventional": "reconstruction.pt", "fourier": "fpm_reconstruction.pt",
                             "coded": "coded_reconstruction.pt", "nearfield": "coded_reconstruction.pt"}


def test_round_trip(tmp_path):
    rng = np.random.default_rng(0)
    obj = (rng.standard_normal((8, 8)) + 1j * rng.standard_normal((8, 8))).astype(np.complex64)
    aux = (rng.standard_normal((4, 4)) + 1j * rng.standard_normal((4, 4))).astype(np.complex64)
    pos = rng.integers(0, 4, (5, 2)).astype(np.int64)
    amp = rng.random((5, 4, 4)).astype(np.float32)
    for modality in ("conventional", "fourier", "coded"):
        path = io.save_reconstruction(tmp_path / modality, modality, torch.from_numpy(obj), aux, pos, amp, {"lr": 0.1})
        got_mod, d = io.load_reconstruction(path)
        assert got_mod == modality
        _, k_obj, k_aux, k_scan = io.KEYS[modality]
        assert d[k_obj].dtype == torch.complex64 and np.array_equal(d[k_obj].numpy(), obj)
        assert np.array_equal(d[k_aux].numpy(), aux) and np.array_equal(d[k_scan].numpy(), pos)
        assert np.array_equal(d["observed_amplitude"].numpy(), amp) and d["args"] == {"lr": 0.1}


def test_matlab_dataset_round_trip(tmp_path):
    """imgRawData.mat as gen_img.m:59 writes it: imRaw [h, w, n] (MATLAB order), ScanPos [n, 2],
    pattern, env struct; read back into [n, h, w] and the near-field arguments."""
    from scipy.io import loadmat

    from ptychox_b200 import io

    rng = np.random.default_rng(0)
    n, pix, mag = 3, 8, 4
    raw = rng.random((n, pix, pix)) * 5 + 1
    pos = rng.uniform(-17, 17, size=(n, 2))
    pattern = (rng.standard_normal((pix * mag, pix * mag)) + 1j * rng.standard_normal((pix * mag, pix * mag)))
    env = {"Fx": rng.random((pix * mag, pix * mag)), "pixSz": 5.86 / mag, "size": np.array([pix * mag, pix * mag])}
    path = io.save_matlab_dataset(tmp_path / "imgRawData.mat", raw, pos, pattern, env)
    m = loadmat(str(path))
    assert m["imRaw"].shape == (pix, pix, n)
    assert np.allclose(m["imRaw"][:, :, 1], raw[1])
    assert m["ScanPos"].shape == (n, 2)
    d = io.load_matlab_dataset(path)
    assert np.allclose(d["im_raw"], raw) and np.allclose(d["scan_pos"], pos)
    assert np.allclose(d["pattern"], pattern.astype(np.complex64))
    assert np.isclose(float(d["env"]["pixSz"]), 5.86 / mag) and np.allclose(d["env"]["Fx"], env["Fx"])
    args = io.nearfield_inputs(d)
    assert args["downsample"] == mag
    assert args["measured"].dtype == np.uint16 and args["measured"].max() == 65535
    assert np.allclose(args["shifts_xy"], pos / pix, atol=1e-6)
    norm = (raw - raw.min()) / (raw - raw.min()).max()
    assert np.max(np.abs(args["measured"] * args["scale"] - norm)) <= 0.5 * args["scale"] + 1e-7
