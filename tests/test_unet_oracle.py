"""Pins the NumPy oracle of the warm-start network (oracle/unet.py) on the
CPU: its analytic FP64 gradients against central finite differences, its
shapes and padding behaviour, and that its BF16-emulating mode stays close
to the FP64 network. The reference has no network, so this is the pin."""

import numpy as np
import pytest

from oracle import unet

N_PARAMS = sum(27 * ci * co + co for _, ci, co in unet.LAYERS)


def random_problem(shape=(8, 8, 8), seed=0):
    rng = np.random.default_rng(seed)
    b = rng.standard_normal(shape)
    p_prev = 0.1 * rng.standard_normal(shape)
    p_target = p_prev + 0.05 * rng.standard_normal(shape)
    params = np.zeros(N_PARAMS)
    for name, (w, bias) in unet.split(params).items():
        cin = w.shape[2]
        w[...] = rng.standard_normal(w.shape) * np.sqrt(2.0 / (27 * cin))
        bias[...] = 0.05 * rng.standard_normal(bias.shape)
    return b, p_prev, p_target, params


def test_parameter_layout():
    assert N_PARAMS == 27 * (16 * 16 * 2 + 16 * 32 + 32 * 32 + 32 * 64 + 64 * 64 + 96 * 32 + 32 * 32 + 48 * 16 + 16 * 16 * 2) + (16 * 2 + 32 * 2 + 64 * 2 + 32 * 2 + 16 * 3)
    flat = np.arange(N_PARAMS, dtype=np.float64)
    assert np.array_equal(unet.join(unet.split(flat)), flat)


def test_conv_gradients_are_adjoint():
    # <conv(x), g> = <x, conv_data_grad(g)> and = <w, conv_weight_grad(x, g)>
    rng = np.random.default_rng(3)
    x = rng.standard_normal((4, 6, 8, 16))
    g = rng.standard_normal((4, 6, 8, 8))
    w = rng.standard_normal((27, 8, 16))
    lhs = np.sum(unet.conv(x, w) * g)
    assert np.isclose(lhs, np.sum(x * unet.conv_data_grad(g, w)), rtol=1e-12)
    dw, db = unet.conv_weight_grad(x, g)
    assert np.isclose(lhs, np.sum(w * dw), rtol=1e-12)
    assert np.allclose(db, g.reshape(-1, 8).sum(0))


def test_gradients_match_finite_differences():
    b, p_prev, p_target, params = random_problem()
    net = unet.UNet(params)
    loss, grad = net.loss_and_gradients(b, p_prev, p_target, 1.0)
    rng = np.random.default_rng(1)
    # every layer's weights and biases, live entries only (input channels
    # 2..15 of the first layer see zeros; only output channel 0 of the last
    # layer reaches the loss)
    offsets, off = [], 0
    for name, ci, co in unet.LAYERS:
        for _ in range(3):
            tap, o, i = rng.integers(27), rng.integers(1 if name == "out" else co), rng.integers(2 if name == "enc0a" else ci)
            offsets.append(off + (tap * co + o) * ci + i)
        offsets.append(off + 27 * ci * co + (0 if name == "out" else rng.integers(co)))
        off += 27 * ci * co + co
    eps = 1e-6
    for k in offsets:
        p1, p2 = params.copy(), params.copy()
        p1[k] += eps
        p2[k] -= eps
        l1 = unet.UNet(p1).loss_and_gradients(b, p_prev, p_target, 1.0)[0]
        l2 = unet.UNet(p2).loss_and_gradients(b, p_prev, p_target, 1.0)[0]
        fd = (l1 - l2) / (2 * eps)
        assert abs(fd - grad[k]) <= 1e-6 * max(1.0, abs(fd)) + 1e-5 * abs(fd), (k, fd, grad[k])


def test_padding_gradients_are_zero():
    b, p_prev, p_target, params = random_problem(seed=2)
    _, grad = unet.UNet(params).loss_and_gradients(b, p_prev, p_target, 1.0)
    parts = unet.split(grad)
    assert np.all(parts["enc0a"][0][:, :, 2:] == 0)
    assert np.all(parts["out"][0][:, 1:, :] == 0) and np.all(parts["out"][1][1:] == 0)


def test_bf16_mode_is_close_to_fp64():
    b, p_prev, p_target, params = random_problem(seed=4)
    l64, g64 = unet.UNet(params).loss_and_gradients(b, p_prev, p_target, 1.0)
    l16, g16 = unet.UNet(params, bf16=True).loss_and_gradients(b, p_prev, p_target, 1.0)
    assert abs(l16 - l64) <= 2e-2 * l64
    assert np.linalg.norm(g16 - g64) <= 5e-2 * np.linalg.norm(g64)


def test_predict_is_previous_plus_scaled_output():
    b, p_prev, _, params = random_problem(seed=5)
    net = unet.UNet(params)
    a = net.forward(b, p_prev, 1.0)
    assert np.allclose(net.predict(b, p_prev, 1.0), p_prev + a["out"] / a["scale"])
    assert a["scale"] == pytest.approx(1.0 / np.sqrt(np.mean(b * b)))
