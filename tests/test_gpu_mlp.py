"""The closure MLP on the tensor cores (csrc/sw2d_mlp.cu, tcgen05 BF16 GEMMs with FP32
accumulation in TMEM) against the FP64 reference with the same BF16 roundings
(closure.reference_forward / reference_loss_grad): the first layer's pre-activations, the
outputs, the loss and the parameter gradient; training with Adam reduces the loss and is
deterministic."""
import numpy as np
import pytest

from tests.conftest import load_pkg

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def C():
    p = load_pkg()
    p.build.build()
    return p.closure


def _setup(seed, n):
    rng = np.random.default_rng(seed)
    norm = np.concatenate([rng.normal(0, 1, 10), rng.uniform(0.5, 2, 10), rng.normal(0, 1, 2),
                           rng.uniform(0.5, 2, 2)]).astype(np.float32)
    x = (rng.normal(0, 1.5, (n, 10)) * norm[10:20] + norm[:10]).astype(np.float32)
    return rng, norm, x


def test_forward_matches_fp64(C):
    """Layer by layer against FP64 with the kernels' BF16 roundings.  Each GEMM is checked on the
    kernel's own inputs (its BF16 activations), so only the FP32 accumulation differs: a wrong
    accumulation order or a dropped K-chunk shows as an error far above 1e-5.  The activations
    (GELU with the hardware tanh, relative error about 2^-11) are within one BF16 unit of the
    FP64 GELU of the kernel's pre-activations, and almost always equal to it.  End to end, the
    outputs are within 1e-3 (norm-wise) of the all-FP64 forward with the same roundings."""
    rng, norm, x = _setup(1, 1000)          # not a multiple of 128: the padded tail
    p = C.init_params(2)
    p[640:704] = rng.normal(0, 0.2, 64)
    net = C.MLP(p, norm)
    y, lay = net.infer(x, layers=True)
    ref = C.reference_forward(p, norm, x)
    w = C.unpack(p)
    z1, h1, z2, h2 = (lay[k].astype(np.float64) for k in range(4))
    # first GEMM + bias: exact products of BF16 operands summed in FP32
    assert np.max(np.abs(z1 - ref["z1"])) <= 1e-5 * (1.0 + np.max(np.abs(ref["z1"])))
    # activations against the FP64 GELU of the kernel's own pre-activations: the hardware tanh's
    # error (about 2^-11 relative to tanh) moves 0.5 z (1 + t) by up to 0.5 |z| 2^-11, which for
    # very negative z is large next to the activation itself; beyond that, one BF16 unit
    for z, h in ((z1, h1), (z2, h2)):
        g = C.bf16(C.gelu(z))
        tol = np.abs(g) * 2.0 ** -7 + np.abs(z) * 2.0 ** -11
        assert np.all(np.abs(h - g) <= tol)
        assert np.mean(h == g) >= 0.95
    # second and third GEMMs on the kernel's activations
    z2_k = h1 @ C.bf16(w["W2"]).T + w["b2"]
    assert np.max(np.abs(z2 - z2_k)) <= 1e-5 * (1.0 + np.max(np.abs(z2_k)))
    ym, ys = norm[20:22].astype(np.float64), norm[22:24].astype(np.float64)
    y_k = (h2 @ C.bf16(w["W3"]).T + w["b3"]) * ys + ym
    assert np.max(np.abs(y - y_k)) <= 1e-5 * (1.0 + np.max(np.abs(y_k)))
    # end to end against the all-FP64 forward
    err_z2 = np.linalg.norm(z2 - ref["z2"]) / np.linalg.norm(ref["z2"])
    err_y = np.linalg.norm(y - ref["y"]) / np.linalg.norm(ref["y"] - ym)
    print(f"forward: z2 norm-wise {err_z2:.2e}, y norm-wise {err_y:.2e}")
    assert err_z2 <= 1e-3 and err_y <= 1e-3


def test_gradient_matches_fp64(C):
    rng, norm, x = _setup(4, 4096)
    t = rng.normal(0, 1, (4096, 2)).astype(np.float32) * norm[22:24] + norm[20:22]
    p = C.init_params(6)
    net = C.MLP(p, norm)
    loss, g = net.loss_grad(x, t)
    rloss, rg = C.reference_loss_grad(p, norm, x, t)
    assert abs(loss - rloss) <= 1e-4 * abs(rloss)
    k = 0
    errs = {}
    for name, shape in C.SHAPES:
        nk = int(np.prod(shape))
        a, b = g[k:k + nk].astype(np.float64), rg[k:k + nk]
        errs[name] = float(np.linalg.norm(a - b) / (np.linalg.norm(b) + 1e-30))
        k += nk
    print("gradient norm-wise errors:", {n: f"{e:.2e}" for n, e in errs.items()})
    # the backward layers differ from FP64 only by the hardware tanh in GELU' and the BF16
    # roundings of dZ2, dZ1 that it flips
    for name, e in errs.items():
        assert e <= 1e-3, (name, e)


def test_training_reduces_loss_and_is_deterministic(C):
    rng = np.random.default_rng(7)
    x = rng.uniform(-2, 2, (16384, 10)).astype(np.float32)
    t = np.stack([np.sin(x[:, 0]) + 0.5 * x[:, 1] * x[:, 2], np.tanh(x[:, 3]) - 0.3 * x[:, 4] ** 2], 1)
    t = t.astype(np.float32)
    norm = np.concatenate([x.mean(0), x.std(0), t.mean(0), t.std(0)]).astype(np.float32)
    runs = []
    for _ in range(2):
        net = C.MLP(C.init_params(8), norm)
        hist = net.train(x, t, epochs=12, batch=2048, lr=3e-3, seed=9)
        runs.append((hist, net.params))
    hist = runs[0][0]
    assert hist[-1] < 0.05 * hist[0], hist
    assert np.array_equal(runs[0][1].view(np.int32), runs[1][1].view(np.int32))


def test_tensor_core_wait_that_runs_out(C):
    """A first wait on the tensor core that gives up at once (poll limit 0): the GEMM kernel sets
    the status, waits once more with the full limit for the MMA in flight, frees its TMEM and
    returns; the call fails with "tensor-core wait ran out".  Back to the default limit, the same
    network gives the same outputs as before, twice (its TMEM was released and the status was
    cleared after being reported)."""
    rng, norm, x = _setup(9, 700)
    net = C.MLP(C.init_params(3), norm)
    y0 = net.infer(x)
    net.set_wait_polls(0)
    for _ in range(2):
        with pytest.raises(RuntimeError, match="tensor-core wait ran out"):
            net.infer(x)
    net.set_wait_polls(-1)
    for _ in range(2):
        y1 = net.infer(x)
        assert np.array_equal(y0.view(np.int32), y1.view(np.int32))
