"""The closure MLP's FP64 reference (closure.reference_forward / reference_loss_grad): its
backward formulas against central differences of its forward (no rounding), and the BF16
rounding helper.  CPU only; tests/test_gpu_mlp.py checks the tensor-core kernels against it."""
import numpy as np

from tests.conftest import load_pkg

C = load_pkg().closure


def test_bf16_rounding():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 2 ** -9, 1.0 + 3 * 2 ** -9, -2.5, 3.0e-3], dtype=np.float32)
    r = C.bf16(x)
    assert r[0] == 1.0 and r[2] == 1.0 and r[3] == 1.0 + 2 ** -7  # ties to even
    # bfloat16 keeps 8 significant bits: values are multiples of 2^(e-7)
    for v, w in zip(x.astype(np.float64), r):
        e = np.floor(np.log2(abs(v)))
        q = 2.0 ** (e - 7)
        assert abs(w - v) <= q / 2 + 1e-30
        assert abs(w / q - round(w / q)) < 1e-9


def test_reference_gradient_matches_central_differences():
    rng = np.random.default_rng(3)
    p = C.init_params(5).astype(np.float64)
    p[C.N_HID * C.N_IN:C.N_HID * C.N_IN + C.N_HID] = rng.normal(0, 0.1, C.N_HID)
    norm = np.concatenate([rng.normal(0, 1, 10), rng.uniform(0.5, 2, 10), rng.normal(0, 1, 2), rng.uniform(0.5, 2, 2)])
    x = rng.normal(0, 1.5, (37, 10))
    t = rng.normal(0, 1, (37, 2))
    loss, g = C.reference_loss_grad(p, norm, x, t, rounding=False)
    for k in rng.choice(p.size, 40, replace=False):
        e = 1e-6
        pp, pm = p.copy(), p.copy()
        pp[k] += e
        pm[k] -= e
        fd = (C.reference_loss_grad(pp, norm, x, t, rounding=False)[0] -
              C.reference_loss_grad(pm, norm, x, t, rounding=False)[0]) / (2 * e)
        assert abs(fd - g[k]) <= 1e-6 * max(1.0, abs(fd)), (k, fd, g[k])
