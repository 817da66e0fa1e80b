"""The CPU restatement of the learned closure's network (oracle/oracle_mlp.c),
which the GPU training and inference kernels are held to: its analytic
gradients against central finite differences, and one Adam step against
the textbook update."""
import numpy as np
import pytest


@pytest.fixture(scope="module")
def mods():
    import pyoracle
    from fesomc import abi
    pyoracle.build()
    return abi, pyoracle


def _random_net(nparams, seed):
    rng = np.random.default_rng(seed)
    return (rng.standard_normal(nparams) * 0.08).astype(np.float32)


@pytest.mark.parametrize("nsigma", [5, 11])
def test_mlp_gradient_matches_finite_differences(mods, nsigma):
    abi, pyoracle = mods
    n_in, n_out = 3 * nsigma + 3, nsigma
    npar = pyoracle.mlp_nparams(abi, nsigma)
    assert npar == n_in * 256 + 256 + 2 * (256 * 256 + 256) + 256 * n_out + n_out
    rng = np.random.default_rng(3)
    p = _random_net(npar, 4)
    X = rng.standard_normal((6, n_in)).astype(np.float32)
    T = rng.standard_normal((6, n_out)).astype(np.float32)
    loss, g = pyoracle.mlp_grad(abi, nsigma, p, X, T)
    Y = pyoracle.mlp_forward(abi, nsigma, p, X)
    assert abs(loss - np.mean((Y.astype(np.float64) - T) ** 2)) < 1e-6 * loss
    # parameters of every layer: some weights and every kind of bias
    offs, o = [], 0
    dims = [n_in, 256, 256, 256, n_out]
    for l in range(4):
        offs.append(o)
        o += dims[l + 1] * dims[l] + dims[l + 1]
    picks = []
    for l in range(4):
        w = dims[l + 1] * dims[l]
        picks += list(offs[l] + rng.integers(0, w, 6)) + list(offs[l] + w + rng.integers(0, dims[l + 1], 2))
    for i in picks:
        h = 1e-2 * max(abs(float(p[i])), 0.05)
        pp, pm = p.copy(), p.copy()
        pp[i] = np.float32(p[i] + h)
        pm[i] = np.float32(p[i] - h)
        hh = float(pp[i]) - float(pm[i])
        fd = (pyoracle.mlp_grad(abi, nsigma, pp, X, T)[0] - pyoracle.mlp_grad(abi, nsigma, pm, X, T)[0]) / hh
        assert abs(fd - g[i]) <= 2e-3 * max(abs(g[i]), 1e-4), (i, fd, g[i])


def test_mlp_adam_step(mods):
    abi, pyoracle = mods
    import ctypes as C
    lib = pyoracle.load(abi)
    p = np.array([1.0, -2.0, 0.5], dtype=np.float32)
    g = np.array([0.1, -0.3, 0.0])
    m = np.zeros(3)
    v = np.zeros(3)
    f = C.POINTER(C.c_float)
    d = C.POINTER(C.c_double)
    lib.oracle_mlp_adam(3, p.ctypes.data_as(f), g.ctypes.data_as(d), m.ctypes.data_as(d), v.ctypes.data_as(d), 1, 0.01)
    # the first Adam step moves every parameter with a non-zero gradient by lr against its sign
    np.testing.assert_allclose(p, [1.0 - 0.01, -2.0 + 0.01, 0.5], rtol=0, atol=1e-6)
