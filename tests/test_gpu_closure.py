"""Learned vertical-mixing closure on the GPU, through the C-ABI: the
hand-written FP32 training kernels against the CPU restatement of the
network (oracle/oracle_mlp.c); the fallback and judge paths, which must give
the plain closure's bits; and training on columns harvested from the plain
closure, with what the trained network gains over running without it."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIELDS = ["eta_n", "U_n_2D", "U_n", "V_n", "TF", "SF", "bt", "snu", "Kv", "Av", "Wvel", "mask_wd_node"]


@pytest.fixture(scope="module")
def mods(built):
    import pyoracle
    from fesomc import abi, cases, closure, model
    return abi, cases, closure, model, pyoracle


def _rand(shape, seed, scale=1.0):
    return (np.random.default_rng(seed).standard_normal(shape) * scale).astype(np.float32)


@pytest.mark.parametrize("nsigma,batch", [(21, 96), (11, 700)])
def test_gradients_match_oracle(mods, nsigma, batch):
    """Loss and every parameter's gradient of one batch (FP32 tiled SGEMM
    forward / backward on the GPU) against the CPU restatement (double
    accumulation): relative 1e-3 on each gradient array, 1e-5 on the loss."""
    abi, cases, closure, model, pyoracle = mods
    c = closure.Closure(nsigma)
    try:
        p = _rand(c.nparams, 1, 0.06)
        c.params(p)
        X = _rand((batch, c.n_in), 2)
        T = _rand((batch, c.n_out), 3)
        loss, g = c.grad(X, T)
        lo, go = pyoracle.mlp_grad(abi, nsigma, p, X, T)
        assert abs(loss - lo) <= 1e-5 * lo
        dims = [c.n_in, 256, 256, 256, c.n_out]
        o = 0
        for l in range(4):
            for n in (dims[l + 1] * dims[l], dims[l + 1]):
                a, b = g[o:o + n].astype(np.float64), go[o:o + n]
                assert np.linalg.norm(a - b) <= 1e-3 * np.linalg.norm(b), (l, n)
                o += n
        assert o == c.nparams
        Y = c.forward(X)
        Yo = pyoracle.mlp_forward(abi, nsigma, p, X)
        assert np.max(np.abs(Y - Yo)) <= 1e-5 * np.max(np.abs(Yo)) + 1e-6
    finally:
        c.close()


def _bf16(a):
    """Round float32 values to bfloat16 (nearest even), returned as float32."""
    u = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def _net_bf16_reference(p, X, n_in, n_out):
    """The network with BF16 inputs, weights and hidden activations and FP32
    (here float64) accumulation, as the tensor-core kernel computes it."""
    dims = [n_in, 256, 256, 256, n_out]
    o, a = 0, _bf16(X).astype(np.float64)
    for l in range(4):
        W = _bf16(p[o:o + dims[l + 1] * dims[l]]).reshape(dims[l + 1], dims[l]).astype(np.float64)
        o += dims[l + 1] * dims[l]
        b = p[o:o + dims[l + 1]].astype(np.float64)
        o += dims[l + 1]
        z = a @ W.T + b
        a = _bf16((z / (1.0 + np.exp(-z))).astype(np.float32)).astype(np.float64) if l < 3 else z
    return a


@pytest.mark.parametrize("nsigma,ncol", [(21, 1000), (11, 300), (21, 5)])
def test_tensor_core_inference(mods, nsigma, ncol):
    """The BF16 tensor-core kernel (tcgen05.mma, TMEM accumulators) against
    the same network with the same BF16 roundings on the CPU (relative 2e-3:
    FP32 accumulation order and the SiLU's exp), and against the FP32
    network (relative 3e-2, the BF16 rounding itself); partial last tiles
    included."""
    abi, cases, closure, model, pyoracle = mods
    c = closure.Closure(nsigma)
    try:
        p = _rand(c.nparams, 7, 0.06)
        c.params(p)
        X = _rand((ncol, c.n_in), 8)
        Yt = c.forward(X, bf16=True).astype(np.float64)
        Yb = _net_bf16_reference(p, X, c.n_in, c.n_out)
        Yf = pyoracle.mlp_forward(abi, nsigma, p, X).astype(np.float64)
        scale = np.max(np.abs(Yf))
        assert np.max(np.abs(Yt - Yb)) <= 2e-3 * scale
        assert np.max(np.abs(Yt - Yf)) <= 3e-2 * scale
        # repeatable, and agrees with the FP32 GPU kernels to the BF16 level
        assert np.array_equal(Yt, c.forward(X, bf16=True).astype(np.float64))
        assert np.max(np.abs(Yt - c.forward(X).astype(np.float64))) <= 3e-2 * scale
    finally:
        c.close()


def _harvested(mods, steps=40, every=4, **kw):
    abi, cases, closure, model, pyoracle = mods
    case = cases.estuary("small", **kw)
    c = closure.Closure(case.mesh.NS, capacity=200_000)
    g = model.GpuModel(case)
    g.set_forcing(case.forcing_fn(1, cases.advance_time(g.time_jd, case.params.dt)))
    c.harvest(g, steps, every)
    g.close()
    c.fit()
    return case, c


def _run(mods, case, steps, c=None, judge=0, ver_mix=None):
    abi, cases, closure, model, pyoracle = mods
    if ver_mix is not None:
        case.params.ver_mix = ver_mix
    g = model.GpuModel(case)
    try:
        g.set_forcing(case.forcing_fn(1, cases.advance_time(g.time_jd, case.params.dt)))
        if c is not None:
            c.attach(g, judge)
        g.run(steps)
        st = g.state()
        rep = closure.Closure.stats(g) if c is not None else None
    finally:
        g.close()
    return st, rep


def test_harvest_and_envelope(mods):
    """Harvest appends the wet columns of every 'every'-th step; the
    statistics give a finite normalisation and an envelope around every
    input."""
    abi, cases, closure, model, pyoracle = mods
    case, c = _harvested(mods, steps=12, every=4)
    try:
        wet = int(case.state0["mask_wd_node"].sum())
        n = c.harvested()
        assert 2 * wet <= n <= 3 * case.mesh.N
        st = c.norm()
        assert np.all(np.isfinite(st[:4])) and np.all(st[1, :c.n_in] > 0) and np.all(st[3, :c.n_out] > 0)
        assert np.all(st[4, :c.n_in] <= 0.0) and np.all(st[5, :c.n_in] >= 0.0)
        # targets: log bt of the plain closure (bt >= 1e-8), their range kept
        lo, hi = st[6, :c.n_out], st[7, :c.n_out]
        assert np.all(np.isfinite(lo)) and np.all(lo <= hi) and np.all(lo >= np.log(1e-8) - 1e-4)
    finally:
        c.close()


def test_fallback_everywhere_gives_the_plain_step(mods):
    """With an envelope no column fits, every column goes to the plain
    closure through the column list: the run equals the plain run bit for bit,
    and the counters say every wet column fell back."""
    abi, cases, closure, model, pyoracle = mods
    case, c = _harvested(mods)
    try:
        st = c.norm()
        st[4, :] = 1.0e30            # envelope low above every input
        c.norm(st)
        ref, _ = _run(mods, case, 15)
        got, rep = _run(mods, case, 15, c)
        for f in FIELDS:
            assert np.array_equal(ref[f], got[f]), f
        assert rep["steps"] == 15 and rep["wet_columns"] > 0
        assert rep["out_of_envelope"] == rep["wet_columns"]
    finally:
        c.close()


def test_judge_every_step_gives_the_plain_step(mods):
    """judge_every = 1: the plain closure runs on every column every step and
    the network is only compared with it, so the run equals the plain run bit
    for bit and the judge has compared values."""
    abi, cases, closure, model, pyoracle = mods
    case, c = _harvested(mods)
    try:
        ref, _ = _run(mods, case, 12)
        got, rep = _run(mods, case, 12, c, judge=1)
        for f in FIELDS:
            assert np.array_equal(ref[f], got[f]), f
        assert rep["judge_steps"] == 12 and rep["judge_values"] > 0 and np.isfinite(rep["judge_rms_log"])
    finally:
        c.close()


def test_training_learns_and_beats_no_closure(mods):
    """Columns harvested from the plain closure under wind and a surface heat
    loss train the network (loss falls); the trained network is closer to
    the plain closure than the untrained one (judge); and a run with the
    trained closure stays closer to the plain-closure run than a run without
    any turbulence closure (ver_mix = 0: background viscosity only), in
    temperature, salinity and velocity."""
    abi, cases, closure, model, pyoracle = mods
    atm = {"qns": -100.0, "qsr": 0.0, "emp": 0.0}
    case, c = _harvested(mods, steps=300, every=3, atm=atm)
    try:
        _, rep0 = _run(mods, case, 6, c, judge=1)
        losses = c.train(24, batch=512, lr=5e-4, seed=2)
        # the epoch losses of small minibatches are noisy: the best of the
        # last six against the first
        assert np.all(np.isfinite(losses)) and np.min(losses[-6:]) < 0.5 * losses[0], list(losses)
        _, rep1 = _run(mods, case, 6, c, judge=1)
        assert rep1["judge_rms_log"] < 0.6 * rep0["judge_rms_log"], (rep0, rep1, list(losses))
        steps = 120
        ref, _ = _run(mods, case, steps)
        lc, rep = _run(mods, case, steps, c, judge=20)
        none, _ = _run(mods, cases.estuary("small", atm=atm), steps, ver_mix=0)
        assert rep["wet_columns"] > 0
        assert rep["out_of_envelope"] < 0.5 * rep["wet_columns"]
        for f in ("TF", "SF", "U_n"):
            assert np.all(np.isfinite(lc[f]))
            e_lc = np.sqrt(np.mean((lc[f] - ref[f]) ** 2))
            e_none = np.sqrt(np.mean((none[f] - ref[f]) ** 2))
            assert e_lc < e_none, (f, e_lc, e_none)
    finally:
        c.close()


def test_fallback_rules_take_their_columns(mods):
    """The boundary and convective-column rules hand more columns to the
    plain closure than the envelope alone (counted as out of the envelope);
    judging every step keeps the plain closure's state, so the three runs
    see the same columns.  Unknown rule bits are refused."""
    abi, cases, closure, model, pyoracle = mods
    case, c = _harvested(mods)
    try:
        assert c.lib.fesomc_closure_set_rules(c.h, 8) == 1
        counts = {}
        for name, kw in (("none", {}), ("boundary", {"boundary": True}), ("unstable", {"unstable": True})):
            c.set_rules(**kw)
            _, rep = _run(mods, case, 4, c, judge=1)
            counts[name] = rep["out_of_envelope"]
            assert rep["wet_columns"] > 0
        nb = int(np.count_nonzero(case.mesh.index_nod2D != 0))
        assert counts["boundary"] > counts["none"]
        assert counts["boundary"] - counts["none"] <= 4 * nb
        assert counts["unstable"] >= counts["none"]
    finally:
        c.set_rules()
        c.close()
