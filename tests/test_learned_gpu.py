"""GPU parity and behaviour of the learned gauge-covariant preconditioner:
forward pass and training gradient of the CUDA kernels against the numpy
oracle (itself checked by finite differences), training on CG (residual,
error) pairs, and the flexible CG with its true-residual judged fallback."""
import numpy as np
import pytest

from b200dwf import synth

pytestmark = pytest.mark.gpu

# FP32 arithmetic with BF16-valued weights (and the FP32 operator inside the
# loss): the oracle runs in FP64 with the same (deployed) weights, so only
# FP32 rounding separates the two.
TOL_FWD = 2e-5
TOL_GRAD = 5e-4


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def setup(lat, ls, hidden=8, seed=0, kind="hot", mq=0.01, bc=(1, 1, 1, -1)):
    import b200dwf
    u = synth.gauge_field(lat, 300 + seed, kind)
    dev = b200dwf.DomainWall(lat, ls, mq, 1.8, bc=bc)
    dev.set_config(u)
    lp = b200dwf.LearnedPrecond(dev, hidden=hidden, seed=seed + 1)
    return u, dev, lp


def upload_f32(dev, host):
    import b200dwf
    f64 = dev.new_field(b200dwf.F64)
    dev.convert(f64, host)
    f32 = dev.new_field(b200dwf.F32)
    dev.copy_convert(f32, f64)
    return f32


def download(dev, f32):
    import b200dwf
    f64 = dev.new_field(b200dwf.F64)
    dev.copy_convert(f64, f32)
    return dev.reverse(f64)


def random_weights(lp, rng, scale=0.3):
    w = scale * (rng.standard_normal(lp.nparams) + 1j * rng.standard_normal(lp.nparams))
    lp.set_weights(w)


# tc1 rounds the transported inputs to BF16 (8 significant bits) before the
# tensor-core product: its bound is that rounding, not FP32's
KERNEL_TOL = {"tc": (TOL_FWD, 1e-4, TOL_GRAD), "ffma2": (TOL_FWD, 1e-4, TOL_GRAD),
              "tc1": (6e-3, 2e-2, 3e-2)}


@pytest.mark.parametrize("kernel", ["tc", "tc1", "ffma2"])
@pytest.mark.parametrize("lat,ls,hidden,bc", [
    ([4, 4, 4, 4], 4, 8, (1, 1, 1, -1)),
    ([4, 4, 2, 8], 8, 4, (1, -1, 1, -1)),
    ([6, 4, 2, 6], 12, 8, (1, 1, -1, -1)),
])
def test_forward_and_gradient_match_oracle(lat, ls, hidden, bc, kernel, monkeypatch):
    """Every convolution kernel: the tensor-core form (tcgen05, BF16 hi + lo
    split of the transported inputs, FP32 accumulation in tensor memory; the
    default), the tensor-core form on BF16 inputs (B200_LP_CONV=tc1) and the
    packed-FFMA2 form (B200_LP_CONV=ffma2).  The 6x4x2x6
    Ls=12 case has 1728 rows: 13 full 128-row tiles and a ragged 14th."""
    from oracle import learned_oracle as lo
    monkeypatch.setenv("B200_LP_CONV", kernel)
    u, dev, lp = setup(lat, ls, hidden=hidden, bc=bc)
    rng = np.random.default_rng(4)
    random_weights(lp, rng)
    w = lp.weights(deployed=True)
    Ws = lo.split_weights(w, hidden)
    geo = lo.Geometry(lat, u, bc=bc)
    vh = geo.vh
    # the oracle sees the FP32-rounded inputs the kernels see
    r_host = synth.spinor_field(lat, ls, 21).astype(np.float32).astype(np.float64)
    e_host = synth.spinor_field(lat, ls, 22).astype(np.float32).astype(np.float64)
    r = upload_f32(dev, r_host)
    e = upload_f32(dev, e_host)
    z = dev.new_field(1)
    lp.apply(z, r)
    z_dev = lo.spinor_to_act(download(dev, z), vh, ls)
    ra = lo.spinor_to_act(r_host, vh, ls)
    ea = lo.spinor_to_act(e_host, vh, ls)
    from oracle.oracle import OracleDWF
    ora = OracleDWF(lat, ls, 0.01, 1.8, bc=bc)
    ora.set_links(u)

    def A(v):
        return lo.spinor_to_act(ora.mult("DdagD", lo.act_to_spinor(v)), vh, ls)

    loss_ref, G_ref, y_ref = lo.loss_and_grad(geo, Ws, ra, ea, A)
    tol_fwd, tol_loss, tol_grad = KERNEL_TOL[kernel]
    assert rel(z_dev, y_ref) < tol_fwd
    loss = lp.loss_grad(r, e)
    assert abs(loss - loss_ref) < tol_loss * loss_ref
    g = lp.grad()
    assert rel(g, lo.join_weights(G_ref)) < tol_grad
    for layer, (a, b) in enumerate(zip(lo.split_weights(g, hidden), G_ref)):
        assert rel(a, b) < tol_grad, layer


def test_deployed_weights_are_bf16():
    _, dev, lp = setup([4, 4, 4, 4], 4)
    rng = np.random.default_rng(8)
    random_weights(lp, rng)
    w = lp.weights(deployed=True)
    for part in (w.real, w.imag):
        bits = part.astype(np.float32).view(np.uint32)
        assert np.all((bits & 0xFFFF) == 0)
    m = lp.weights(deployed=False)
    assert np.max(np.abs(w - m)) <= 2 ** -8 * np.max(np.abs(m))


def train_network(dev, lp, lat, ls, nsrc=2, nsnap=12, epochs=20, lr=3e-3):
    import b200dwf
    rs, es = [], []
    for k in range(nsrc):
        b = dev.new_field(b200dwf.F64)
        dev.convert(b, synth.spinor_field(lat, ls, 500 + k))
        n_ref, _, _ = dev.cg(dev.new_field(b200dwf.F64), b, 1e-20)
        iters = sorted(set(int(v) for v in np.linspace(2, max(3, n_ref - 2), nsnap)))
        r_k, e_k = b200dwf.cg_training_pairs(dev, b, iters)
        rs += r_k
        es += e_k
    return lp.train(rs, es, epochs, lr)


def test_training_and_flexible_cg():
    import b200dwf
    lat, ls = [4, 4, 4, 8], 8
    _, dev, lp = setup(lat, ls, hidden=8, kind="near")
    l0, l1 = train_network(dev, lp, lat, ls)
    assert l1 < 0.9 * l0, (l0, l1)
    b = dev.new_field(b200dwf.F64)
    dev.convert(b, synth.spinor_field(lat, ls, 77))
    x_cg = dev.new_field(b200dwf.F64)
    n_cg, d_cg, _ = dev.cg(x_cg, b, 1e-20)
    x = dev.new_field(b200dwf.F64)
    n, nfb, d, rc = dev.fcg(x, b, lp, 1e-20, maxiter=2000, mtrunc=8)
    assert rc == 0 and d < 1e-10
    assert rel(dev.reverse(x), dev.reverse(x_cg)) < 1e-8
    # the trained network must save iterations over plain CG
    assert n + nfb < n_cg, (n, nfb, n_cg)


def test_fallback_to_plain_cg_on_useless_network():
    import b200dwf
    lat, ls = [4, 4, 4, 4], 4
    _, dev, lp = setup(lat, ls, hidden=4)
    lp.set_weights(np.zeros(lp.nparams, np.complex128))   # N(r) = 0
    b = dev.new_field(b200dwf.F64)
    dev.convert(b, synth.spinor_field(lat, ls, 5))
    x = dev.new_field(b200dwf.F64)
    n, nfb, d, rc = dev.fcg(x, b, lp, 1e-20, maxiter=20, mtrunc=1)
    assert rc == 0
    assert n == 20 and nfb > 0 and d < 1e-10
