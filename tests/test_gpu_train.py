"""GPU training of the learned correction: the forward / backward kernels'
gradients against the CPU restatement (oracle/mlp_ref.py), and a small
end-to-end run (pairs from the compressor, float + quantization-aware
training, int8 export) whose model the oracle decodes bit for bit and whose
gain over the plain predictor is measured on held-out fields."""
import numpy as np
import pytest

import mlp_ref
import pyoracle as po
import stz_b200

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def random_params(rng):
    p = np.zeros(mlp_ref.NP, np.float32)
    w1 = rng.normal(0, 0.5, (32, 16)).astype(np.float32)
    w1[:, 14:] = 0
    p[mlp_ref.PW1:mlp_ref.PB1] = w1.ravel()
    p[mlp_ref.PB1:mlp_ref.PW2] = rng.normal(0, 0.1, 32)
    p[mlp_ref.PW2:mlp_ref.PB2] = rng.normal(0, 0.3, 1024)
    p[mlp_ref.PB2:mlp_ref.PW3] = rng.normal(0, 0.1, 32)
    w3 = rng.normal(0, 0.3, (8, 32)).astype(np.float32)
    w3[7] = 0
    p[mlp_ref.PW3:mlp_ref.PB3] = w3.ravel()
    p[mlp_ref.PB3:mlp_ref.PB3 + 7] = rng.normal(0, 0.1, 7)
    return p


@pytest.mark.parametrize("qat", [False, True])
@pytest.mark.parametrize("n", [100, 1000, 4096])
def test_gradients_match_cpu_reference(ctx, qat, n):
    rng = np.random.default_rng(n + 7 * qat)
    p = random_params(rng)
    x = np.zeros((n, 16), np.float32)
    x[:, :14] = rng.standard_t(3, (n, 14)) * 30  # heavy tails: some inputs clamp at +-127 s_in
    t = np.zeros((n, 8), np.float32)
    t[:, :7] = rng.standard_t(3, (n, 7)) * 4  # some residuals beyond the Huber delta
    s_in, s_t, delta, sa = 0.6, 3.0, 2.0, (0.004, 0.003)
    loss, g = stz_b200.mlp_grad(ctx, p, x, t, s_in, s_t, delta, qat=qat, sa=sa)
    rl, rg = mlp_ref.step(p, x, t, s_in, s_t, delta, qat=qat, sa=sa)
    assert abs(loss - rl) <= 1e-4 * abs(rl) + 1e-7
    scale = np.abs(rg).max()
    assert scale > 0
    assert np.abs(g - rg).max() <= 2e-4 * scale, np.abs(g - rg).max() / scale
    # structural zeros stay zero
    assert not g[mlp_ref.PW1:mlp_ref.PB1].reshape(32, 16)[:, 14:].any()
    assert not g[mlp_ref.PW3 + 7 * 32:mlp_ref.PB3].any() and g[mlp_ref.PB3 + 7] == 0


def _fields(gens, seeds, shape):
    from stz_b200 import fields

    out = []
    for gen in gens:
        for s in seeds:
            if gen == "grf":
                f = fields.grf(shape, 11.0 / 3.0, s)
            elif gen == "logn":
                f = fields.lognormal(shape, s)
            else:
                f = fields.fronts(shape, s, np.float32)
            out.append((gen, f.astype(np.float32)))
    return out


def test_training_end_to_end_and_gain(ctx):
    shape = (64, 64, 64)
    train = _fields(("grf", "logn", "fronts"), (101, 102), shape)
    held = _fields(("grf", "logn", "fronts"), (201,), (128, 128, 128))
    topts = stz_b200.default_train_opts(epochs=6, qat_epochs=2, batch=2048, sample_step=1, max_pairs=1 << 20)
    tr = stz_b200.Trainer(ctx, train=topts, eb=1e-3, eb_mode="rel", chunk_high=16, chunk_low=8)
    for _, f in train:
        tr.add_field(torch.from_numpy(f).cuda())
    model = tr.fit()
    st = tr.stats()
    tr.close()
    for i in range(2):
        assert st["pairs"][i] > 0
        # the network learned something, and the int8 export kept it
        assert st["loss_float"][i] < st["loss_zero"][i]
        assert st["loss_int8"][i] < st["loss_zero"][i]
        assert st["loss_int8"][i] <= 1.25 * st["loss_qat"][i] + 1e-9
    print("train stats", {k: v for k, v in st.items()})
    m2 = stz_b200.Model.from_bytes(model.to_bytes())
    assert m2.to_bytes() == model.to_bytes()
    gains = {}
    for gen, f in held:
        plain = ctx.compress(f, eb=1e-3, eb_mode="rel", chunk_high=16, chunk_low=8)
        learned = ctx.compress(f, eb=1e-3, eb_mode="rel", chunk_high=16, chunk_low=8, model=model)
        b = learned.to_bytes()
        gains[gen] = len(plain) / len(learned)
        # never worse than the plain stream by more than the model record and flags
        assert len(learned) <= len(plain) + 2 * 2112 + 64
        # the oracle decodes the learned stream bit for bit and the bound holds
        out = ctx.decompress(learned)
        assert np.array_equal(out.view(np.uint32), po.decompress(b).view(np.uint32))
        E = 1e-3 * (float(f.max()) - float(f.min()))
        assert np.abs(out.astype(np.float64) - f).max() <= E
    print("CR learned / plain:", gains)
    # the trained network pays on at least one held-out generator (the flags
    # keep plain cubic wherever it does not)
    assert max(gains.values()) > 1.0, gains
