"""The learned mismatch coder on a B200: FP32 gradients of the training
kernels against a float64 numpy restatement, and the trained int8 coder on
disjoint evaluation seeds: every stream decodes back to its block (host
decoder, same integer model), and it codes the mismatch gaps and bases in
fewer bytes than the plain coders."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

IN, HID, NB = 128, 128, 4


def _out():
    # output logits (base outcomes + gap bins), from the library's parameter count
    from curc_b200 import learn_param_count
    return (learn_param_count() - (HID * IN + HID + HID * HID + HID)) // (HID + 1)



def _unpack(p):
    OUT = _out()
    o = 0
    out = []
    for shape in [(HID, IN), (HID,), (HID, HID), (HID,), (OUT, HID), (OUT,)]:
        n = int(np.prod(shape))
        out.append(p[o:o + n].reshape(shape))
        o += n
    return out


def _numpy_loss_grads(p, x, tb, tg):
    OUT = _out()
    W1, b1, W2, b2, W3, b3 = _unpack(p.astype(np.float64))
    B = x.shape[0]
    h1 = np.maximum(x @ W1.T + b1, 0)
    h2 = np.maximum(h1 @ W2.T + b2, 0)
    z = h2 @ W3.T + b3
    dz = np.zeros_like(z)
    loss = 0.0
    for b in range(B):
        for o, k, t in ((0, NB, tb[b]), (NB, OUT - NB, tg[b])):
            if t < 0:
                continue
            zz = z[b, o:o + k]
            e = np.exp(zz - zz.max())
            sm = e / e.sum()
            loss += (np.log(e.sum()) + zz.max() - zz[t]) / B
            g = sm.copy()
            g[t] -= 1
            dz[b, o:o + k] = g / B
    dW3 = dz.T @ h2
    db3 = dz.sum(0)
    dh2 = (dz @ W3) * (h2 > 0)
    dW2 = dh2.T @ h1
    db2 = dh2.sum(0)
    dh1 = (dh2 @ W2) * (h1 > 0)
    dW1 = dh1.T @ x
    db1 = dh1.sum(0)
    return loss, np.concatenate([a.ravel() for a in (dW1, db1, dW2, db2, dW3, db3)])


def test_gradients_match_float64():
    from curc_b200 import Learner, learn_param_count
    rng = np.random.default_rng(3)
    n = learn_param_count()
    p = (rng.standard_normal(n) * 0.1).astype(np.float32)
    B = 48
    x = (rng.random((B, IN)) < 0.15).astype(np.float32)
    tb = rng.integers(-1, NB, B).astype(np.int8)
    tg = rng.integers(-1, _out() - NB, B).astype(np.int8)
    with Learner(0) as lrn:
        loss, g = lrn.grad(p, x, tb, tg)
    ref_loss, ref_g = _numpy_loss_grads(p, x, tb, tg)
    assert abs(loss - ref_loss) <= 1e-4 * max(1.0, abs(ref_loss))
    np.testing.assert_allclose(g, ref_g, rtol=1e-3, atol=1e-5)


def test_tensor_core_inference_equals_host_model():
    # the int8 network on tcgen05 (kind::i8, s32 accumulators in TMEM) must
    # give every anchor exactly the frequencies of the host decoder's model
    from curc_b200 import Context, Learner, synth
    w = synth.paired_repeats(seed=77, pairs=40_000, genome_len=400_000, preserve_order=False,
                             ti_tv=2.0, err=synth.position_ramp(150, 0.001, 0.01))
    with Context(0) as ctx, Learner(0) as lrn:
        ctx.block_run(w.sequences(), False, True)
        lrn.add_block(ctx)
        lrn.train(epochs=1, batch=2048)
        n, bad = lrn.infer_check(ctx)
    assert n > 1000
    assert bad == 0, f"{bad} of {n} anchors differ from the host model"


def test_learned_coder_is_lossless_and_smaller():
    from curc_b200.learned import train_and_evaluate
    r = train_and_evaluate(train_seeds=[101, 102, 103, 104], eval_seeds=[201], pairs=60_000, genome_len=600_000,
                           epochs=3, batch=2048)
    assert r["lossless"]
    assert r["train_anchors"] > 10_000
    # gaps and bases: learned stream against the plain base and offset streams
    assert r["gaps_and_bases_ratio"] < 1.0, r
