"""The U-Net prior on the B200 against its float64 oracle (oracle/unet.py,
itself held to finite differences on the CPU).

The oracle rounds to BF16 where the GPU stores BF16 (activations, their
gradients, the tensor-core convolutions' weights), so the two differ only
by FP32 summation order and the roundings that order moves:
- forward: every layer's activation within relative L2 1e-2 of the oracle's;
- backward: every parameter gradient within relative L2 1e-2, computed by
  the oracle on the GPU's own forward activations. A ReLU whose input lies
  within a rounding of zero can switch either way in two computations of
  the forward; its gradient then differs at full size, so the backward is
  compared on one set of switches (about 0.07% of the elements switch
  between the two forwards, which alone moves the gradients by 4%)."""

import numpy as np
import pytest
import torch

from oracle import unet as ref
from rexlib_b200 import prior

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm((np.asarray(a) - np.asarray(b)).ravel()) / max(np.linalg.norm(np.asarray(b).ravel()),
                                                                              1e-30))


def oracle_params(net):
    flat = net.parameters().cpu().numpy()
    offsets = {l: net.layer(l)[:2] for l in range(prior.UNet.LAYERS)}
    return ref.unpack(flat, offsets), offsets


def smooth_volume(n, rng):
    # A band-limited random volume (a few Gaussian blobs) plus noise.
    z, y, x = np.meshgrid(*[np.arange(n)] * 3, indexing="ij")
    v = np.zeros((n, n, n))
    for _ in range(6):
        c = rng.uniform(0, n, 3)
        v += rng.uniform(0.5, 1.5) * np.exp(-((z - c[0]) ** 2 + (y - c[1]) ** 2 + (x - c[2]) ** 2) / (2 * (n / 8) ** 2))
    return v


@pytest.mark.parametrize("extent", [16, 32, 64])
def test_forward_and_gradients_match_the_oracle(extent):
    rng = np.random.default_rng(extent)
    net = prior.UNet(extent, seed=7)
    clean = smooth_volume(extent, rng)
    noisy = clean + 0.3 * rng.standard_normal(clean.shape)
    x = torch.from_numpy(noisy.astype(np.float32)).cuda()
    t = torch.from_numpy(clean.astype(np.float32)).cuda()
    y = net.forward(x)
    loss = net.backward(t)
    torch.cuda.synchronize()
    assert net.error() == 0
    params, offsets = oracle_params(net)
    x64 = noisy.astype(np.float32).astype(np.float64)
    t64 = clean.astype(np.float32).astype(np.float64)
    o = ref.Network(params, bf16=True)
    want_y = o.forward(x64)
    gpu_a = {l: net.tensor(l).float().cpu().numpy().astype(np.float64) for l in range(17)}
    for l in range(17):
        assert rel(gpu_a[l], o.a[l]) <= 1e-2, (l, rel(gpu_a[l], o.a[l]))
    y_host = y.cpu().numpy().astype(np.float64)
    assert rel(y_host - x64, want_y - x64) <= 1e-2
    # The backward on the GPU's forward.
    o.a = gpu_a
    o.pools = [ref.to_bf16(ref.pool(gpu_a[l])) for l in (ref.E0, ref.E1, ref.E2)]
    o.y = y_host
    want_loss, want_grads = o.backward(t64)
    assert abs(float(loss.item()) - want_loss) <= 1e-4 * want_loss
    grads = net.gradients().cpu().numpy()
    for layer, (wo, bo) in offsets.items():
        dw, db = want_grads[layer]
        got_w = grads[wo:wo + dw.size].reshape(dw.shape)
        got_b = grads[bo:bo + db.size]
        assert rel(got_w, dw) <= 1e-2, (layer, rel(got_w, dw))
        assert rel(got_b, db) <= 1e-2, (layer, rel(got_b, db))
    net.close()


def test_training_reduces_the_loss():
    # Denoising pairs at 32^3: the loss after 60 Adam steps is well below
    # the first.
    rng = np.random.default_rng(5)
    net = prior.UNet(32, seed=1)
    pairs = []
    for _ in range(8):
        clean = smooth_volume(32, rng)
        pairs.append((torch.from_numpy((clean + 0.3 * rng.standard_normal(clean.shape)).astype(np.float32)).cuda(),
                      torch.from_numpy(clean.astype(np.float32)).cuda()))
    losses = []
    for step in range(60):
        x, t = pairs[step % len(pairs)]
        net.forward(x)
        losses.append(float(net.backward(t).item()))
        net.step(1e-3)
    assert net.error() == 0
    assert np.mean(losses[-8:]) < 0.5 * np.mean(losses[:8]), losses
    net.close()


def test_the_trained_prior_raises_the_resolution():
    # What the trained network gains over the method without it: trained on
    # pairs the library generates at 64^3, then applied as the regulariser
    # (10 iterations) to an unseen phantom, the FSC-0.143 shell against the
    # phantom beats the plain Wiener map from the same particles.
    inputs, targets = prior.make_pairs(64, 64, seed=7, particles=(2000, 10000))
    net = prior.UNet(64, seed=3)
    losses = prior.train(net, inputs, targets, 800, 1e-3)
    assert net.error() == 0
    # One pair a step, recorded every 50 steps: pairs differ in SNR and
    # phantom, so compare means of four records.
    assert np.mean(losses[-4:]) < np.mean(losses[:4]), losses
    rng = np.random.default_rng(8)
    data = prior.Dataset(prior.blob_phantom(rng, 64, 30), 64, 4000, 0.1, seed=9)
    plain, _ = data.resolution(data.wiener())
    base = float(data.den.mean())
    learned = max(data.resolution(prior.regularised(net, data, 10, f * base))[0] for f in (1.0, 3.0, 10.0))
    net.close()
    assert learned > plain, (learned, plain)


def test_backward_reads_the_forward_output_it_returned():
    # The network keeps the output of forward for backward; allocations in
    # between (here the target itself) must not take its memory.
    rng = np.random.default_rng(12)
    net = prior.UNet(16, seed=2)
    x = torch.from_numpy(rng.standard_normal((16, 16, 16)).astype(np.float32)).cuda()
    y = net.forward(x)
    target = x * 0.5
    loss = float(net.backward(target).item())
    want = 0.5 * float(((y.double() - target.double()) ** 2).mean())
    net.close()
    assert want > 0 and abs(loss - want) <= 1e-4 * want, (loss, want)
