"""The bounce transport and its adjoint on the device (lb_transport_*), against the oracle:

- every recorded gather ray equals the oracle's trace of the same ray (trace.wgsl:245-270), bit for bit;
- the forward at the scene's own theta is the device bake's indirect atlas, bit for bit, and at edited
  albedos and sky it is the bake of the edited scene, bit for bit, the texels lit by the volume's
  fallback included;
- the gradient equals the float64 restatement's autograd gradient (oracle/transport_ref.py) and central
  differences of the forward (h = 1e-3);
- fewer checkpoints than bounces (recomputation) give the same bits, and so does a second call.
"""
import numpy as np
import pytest

import lightbaker_b200 as lb
from lightbaker_b200 import scenes

import oracle
from oracle import transport_ref as T

pytestmark = pytest.mark.gpu

EXPORTS = ["shape", "tiles", "texels", "chart", "gathered", "known", "known_bounce", "state", "direct_light",
           "fixed_indirect", "owner", "gathered_index", "records", "smooth_weights", "sample_points",
           "volume_grid", "volume_items", "volume_slots", "volume_raw", "volume_records"]


@pytest.fixture(scope="module")
def small(gpu):
    scene = scenes.small_map(seed=3, bounces=2)
    tr = lb.Transport(scene, gpu)
    yield scene, tr
    tr.close()


@pytest.fixture(scope="module")
def reftest(gpu):
    scene = scenes.reference_test()
    tr = lb.Transport(scene, gpu)
    yield scene, tr
    tr.close()


@pytest.fixture(scope="module")
def inside(gpu):
    """Boxes sunk into each other and into the ground: texels inside solids lit by the volume's fallback, and
    probes inside solids that the volume's fill gives light."""
    from edge_scenes import EDGE_SCENES
    scene = EDGE_SCENES["inside"]()
    tr = lb.Transport(scene, gpu)
    yield scene, tr
    tr.close()


def _arrays(tr):
    return {k: tr.export(k) for k in EXPORTS}


@pytest.mark.parametrize("which", ["small", "reftest"])
def test_records_are_the_oracle_rays(which, request):
    scene, tr = request.getfixturevalue(which)
    P = lb.prepare(scene)
    sc = oracle.Scene.of(P)
    idx = tr.export("gathered_index")
    tex = tr.export("texels").reshape(-1, 4, 4)
    pos = tr.export("sample_points")
    items = np.zeros(len(idx), lb.TEXEL)
    items["pos"] = pos[idx]
    items["normal"] = tex[idx, 1]
    items["dx"] = tex[idx, 2]
    items["dy"] = tex[idx, 3]
    shape = tr.export("shape")
    want = oracle.gather_records(sc, P.params, items, int(shape[0]) * int(shape[1]))
    got = tr.export("records").reshape(len(idx), -1, 2)
    kind = got[:, :, 0] >> 30
    np.testing.assert_array_equal(kind, want[:, :, 0])
    surf = kind == 2
    np.testing.assert_array_equal((got[:, :, 0] & 0x3FFFFFFF)[surf], want[:, :, 1][surf])
    np.testing.assert_array_equal(got[:, :, 1][surf], want[:, :, 2][surf])
    sky = kind == 0
    np.testing.assert_array_equal(got[:, :, 1][sky], want[:, :, 3][sky])
    assert surf.any() and sky.any()


@pytest.mark.parametrize("which", ["small", "reftest", "inside"])
def test_forward_at_theta0_is_the_bake(which, request, gpu):
    scene, tr = request.getfixturevalue(which)
    got = tr.forward(tr.theta0())
    want = tr.bake_indirect()
    np.testing.assert_array_equal(got.view(np.uint32), want.view(np.uint32))
    baked = lb.bake_device(scene, gpu).indirect
    np.testing.assert_array_equal(got.view(np.uint32), np.asarray(baked, np.float32).reshape(got.shape).view(np.uint32))


def test_forward_is_the_bake_of_the_edited_scene(reftest, gpu):
    scene, tr = reftest
    assert (tr.export("state") == 5).sum() == 0  # no fallback texels: the whole atlas is the transport's
    rng = np.random.default_rng(7)
    th = tr.theta0()
    M = tr.n_materials
    th[:3 * M] = rng.uniform(0.1, 0.9, 3 * M).astype(np.float32)
    th[3 * M:3 * M + 9] = rng.uniform(0.05, 0.6, 9).astype(np.float32)
    edited = scenes.with_light(scene, albedo=th[:3 * M], zenith=th[3 * M:3 * M + 3], horizon=th[3 * M + 3:3 * M + 6],
                               ground=th[3 * M + 6:3 * M + 9])
    want = np.asarray(lb.bake_device(edited, gpu).indirect, np.float32).reshape(tr.ih, tr.iw, 3)
    got = tr.forward(th)
    np.testing.assert_array_equal(got.view(np.uint32), want.view(np.uint32))
    # the sun's scale: the direct light scales with it (rounding aside)
    th2 = tr.theta0()
    th2[-1] = 1.5
    edited = scenes.with_light(scene, irradiance=np.float32(1.5) * np.array([3.0, 3.0, 3.0], np.float32))
    want = np.asarray(lb.bake_device(edited, gpu).indirect, np.float32).reshape(tr.ih, tr.iw, 3)
    np.testing.assert_allclose(tr.forward(th2), want, rtol=1e-5, atol=1e-6)


@pytest.mark.parametrize("which", ["small", "inside"])
def test_forward_with_the_volume_is_the_bake_of_the_edited_scene(which, request, gpu):
    """Texels lit by the volume's fallback (validity 5) take their light from the probes, which the transport
    evaluates from its last bounce's light and theta, fills and interpolates: at edited albedos and sky the
    forward is the bake of the edited scene bit for bit, those texels included."""
    scene, tr = request.getfixturevalue(which)
    assert (tr.export("state") == 5).sum() > 0 and len(tr.export("volume_grid")) == 10
    rng = np.random.default_rng(5)
    th = tr.theta0()
    M = tr.n_materials
    th[:3 * M] = rng.uniform(0.1, 0.9, 3 * M).astype(np.float32)
    th[3 * M:3 * M + 9] = rng.uniform(0.05, 0.6, 9).astype(np.float32)
    edited = scenes.with_light(scene, albedo=th[:3 * M], zenith=th[3 * M:3 * M + 3], horizon=th[3 * M + 3:3 * M + 6],
                               ground=th[3 * M + 6:3 * M + 9])
    want = np.asarray(lb.bake_device(edited, gpu).indirect, np.float32).reshape(tr.ih, tr.iw, 3)
    got = tr.forward(th)
    np.testing.assert_array_equal(got.view(np.uint32), want.view(np.uint32))


def test_fallback_texels_have_a_gradient(inside):
    """On a scene whose fallback texels are lit through filled probes, the gradient of a loss on the whole
    atlas (the fallback texels' share reaching the sky and the albedos through the probes) equals central
    differences of the forward."""
    scene, tr = inside
    th = tr.theta0()
    state = tr.export("state")
    tr.forward(th)
    # the composite spreads a texel over its block: weigh the whole atlas, the fallback texels' blocks most
    g = np.full((tr.ih, tr.iw, 3), 0.1, np.float32)
    grad = tr.backward(g)
    M = tr.n_materials
    h = 1e-3
    for j in [3 * M, 3 * M + 4, 3 * M + 7, 0, 4]:
        tp, tm = th.copy(), th.copy()
        tp[j] += h
        tm[j] -= h
        fd = ((tr.forward(tp).astype(np.float64) * g).sum() - (tr.forward(tm).astype(np.float64) * g).sum()) / (2 * h)
        assert abs(fd - grad[j]) <= 2e-3 * max(abs(grad[j]), 1e-3 * np.abs(grad).max()), (j, fd, grad[j])
    assert (state == 5).sum() > 0


@pytest.mark.parametrize("which", ["small", "reftest", "inside"])
def test_gradient_is_the_float64_reference(which, request):
    scene, tr = request.getfixturevalue(which)
    ref = T.TransportRef(_arrays(tr))
    rng = np.random.default_rng(11)
    th = tr.theta0()
    th[:-1] *= rng.uniform(0.8, 1.2, len(th) - 1).astype(np.float32)
    th[-1] = 1.1
    g = rng.normal(size=(tr.ih, tr.iw, 3)).astype(np.float32)
    out = tr.forward(th)
    grad = tr.backward(g)
    want_out, want_grad = ref.gradient(th.astype(np.float64), g.astype(np.float64))
    np.testing.assert_allclose(out.reshape(-1, 3), want_out, rtol=1e-4, atol=1e-5)
    scale = np.abs(want_grad).max()
    # float32 forward sums against float64: 1e-4 of the largest component
    np.testing.assert_allclose(grad, want_grad, rtol=0, atol=1e-4 * scale)
    assert np.count_nonzero(want_grad) > 0


def test_gradient_is_central_differences(small):
    scene, tr = small
    rng = np.random.default_rng(2)
    th = tr.theta0()
    g = np.ones((tr.ih, tr.iw, 3), np.float32) + rng.uniform(0, 1, (tr.ih, tr.iw, 3)).astype(np.float32)
    tr.forward(th)
    grad = tr.backward(g)
    M = tr.n_materials
    h = 1e-3
    # the ground's albedo, a box's, the sky's three colours, the sun
    for j in [0, 1, 2, 3 * 3 + 1, 3 * M, 3 * M + 4, 3 * M + 8, 3 * M + 9]:
        tp, tm = th.copy(), th.copy()
        tp[j] += h
        tm[j] -= h
        fd = ((tr.forward(tp).astype(np.float64) * g).sum() - (tr.forward(tm).astype(np.float64) * g).sum()) / (2 * h)
        assert abs(fd - grad[j]) <= 2e-3 * max(abs(grad[j]), 1e-3 * np.abs(grad).max()), (j, fd, grad[j])


def test_l2_loss_to_a_perturbed_target(small):
    """The differentiation workload's loss: L2 between the atlas and one baked at theta0 + N(0, 0.05); its
    gradient against the float64 reference's."""
    scene, tr = small
    rng = np.random.default_rng(9)
    th0 = tr.theta0()
    target = tr.forward(th0 + rng.normal(0, 0.05, th0.shape).astype(np.float32)).astype(np.float64)
    y = tr.forward(th0).astype(np.float64)
    grad = tr.backward(2 * (y - target))
    ref = T.TransportRef(_arrays(tr))
    th = th0.astype(np.float64)
    import torch
    t = torch.tensor(th, requires_grad=True)
    loss = ((ref.forward(t) - torch.from_numpy(target.reshape(-1, 3))) ** 2).sum()
    loss.backward()
    want = t.grad.numpy()
    np.testing.assert_allclose(grad, want, rtol=0, atol=1e-4 * np.abs(want).max())


def test_differentiation_workload(gpu):
    """The differentiation workload as stated for the small map: three bounces; the parameters are the 16
    box albedos (the ground's held fixed), one sky colour (zenith = horizon = ground) and the sun's scale;
    the loss is L2 to a target baked at the parameters + N(0, 0.05) (seed 1). The adjoint's gradient is
    checked against the float64 restatement's autograd gradient and against central differences
    (h = 1e-3) of the float64 loss."""
    import torch
    tr = lb.Transport(scenes.small_map(seed=0, bounces=3), gpu)
    assert tr.shape.bounces == 3 and tr.n_materials == 17
    th0 = tr.theta0()
    M = tr.n_materials

    def full(phi):  # the reduced parameters into theta (numpy or torch)
        cat = torch.cat if isinstance(phi, torch.Tensor) else np.concatenate
        head = th0[:3] if not isinstance(phi, torch.Tensor) else torch.tensor(th0[:3], dtype=phi.dtype)
        sky = phi[48:51]
        return cat([head, phi[:48], sky, sky, sky, phi[51:52]])

    phi0 = np.concatenate([th0[3:3 * M], th0[3 * M:3 * M + 3], th0[-1:]]).astype(np.float64)
    target_phi = phi0 + np.random.default_rng(1).normal(0.0, 0.05, phi0.shape)
    target = tr.forward(full(target_phi).astype(np.float32)).astype(np.float64)
    y = tr.forward(full(phi0).astype(np.float32)).astype(np.float64)
    g_full = tr.backward(2.0 * (y - target))
    g_phi = np.concatenate([g_full[3:3 * M], g_full[3 * M:3 * M + 3] + g_full[3 * M + 3:3 * M + 6] +
                            g_full[3 * M + 6:3 * M + 9], g_full[-1:]])
    ref = T.TransportRef(_arrays(tr))
    tgt = torch.from_numpy(target.reshape(-1, 3))

    def loss64(phi):
        return ((ref.forward(full(phi)) - tgt) ** 2).sum()

    p = torch.tensor(phi0, requires_grad=True)
    loss64(p).backward()
    want = p.grad.numpy()
    scale = np.abs(want).max()
    np.testing.assert_allclose(g_phi, want, rtol=0, atol=1e-4 * scale)
    h = 1e-3
    for j in [0, 1, 2, 20, 47, 48, 49, 50, 51]:
        e = np.zeros_like(phi0)
        e[j] = h
        with torch.no_grad():
            fd = (loss64(torch.from_numpy(phi0 + e)) - loss64(torch.from_numpy(phi0 - e))).item() / (2 * h)
        assert abs(fd - want[j]) <= 1e-5 * scale, (j, fd, want[j])
        assert abs(fd - g_phi[j]) <= 1e-4 * scale, (j, fd, g_phi[j])
    tr.close()


def test_checkpoints_recompute_the_same_bits(small, gpu):
    scene, tr = small
    assert tr.shape.bounces == 2 and tr.shape.checkpoints == 2
    one = lb.Transport(scene, gpu, max_checkpoints=1)
    assert one.shape.checkpoints == 1 and one.shape.checkpoint_bytes * 2 == tr.shape.checkpoint_bytes
    rng = np.random.default_rng(4)
    th = tr.theta0() * np.float32(1.05)
    g = rng.normal(size=(tr.ih, tr.iw, 3)).astype(np.float32)
    a_out, b_out = tr.forward(th), one.forward(th)
    np.testing.assert_array_equal(a_out.view(np.uint32), b_out.view(np.uint32))
    a, b = tr.backward(g), one.backward(g)
    np.testing.assert_array_equal(a.view(np.uint32), b.view(np.uint32))
    # and again: the same bits
    np.testing.assert_array_equal(tr.backward(g).view(np.uint32), a.view(np.uint32))
    one.close()


def test_torch_op(small):
    import torch
    scene, tr = small
    th = torch.tensor(tr.theta0(), device="cuda", requires_grad=True)
    out = lb.transport(th, tr)
    g = torch.rand_like(out)
    (out * g).sum().backward()
    want = tr.backward(g.cpu().numpy())
    np.testing.assert_array_equal(th.grad.cpu().numpy().view(np.uint32), want.view(np.uint32))


def test_backward_needs_a_forward(gpu):
    tr = lb.Transport(scenes.small_map(seed=3), gpu)
    with pytest.raises(lb.LightbakerError, match="no forward"):
        tr.backward(np.zeros((tr.ih, tr.iw, 3), np.float32))
    tr.close()
