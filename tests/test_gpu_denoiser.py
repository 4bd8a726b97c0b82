"""The learned denoiser on the GPU: gradients of the tensor-core forward and
backward kernels against the CPU FP64 oracle, and what the trained network
gains over plain Monte Carlo at equal histories."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _case(B, S, seed):
    rng = np.random.default_rng(seed)
    z, y, x = np.meshgrid(*(np.linspace(-1, 1, S),) * 3, indexing="ij")
    base = -2.0 * (x ** 2 + y ** 2 + z ** 2)
    xlog = np.stack([base + 0.3 * rng.normal(size=(S, S, S)) for _ in range(B)]).astype(np.float32)
    mat = rng.integers(0, 4, size=(B, S, S, S)).astype(np.uint8)
    dens = np.array([0.0012, 1.0, 1.85, 11.35], dtype=np.float32)[mat]
    target = (np.stack([base] * B) + 0.05).astype(np.float32)
    weight = np.where(mat > 0, 1.0, 0.1).astype(np.float32)
    return xlog, dens, mat, target, weight


def _run_gpu_step(B, S, seed):
    import torch
    from chatcarlo_b200 import denoiser as DN
    xlog, dens, mat, target, weight = _case(B, S, seed)
    params = DN.init_params(5)
    ho, _, _, _ = DN.param_layout()["head"]
    params[ho:ho + 17] = np.random.default_rng(6).normal(0, 0.3, 17).astype(np.float32)
    for L in DN.LAYERS:                      # small positive biases keep most units active
        _, _, bo, bn = DN.param_layout()[L.name]
        params[bo:bo + bn] = 0.05
    model = DN.UNet3D(params=params)
    model.set_input(xlog, dens, mat, B, S)
    tgt = torch.from_numpy(target.reshape(-1)).cuda()
    wgt = torch.from_numpy(weight.reshape(-1)).cuda()
    model.forward()
    model.backward(tgt, wgt, 1.0 / float(weight.sum()))
    torch.cuda.synchronize()
    model.check_status()
    return model, params, (xlog, dens, mat, target, weight)


def _rel(a, b):
    a, b = np.asarray(a, dtype=np.float64).ravel(), np.asarray(b, dtype=np.float64).ravel()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def test_every_layer_matches_the_cpu_oracle_on_the_gpus_own_tensors():
    """Layer by layer: the oracle recomputes each convolution's forward
    output, weight and bias gradients and data gradient (FP64) from the
    tensors the GPU fed that layer, and the GPU results must agree to the
    FP32-accumulation / BF16-output level.  Isolating the layers keeps a
    ReLU mask flip in one layer from propagating into the comparison."""
    import unet_oracle as UO
    from chatcarlo_b200 import denoiser as DN
    B, S = 2, 16
    model, params, (xlog, dens, mat, target, weight) = _run_gpu_step(B, S, 3)
    lay = DN.param_layout()
    Ls = {L.name: L for L in DN.LAYERS}
    P = params.astype(np.float64)
    g_gpu = model.g.cpu().numpy().astype(np.float64)

    def t(buf, level, c):
        s = S >> level
        return buf.float().cpu().numpy().astype(np.float64).reshape(B, s, s, s, c)

    # head: output and its gradient from the GPU's last activation
    ho = lay["head"][0]
    out_ref = xlog.astype(np.float64) + t(model.a["d0"], 0, 16) @ P[ho:ho + 16] + P[ho + 16]
    out_gpu = model.out.cpu().numpy().astype(np.float64).reshape(out_ref.shape)
    assert _rel(out_gpu, out_ref) < 1e-5
    dout = 2.0 * weight * (out_gpu - target) / float(weight.sum())
    dz_head = UO.bf16(dout[..., None] * P[ho:ho + 16] * (t(model.a["d0"], 0, 16) > 0))
    assert _rel(t(model.gb["dz_d0"], 0, 16), dz_head) < 3e-3
    A = {k: t(model.a[k], lv, c) for k, lv, c in
         [("x0", 0, 16), ("p0", 1, 16), ("p1", 2, 32), ("p2", 3, 64)] +
         [(L.name, L.level, L.cout) for L in DN.LAYERS]}
    Z = {L.name: t(model.gb["dz_" + L.name], L.level, L.cout) for L in DN.LAYERS}
    inputs = {"e0a": ("x0", None), "e0": ("e0a", None), "e1a": ("p0", None), "e1": ("e1a", None),
              "e2a": ("p1", None), "e2": ("e2a", None), "b3a": ("p2", None), "b3": ("b3a", None),
              "d2a": ("e2", "b3"), "d2": ("d2a", None), "d1a": ("e1", "d2"), "d1": ("d1a", None),
              "d0a": ("e0", "d1"), "d0": ("d0a", None)}
    for name, (ka, kb) in inputs.items():
        L = Ls[name]
        o, n, bo, bn = lay[name]
        W = UO.bf16(P[o:o + n]).reshape(27, L.cout, L.cin)
        x = A[ka] if kb is None else np.concatenate([A[ka], UO.up(A[kb])], axis=-1)
        y = UO.bf16(np.maximum(UO.conv3d(x, W) + P[bo:bo + bn], 0.0))
        assert _rel(A[name], y) < 3e-3, (name, "forward", _rel(A[name], y))
        assert _rel(g_gpu[o:o + n], UO.conv3d_wgrad(x, Z[name]).ravel()) < 1e-4, (name, "weight grad")
        assert _rel(g_gpu[bo:bo + bn], Z[name].reshape(-1, L.cout).sum(axis=0)) < 1e-4, (name, "bias grad")
    # data gradients and the pooling / upsampling backward steps
    def dgrad(name):
        L = Ls[name]
        o, n, _, _ = lay[name]
        return UO.conv3d_dgrad(Z[name], UO.bf16(P[o:o + n]).reshape(27, L.cout, L.cin), L.cin)
    for name, below in (("d0", "d0a"), ("d1", "d1a"), ("d2", "d2a"), ("b3", "b3a"), ("e2", "e2a"),
                        ("e1", "e1a"), ("e0", "e0a")):
        ref = UO.bf16(dgrad(name) * (A[below] > 0))
        assert _rel(Z[below], ref) < 3e-3, (name, "data grad", _rel(Z[below], ref))
    for name, coarse, g_key, skip in (("d0a", "d1", "g_up1", "e0"), ("d1a", "d2", "g_up2", "e1"),
                                      ("d2a", "b3", "g_up3", "e2")):
        L = Ls[name]
        gx = dgrad(name)
        g_up = t(model.gb[g_key], L.level, L.cb)
        assert _rel(g_up, UO.bf16(gx[..., L.ca:])) < 3e-3, (name, "upsampled-input grad")
        assert _rel(Z[coarse], UO.bf16(UO.up_sum(g_up) * (A[coarse] > 0))) < 3e-3, (coarse, "up reduce")
    for name, skip_src, g_key, skip in (("e1a", "d0a", "g_p0", "e0"), ("e2a", "d1a", "g_p1", "e1"),
                                        ("b3a", "d2a", "g_p2", "e2")):
        L = Ls[name]
        g_p = t(model.gb[g_key], L.level, L.cin)
        assert _rel(g_p, UO.bf16(dgrad(name))) < 3e-3, (name, "pooled-input grad")
        part = UO.bf16(dgrad(skip_src)[..., :Ls[skip_src].ca] * (A[skip] > 0))
        ref = UO.bf16(part + 0.125 * UO.up(g_p) * (A[skip] > 0))
        assert _rel(Z[skip], ref) < 3e-3, (skip, "skip grad")


def test_gradients_end_to_end_against_the_cpu_oracle():
    """The whole step against the oracle run on its own (FP64 sums, BF16
    storage): the loss agrees to 1e-4; the gradients differ where a
    pre-activation within a BF16 rounding of zero flips its ReLU on one side
    only, so the bound is a few percent and the directions must agree."""
    import unet_oracle as UO
    from chatcarlo_b200 import denoiser as DN
    model, params, (xlog, dens, mat, target, weight) = _run_gpu_step(2, 16, 3)
    g_gpu = model.g.cpu().numpy().astype(np.float64)
    loss_ref, g_ref, _ = UO.loss_and_grads(params, xlog.astype(np.float64), dens, mat, target.astype(np.float64),
                                           weight.astype(np.float64))
    assert abs(model.loss() - loss_ref) < 1e-4 * abs(loss_ref)
    for name, (o, n, bo, bn) in DN.param_layout().items():
        a, b = g_gpu[o:o + n], g_ref[o:o + n]
        assert _rel(a, b) < 0.1, (name, _rel(a, b))
        assert float(a @ b) / (np.linalg.norm(a) * np.linalg.norm(b)) > 0.995, name
    assert _rel(g_gpu, g_ref) < 0.03


def test_trained_denoiser_beats_plain_monte_carlo_at_equal_histories():
    """Small-scale training on the engine's own Monte Carlo (32^3 phantoms,
    1e5-history inputs, 1e7-history targets); on held-out phantoms the
    denoised 1e5-history maps must be clearly closer to a 1e8-history
    reference than the plain 1e5-history maps."""
    from chatcarlo_b200 import denoise_run as R
    from chatcarlo_b200 import denoiser as DN
    from chatcarlo_b200 import phantoms as PH
    from chatcarlo_b200.transport import default_engine
    eng = default_engine()
    S = 32
    tr_sc, tr_gr = PH.phantoms(48, 11, S, 0.5)
    te_sc, te_gr = PH.phantoms(6, 12, S, 0.5)
    tr = [PH.voxel_maps(s, g) for s, g in zip(tr_sc, tr_gr)]
    te = [PH.voxel_maps(s, g) for s, g in zip(te_sc, te_gr)]
    runs = [R.mc_maps(tr_sc, tr_gr, n, 1 + n % 7, eng, stats_slots=16) for n in (100_000, 400_000)]
    k_tg, _, _ = R.mc_maps(tr_sc, tr_gr, 10_000_000, 2, eng)
    data = R.Dataset([r[0] for r in runs], k_tg, np.stack([m for m, _ in tr]), np.stack([d for _, d in tr]),
                     rel=[r[1] for r in runs])
    model = DN.UNet3D(seed=1)
    losses, _ = R.train(model, data, steps=400, batch=4, lr=2e-3, seed=1)
    assert losses[-1][1] < 0.5 * losses[0][1], losses
    te_mat = np.stack([m for m, _ in te])
    k_ref, _, _ = R.mc_maps(te_sc, te_gr, 100_000_000, 3, eng)
    k_lo, r_lo, _ = R.mc_maps(te_sc, te_gr, 100_000, 4, eng, stats_slots=16)
    k_dn, _ = R.denoise(model, R.Dataset(k_lo, None, te_mat, np.stack([d for _, d in te]), rel=r_lo))
    inside = R.inside_mask(te_mat)
    e_plain = R.median_rel_error(k_lo, k_ref, inside)
    e_dn = R.median_rel_error(k_dn, k_ref, inside)
    assert e_dn < 0.7 * e_plain, (e_dn, e_plain)


def test_shipped_network_denoises_held_out_phantoms():
    """The pretrained network shipped with the package, on phantoms it was
    not trained on: at 1e6 histories its median voxel-kerma error against a
    2e8-history reference must be under half that of plain Monte Carlo."""
    from chatcarlo_b200 import denoise_run as R
    from chatcarlo_b200 import denoiser as DN
    from chatcarlo_b200 import phantoms as PH
    from chatcarlo_b200.transport import default_engine
    eng = default_engine()
    sc, gr = PH.phantoms(4, 2002, 64, 0.5)
    maps = [PH.voxel_maps(a, b) for a, b in zip(sc, gr)]
    mat = np.stack([m for m, _ in maps])
    den = np.stack([d for _, d in maps])
    k_ref, _, _ = R.mc_maps(sc, gr, 200_000_000, 5, eng)
    k_n, rel_n, _ = R.mc_maps(sc, gr, 1_000_000, 6, eng, stats_slots=16)
    k_dn = DN.denoise_kerma(k_n, rel_n, mat, den)
    inside = R.inside_mask(mat)
    e_plain = R.median_rel_error(k_n, k_ref, inside)
    e_dn = R.median_rel_error(k_dn, k_ref, inside)
    assert e_dn < 0.5 * e_plain, (e_dn, e_plain)


def test_shipped_ct_network_denoises_the_ct_configuration():
    """The CT network shipped with the package on the CT configuration's own
    phantom (not among its training phantoms), 1 mm voxels: at 3e6
    histories its median voxel-kerma error inside the phantom against a
    1e9-history reference must be under a quarter of plain Monte Carlo's."""
    from chatcarlo_b200 import ct_denoise as CD
    from chatcarlo_b200 import phantoms as PH
    from chatcarlo_b200 import workloads as W
    from chatcarlo_b200.transport import default_engine
    eng = default_engine()
    grid = W.make_grid(W.CT_GRID, track_uncertainty=True, pinned=True)
    sc = W.ct()
    mat, dens = PH.voxel_maps(sc, W.CT_GRID, CD.CT_MATERIALS)
    k_ref, _, _ = CD.scan(sc, 1_000_000_000, 7, eng, grid, batches=20)
    k_n, rel_n, _ = CD.scan(sc, 3_000_000, 11, eng, grid)
    k_dn = CD.denoise_ct_kerma(k_n, rel_n, mat, dens)
    sel = (mat != 0) & (k_ref > 0)
    err = lambda k: float(np.median(np.abs(k[sel] - k_ref[sel]) / k_ref[sel]))  # noqa: E731
    e_plain, e_dn = err(k_n), err(k_dn)
    assert e_dn < 0.25 * e_plain, (e_dn, e_plain)


def test_whole_volume_pass_equals_the_oracle_on_a_non_cubic_volume():
    """The network on a non-cubic volume (16 x 32 x 24 voxels, one pass): its
    first layer's output against the denoiser's oracle, and a finite
    prediction of the right shape."""
    import unet_oracle as UO
    from chatcarlo_b200 import denoiser as DN
    params, _ = DN.load_params()
    model = DN.UNet3D(params=params)
    rng = np.random.default_rng(4)
    shape = (16, 32, 24)
    xl = rng.normal(size=(1, *shape)).astype(np.float32)
    mt = rng.integers(0, 4, size=(1, *shape)).astype(np.uint8)
    dn = np.array([0.0012, 1.0, 1.85, 11.35], dtype=np.float32)[mt]
    un = np.full((1, *shape), 0.2, np.float32)
    model.set_input(xl, dn, mt, 1, shape, unc=un)
    out = model.predict().cpu().numpy().reshape(shape)
    model.check_status()
    o, nw, bo, bn = DN.param_layout()["e0a"]
    x0 = UO.bf16(UO.make_input(xl.astype(np.float64), dn, mt, un))
    y = UO.bf16(np.maximum(UO.conv3d(x0, UO.bf16(params[o:o + nw]).reshape(27, 16, 16)) + params[bo:bo + bn], 0))
    got = model.a["e0a"].float().cpu().numpy().reshape(y.shape)
    assert np.all(np.isfinite(out))
    assert float(np.linalg.norm(got - y) / np.linalg.norm(y)) < 3e-3


def test_layer_times_cover_every_convolution():
    """ct_denoise.layer_times: one entry per convolution of the network,
    positive device times and FLOP rates, and a timed whole prediction."""
    from chatcarlo_b200 import ct_denoise as CD
    from chatcarlo_b200 import denoiser as DN
    r = CD.layer_times((64, 48, 16), repeats=2)
    assert [x["layer"] for x in r["layers"]] == [L.name for L in DN.LAYERS]
    assert all(x["ms"] > 0 and x["tflops"] > 0 for x in r["layers"])
    assert r["predict_ms"] > 0 and r["conv_ms"] > 0
