"""Tensor-core kernels of the denoiser vs a plain PyTorch FP32 reference of the
same operation on the same BF16 values (torch is only the reference here)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def U():
    from chatcarlo_b200 import _unet_native as U
    U.lib()
    U.status(reset=True)
    return U


def _ptr(t):
    return t.data_ptr()


def _bf(shape, gen, scale=1.0):
    return (torch.randn(*shape, generator=gen) * scale).to(torch.bfloat16).cuda()


@pytest.mark.parametrize("n,a_mn,b_mn", [(16, 0, 0), (64, 0, 0), (256, 0, 0), (48, 1, 1), (128, 1, 1),
                                         (32, 0, 1)])
def test_gemm_descriptors(U, n, a_mn, b_mn):
    gen = torch.Generator().manual_seed(n + 7 * a_mn)
    m, k = 256, 192
    a = _bf((m, k), gen)
    b = _bf((n, k), gen)
    d = torch.empty(m, n, dtype=torch.float32, device="cuda")
    aa = a.t().contiguous() if a_mn else a
    bb = b.t().contiguous() if b_mn else b
    U.check(U.lib().ccu_gemm_test(_ptr(aa), _ptr(bb), _ptr(d), m, n, k, a_mn, b_mn, None))
    torch.cuda.synchronize()
    assert U.status() == 0
    ref = a.float() @ b.float().t()
    torch.testing.assert_close(d, ref, rtol=1e-4, atol=1e-3)


def _torch_w(w_mine, cout, cin):
    return w_mine.float().reshape(3, 3, 3, cout, cin).permute(3, 4, 0, 1, 2).contiguous()


def _to_ncdhw(x):
    return x.float().permute(0, 4, 1, 2, 3).contiguous()


def _up(x):
    return x.repeat_interleave(2, 2).repeat_interleave(2, 3).repeat_interleave(2, 4)


@pytest.mark.parametrize("ca,cb,cout,dims", [(16, 0, 16, (2, 6, 8, 10)), (16, 32, 48, (1, 8, 8, 8)),
                                             (64, 128, 64, (1, 4, 6, 8)), (32, 64, 96, (1, 6, 4, 4)),
                                             (128, 0, 128, (1, 5, 3, 7)), (16, 0, 192, (1, 4, 4, 4)),
                                             # shapes of the shared-memory halo kernel (H % 16, W % 8)
                                             (16, 0, 16, (2, 3, 16, 8)), (16, 32, 48, (1, 4, 32, 16)),
                                             (32, 0, 32, (1, 2, 16, 24)), (16, 32, 16, (2, 2, 16, 16)),
                                             # plane-stationary kernel: 2 and 3 channel passes (FP32
                                             # partial sums), split outputs with fine and coarse
                                             # channels in one pass, edge tiles
                                             (32, 64, 32, (1, 6, 8, 8)), (64, 128, 32, (1, 4, 6, 8)),
                                             (16, 16, 32, (2, 6, 12, 10)), (16, 0, 16, (1, 1, 19, 9))])
def test_conv3d_forward(U, ca, cb, cout, dims):
    gen = torch.Generator().manual_seed(ca * 1000 + cb * 10 + cout)
    B, D, H, W = dims
    a = _bf((B, D, H, W, ca), gen)
    b = _bf((B, D // 2, H // 2, W // 2, cb), gen) if cb else None
    w32 = (torch.randn(27 * cout * (ca + cb), generator=gen) * 0.1).cuda()
    w = torch.empty(U.lib().ccu_packed_weight_elems(cout, ca + cb), dtype=torch.bfloat16, device="cuda")
    U.check(U.lib().ccu_pack_weights(_ptr(w32), cout, ca + cb, _ptr(w), None, None))
    bias = (torch.randn(cout, generator=gen) * 0.1).cuda()
    split = ca if cb and cout == ca + cb else cout
    out0 = torch.empty(B, D, H, W, split, dtype=torch.bfloat16, device="cuda")
    out1 = torch.empty(B, D, H, W, cout - split, dtype=torch.bfloat16, device="cuda") if split < cout else None
    U.check(U.lib().ccu_conv3d(_ptr(a), ca, _ptr(b) if b is not None else None, cb, B, D, H, W, _ptr(w),
                               _ptr(bias), cout, 1, _ptr(out0), split, None,
                               _ptr(out1) if out1 is not None else None, None))
    torch.cuda.synchronize()
    assert U.status() == 0
    x = _to_ncdhw(a)
    if cb:
        x = torch.cat([x, _up(_to_ncdhw(b))], dim=1)
    ref = torch.relu(torch.nn.functional.conv3d(x, _torch_w(w32.to(torch.bfloat16), cout, ca + cb), bias, padding=1))
    ref = ref.permute(0, 2, 3, 4, 1)
    got = out0.float() if out1 is None else torch.cat([out0.float(), out1.float()], dim=-1)
    torch.testing.assert_close(got, ref, rtol=1.6e-2, atol=1e-2)


@pytest.mark.parametrize("ca,cb,cout,dims", [(16, 0, 16, (2, 6, 8, 10)), (16, 32, 16, (1, 8, 8, 8)),
                                             (64, 128, 64, (1, 4, 6, 8)), (64, 0, 128, (1, 5, 3, 7)),
                                             (32, 0, 32, (3, 4, 4, 4)),
                                             # data gradients through the halo kernel
                                             (16, 0, 16, (1, 4, 16, 8)), (16, 32, 16, (2, 2, 16, 16))])
def test_conv3d_weight_and_data_gradients(U, ca, cb, cout, dims):
    """Weight gradient (tcgen05, MN-major operands) and the data gradient
    (the forward kernel on flipped, transposed weights with the ReLU mask
    of the input in its epilogue) vs torch autograd."""
    gen = torch.Generator().manual_seed(ca + 3 * cb + 5 * cout)
    B, D, H, W = dims
    cin = ca + cb
    a = torch.relu(_bf((B, D, H, W, ca), gen).float()).to(torch.bfloat16)
    b = torch.relu(_bf((B, D // 2, H // 2, W // 2, cb), gen).float()).to(torch.bfloat16) if cb else None
    dz = _bf((B, D, H, W, cout), gen)
    w32 = (torch.randn(27 * cout * cin, generator=gen) * 0.1).cuda()
    wbf = torch.empty(U.lib().ccu_packed_weight_elems(cout, cin), dtype=torch.bfloat16, device="cuda")
    wt = torch.empty(U.lib().ccu_packed_weight_elems(cin, cout), dtype=torch.bfloat16, device="cuda")
    U.check(U.lib().ccu_pack_weights(_ptr(w32), cout, cin, _ptr(wbf), _ptr(wt), None))
    dw = torch.zeros(27 * cout * cin, dtype=torch.float32, device="cuda")
    U.check(U.lib().ccu_conv3d_wgrad(_ptr(a), ca, _ptr(b) if b is not None else None, cb, B, D, H, W, _ptr(dz),
                                     cout, _ptr(dw), 7, None))
    # data gradient wrt the concatenated input, masked by the input's ReLU
    # (the skip part) and written unmasked for the upsampled part
    g0 = torch.empty(B, D, H, W, ca, dtype=torch.bfloat16, device="cuda")
    g1 = torch.empty(B, D, H, W, cb, dtype=torch.bfloat16, device="cuda") if cb else None
    U.check(U.lib().ccu_conv3d(_ptr(dz), cout, None, 0, B, D, H, W, _ptr(wt), None, cin, 0, _ptr(g0), ca,
                               _ptr(a), _ptr(g1) if g1 is not None else None, None))
    torch.cuda.synchronize()
    assert U.status() == 0

    x = _to_ncdhw(a).requires_grad_(True)
    xb = _to_ncdhw(b).requires_grad_(True) if cb else None
    xin = torch.cat([x, _up(xb)], dim=1) if cb else x
    wt_ref = _torch_w(w32.to(torch.bfloat16), cout, cin).requires_grad_(True)
    y = torch.nn.functional.conv3d(xin, wt_ref, None, padding=1)
    y.backward(_to_ncdhw(dz))
    dw_ref = wt_ref.grad.permute(2, 3, 4, 0, 1).reshape(-1)
    torch.testing.assert_close(dw, dw_ref, rtol=2e-3, atol=2e-3 * float(dw_ref.abs().max()))
    ga = (x.grad * (x > 0)).permute(0, 2, 3, 4, 1)
    torch.testing.assert_close(g0.float(), ga, rtol=1.6e-2, atol=1e-2)
    if cb:
        # the upsampled part, before its 2x2x2 reduction
        xin_up = _up(xb).detach().requires_grad_(True)
        y2 = torch.nn.functional.conv3d(torch.cat([x.detach(), xin_up], dim=1), wt_ref.detach(), None, padding=1)
        y2.backward(_to_ncdhw(dz))
        torch.testing.assert_close(g1.float(), xin_up.grad.permute(0, 2, 3, 4, 1), rtol=1.6e-2, atol=1e-2)


def test_pool_upsample_bias_helpers(U):
    gen = torch.Generator().manual_seed(5)
    B, D, H, W, c = 2, 4, 6, 8, 32
    x = torch.relu(_bf((B, D, H, W, c), gen).float()).to(torch.bfloat16)
    y = torch.empty(B, D // 2, H // 2, W // 2, c, dtype=torch.bfloat16, device="cuda")
    U.check(U.lib().ccu_avgpool(_ptr(x), B, D, H, W, c, _ptr(y), None))
    ref = torch.nn.functional.avg_pool3d(_to_ncdhw(x), 2).permute(0, 2, 3, 4, 1)
    gy = _bf((B, D // 2, H // 2, W // 2, c), gen)
    dz = torch.zeros(B, D, H, W, c, dtype=torch.bfloat16, device="cuda")
    U.check(U.lib().ccu_pool_backward(_ptr(gy), _ptr(x), B, D, H, W, c, _ptr(dz), None))
    gfull = _bf((B, D, H, W, c), gen)
    coarse = torch.relu(_bf((B, D // 2, H // 2, W // 2, c), gen).float()).to(torch.bfloat16)
    dzc = torch.empty_like(coarse)
    U.check(U.lib().ccu_up_reduce(_ptr(gfull), _ptr(coarse), B, D, H, W, c, _ptr(dzc), None))
    db = torch.zeros(c, dtype=torch.float32, device="cuda")
    U.check(U.lib().ccu_bias_grad(_ptr(gfull), B * D * H * W, c, _ptr(db), None))
    torch.cuda.synchronize()
    torch.testing.assert_close(y.float(), ref, rtol=1.6e-2, atol=1e-2)
    up = gy.float().repeat_interleave(2, 1).repeat_interleave(2, 2).repeat_interleave(2, 3) / 8
    torch.testing.assert_close(dz.float(), up * (x.float() > 0), rtol=1.6e-2, atol=1e-2)
    red = gfull.float().reshape(B, D // 2, 2, H // 2, 2, W // 2, 2, c).sum(dim=(2, 4, 6))
    torch.testing.assert_close(dzc.float(), red * (coarse.float() > 0), rtol=1.6e-2, atol=2e-2)
    torch.testing.assert_close(db, gfull.float().sum(dim=(0, 1, 2, 3)), rtol=1e-4, atol=1e-2)


@pytest.mark.parametrize("ca,cb,cout,dims", [(16, 0, 16, (2, 5, 12, 64)),    # x runs of 64, one y row per stage
                                              (32, 0, 32, (1, 3, 10, 24)),    # 8 x 8 stages, a partial y block
                                              (64, 0, 64, (2, 4, 6, 16)),     # 16 x 4 stages
                                              (16, 0, 128, (1, 3, 5, 40)),    # 432 rows: a partial M tile
                                              (128, 0, 64, (1, 2, 4, 32)),    # 27 M tiles
                                              (16, 0, 16, (1, 4, 16, 8)),
                                              # concatenated inputs: the upsampled part from its copy
                                              (16, 32, 16, (1, 4, 8, 16)), (32, 64, 32, (2, 2, 4, 8)),
                                              (64, 128, 64, (1, 2, 6, 8))])
def test_weight_gradient_tile_loads(U, ca, cb, cout, dims):
    """The weight gradient from tensor-memory-accelerator tile loads (the
    default for w % 8 == 0 and 16, 32 or 64k channels per input part)
    against torch autograd and against the gathering kernel (wgrad path 1),
    with more splits than some volumes have stages."""
    gen = torch.Generator().manual_seed(11 * ca + 3 * cb + cout + dims[3])
    B, D, H, W = dims
    cin = ca + cb
    a = torch.relu(_bf((B, D, H, W, ca), gen).float()).to(torch.bfloat16)
    b = torch.relu(_bf((B, D // 2, H // 2, W // 2, cb), gen).float()).to(torch.bfloat16) if cb else None
    dz = _bf((B, D, H, W, cout), gen)
    got = []
    try:
        for path, slices in ((0, 7), (0, 1000), (1, 7)):
            U.check(U.lib().ccu_set_wgrad_path(path))
            dw = torch.zeros(27 * cout * cin, dtype=torch.float32, device="cuda")
            U.check(U.lib().ccu_conv3d_wgrad(_ptr(a), ca, _ptr(b) if b is not None else None, cb, B, D, H, W,
                                             _ptr(dz), cout, _ptr(dw), slices, None))
            got.append(dw)
    finally:
        U.check(U.lib().ccu_set_wgrad_path(0))
    torch.cuda.synchronize()
    assert U.status() == 0
    x = _to_ncdhw(a)
    if cb:
        x = torch.cat([x, _up(_to_ncdhw(b))], dim=1)
    wt_ref = torch.zeros(cout, cin, 3, 3, 3, device="cuda", requires_grad=True)
    y = torch.nn.functional.conv3d(x, wt_ref, None, padding=1)
    y.backward(_to_ncdhw(dz))
    ref = wt_ref.grad.permute(2, 3, 4, 0, 1).reshape(-1)
    tol = 2e-3 * float(ref.abs().max())
    for dw in got:
        torch.testing.assert_close(dw, ref, rtol=2e-3, atol=tol)
    torch.testing.assert_close(got[0], got[2], rtol=1e-4, atol=1e-4 * float(ref.abs().max()))


@pytest.mark.parametrize("B,D,H,W,ca,cb,cout", [(2, 4, 32, 16, 16, 32, 48), (1, 37, 16, 8, 16, 0, 16),
                                                (3, 18, 32, 24, 16, 0, 32), (1, 5, 16, 16, 32, 0, 16),
                                                # edge tiles of the streaming kernel (h % 16, w % 8 != 0)
                                                (2, 6, 10, 12, 16, 32, 32), (1, 20, 38, 19, 16, 0, 16)])
def test_halo_and_gathering_kernels_agree(U, B, D, H, W, ca, cb, cout):
    """The forward kernels on the same inputs: the default path 0 (the
    plane-stationary kernel for 16 and 32 output channels), the gathering
    kernel (path 1), the one-tile halo kernel (path 2), the streaming kernel
    with warp roles (path 3) and the streaming halo kernel (path 4; depths
    that are not a multiple of its 16-plane segment, several volumes); paths
    3 and 4 issue the same MMAs in the same order and agree bit for bit."""
    gen = torch.Generator().manual_seed(77 + D)
    a = _bf((B, D, H, W, ca), gen)
    b = _bf((B, D // 2, H // 2, W // 2, cb), gen) if cb else None
    w32 = (torch.randn(27 * cout * (ca + cb), generator=gen) * 0.1).cuda()
    w = torch.empty(U.lib().ccu_packed_weight_elems(cout, ca + cb), dtype=torch.bfloat16, device="cuda")
    U.check(U.lib().ccu_pack_weights(_ptr(w32), cout, ca + cb, _ptr(w), None, None))
    outs = []
    try:
        for path in (0, 1, 2, 3, 4):
            U.check(U.lib().ccu_set_conv_path(path))
            o = torch.empty(B, D, H, W, cout, dtype=torch.bfloat16, device="cuda")
            U.check(U.lib().ccu_conv3d(_ptr(a), ca, _ptr(b) if b is not None else None, cb, B, D, H, W, _ptr(w),
                                       None, cout, 0, _ptr(o), cout, None, None, None))
            outs.append(o.float())
    finally:
        U.check(U.lib().ccu_set_conv_path(0))
    torch.cuda.synchronize()
    assert U.status() == 0
    for k in (0, 2, 4):
        torch.testing.assert_close(outs[k], outs[1], rtol=1.6e-2, atol=1e-2)
    torch.testing.assert_close(outs[3], outs[4], rtol=0, atol=0)
    x = _to_ncdhw(a)
    if cb:
        x = torch.cat([x, _up(_to_ncdhw(b))], dim=1)
    ref = torch.nn.functional.conv3d(x, _torch_w(w32.to(torch.bfloat16), cout, ca + cb), padding=1)
    for k in (0, 4):
        torch.testing.assert_close(outs[k], ref.permute(0, 2, 3, 4, 1), rtol=1.6e-2, atol=1e-2)


@pytest.mark.parametrize("B,D,H,W,ca,cb,cout", [(1, 37, 16, 8, 16, 0, 16), (2, 6, 10, 12, 16, 32, 32),
                                                (1, 3, 40, 24, 16, 0, 48), (3, 1, 16, 16, 32, 0, 16)])
def test_warp_role_kernel_ring_depths(U, B, D, H, W, ca, cb, cout):
    """Path 3 with every ring depth that fits the layer, bit for bit equal to
    path 4 (the same MMAs in the same order); a ring that does not fit the
    layer's shared memory is an error, not a silent fallback."""
    gen = torch.Generator().manual_seed(5 + D + cout)
    a = _bf((B, D, H, W, ca), gen)
    b = _bf((B, max(D // 2, 1), H // 2, W // 2, cb), gen) if cb else None
    cin = ca + cb
    w32 = (torch.randn(27 * cout * cin, generator=gen) * 0.1).cuda()
    w = torch.empty(U.lib().ccu_packed_weight_elems(cout, cin), dtype=torch.bfloat16, device="cuda")
    U.check(U.lib().ccu_pack_weights(_ptr(w32), cout, cin, _ptr(w), None, None))

    def conv():
        o = torch.empty(B, D, H, W, cout, dtype=torch.bfloat16, device="cuda")
        rc = U.lib().ccu_conv3d(_ptr(a), ca, _ptr(b) if b is not None else None, cb, B, D, H, W, _ptr(w), None,
                                cout, 0, _ptr(o), cout, None, None, None)
        return rc, o

    slot, wbytes = cin // 8 * 180 * 16, -(-27 * cin // 64) * 8 * cout * 16
    try:
        U.check(U.lib().ccu_set_conv_path(4))
        rc, ref = conv()
        U.check(rc)
        U.check(U.lib().ccu_set_conv_path(3))
        for ring in (0, 4, 5, 7, 12):
            U.check(U.lib().ccu_set_conv_ring(ring))
            rc, o = conv()
            if ring and ring * slot + wbytes > 200 * 1024:
                assert rc != 0
                continue
            U.check(rc)
            torch.cuda.synchronize()
            assert torch.equal(o, ref), ring
    finally:
        U.check(U.lib().ccu_set_conv_ring(0))
        U.check(U.lib().ccu_set_conv_path(0))
    assert U.status() == 0
    assert U.lib().ccu_set_conv_ring(3) != 0


@pytest.mark.parametrize("B,D,H,W,ca,cb,cout", [(1, 37, 16, 8, 16, 0, 16), (2, 6, 10, 12, 16, 32, 16),
                                                (1, 10, 24, 16, 32, 64, 32), (3, 1, 16, 16, 32, 0, 16)])
def test_plane_stationary_issue_groups(U, B, D, H, W, ca, cb, cout):
    """Path 0 with issue groups 1, 2 and 3 (chains of consecutive planes
    interleaved tap by tap; clamped to 1 for 32 output channels): the same
    MMAs per plane in the same order, so every group gives the same bits."""
    gen = torch.Generator().manual_seed(11 + D + cout)
    a = _bf((B, D, H, W, ca), gen)
    b = _bf((B, max(D // 2, 1), H // 2, W // 2, cb), gen) if cb else None
    cin = ca + cb
    w32 = (torch.randn(27 * cout * cin, generator=gen) * 0.1).cuda()
    w = torch.empty(U.lib().ccu_packed_weight_elems(cout, cin), dtype=torch.bfloat16, device="cuda")
    U.check(U.lib().ccu_pack_weights(_ptr(w32), cout, cin, _ptr(w), None, None))
    outs = []
    try:
        for group in (1, 2, 3):
            U.check(U.lib().ccu_set_conv_group(group))
            o = torch.empty(B, D, H, W, cout, dtype=torch.bfloat16, device="cuda")
            U.check(U.lib().ccu_conv3d(_ptr(a), ca, _ptr(b) if b is not None else None, cb, B, D, H, W, _ptr(w),
                                       None, cout, 0, _ptr(o), cout, None, None, None))
            outs.append(o)
    finally:
        U.check(U.lib().ccu_set_conv_group(0))
    torch.cuda.synchronize()
    assert U.status() == 0
    assert torch.equal(outs[0], outs[1]) and torch.equal(outs[0], outs[2])
    x = _to_ncdhw(a)
    if cb:
        x = torch.cat([x, _up(_to_ncdhw(b))], dim=1)
    ref = torch.nn.functional.conv3d(x, _torch_w(w32.to(torch.bfloat16), cout, cin), padding=1)
    torch.testing.assert_close(outs[0].float(), ref.permute(0, 2, 3, 4, 1), rtol=1.6e-2, atol=1e-2)
    assert U.lib().ccu_set_conv_group(4) != 0


@pytest.mark.parametrize("path", [0, 1])
def test_last_convolution_with_the_head_fused(U, path):
    """ccu_conv3d_head equals ccu_conv3d + ccu_head bit for bit: on path 0
    the head runs in the plane-stationary kernel's epilogue (activations
    stored or not), on path 1 it falls back to the two calls."""
    gen = torch.Generator().manual_seed(31 + path)
    B, D, H, W = 2, 6, 20, 12
    a = _bf((B, D, H, W, 16), gen)
    w32 = (torch.randn(27 * 16 * 16, generator=gen) * 0.1).cuda()
    w = torch.empty(U.lib().ccu_packed_weight_elems(16, 16), dtype=torch.bfloat16, device="cuda")
    U.check(U.lib().ccu_pack_weights(_ptr(w32), 16, 16, _ptr(w), None, None))
    bias = (torch.randn(16, generator=gen) * 0.1).cuda()
    head = (torch.randn(17, generator=gen) * 0.3).cuda()
    xlog = torch.randn(B * D * H * W, generator=gen).cuda()
    n = B * D * H * W
    try:
        U.check(U.lib().ccu_set_conv_path(path))
        act_ref = torch.empty(B, D, H, W, 16, dtype=torch.bfloat16, device="cuda")
        out_ref = torch.empty(n, device="cuda")
        U.check(U.lib().ccu_conv3d(_ptr(a), 16, None, 0, B, D, H, W, _ptr(w), _ptr(bias), 16, 1, _ptr(act_ref), 16,
                                   None, None, None))
        U.check(U.lib().ccu_head(_ptr(act_ref), _ptr(xlog), None, None, _ptr(head), 0.0, n, _ptr(out_ref), None,
                                 None, None, None))
        for store in (0, 1):
            act = torch.zeros(B, D, H, W, 16, dtype=torch.bfloat16, device="cuda")
            out = torch.empty(n, device="cuda")
            U.check(U.lib().ccu_conv3d_head(_ptr(a), 16, B, D, H, W, _ptr(w), _ptr(bias), _ptr(head), _ptr(xlog),
                                            _ptr(out), _ptr(act), store, None))
            torch.cuda.synchronize()
            assert torch.equal(out, out_ref), store
            if store or path == 1:
                assert torch.equal(act, act_ref)
            else:
                assert not bool(act.abs().sum())        # not stored
    finally:
        U.check(U.lib().ccu_set_conv_path(0))
    assert U.status() == 0


def test_adam_with_adaptive_clipping(U):
    """ccu_adam_clipped against a NumPy restatement: the first gradient sets
    the running norm, a ten times larger one is cut to 3x that mean, and
    the moments and parameters follow Adam on the scaled gradient."""
    rng = np.random.default_rng(9)
    n = 50_000
    p0 = rng.normal(size=n).astype(np.float32)
    grads = [rng.normal(size=n).astype(np.float32), 10 * rng.normal(size=n).astype(np.float32),
             rng.normal(size=n).astype(np.float32)]
    p, m, v = (torch.from_numpy(a.copy()).cuda() for a in (p0, np.zeros(n, np.float32), np.zeros(n, np.float32)))
    state = torch.zeros(3, dtype=torch.float64, device="cuda")
    lr, b1, b2, eps, ratio = 1e-2, 0.9, 0.999, 1e-8, 3.0
    rp, rm, rv = p0.astype(np.float64), np.zeros(n), np.zeros(n)
    ema = 0.0
    for step, g in enumerate(grads, start=1):
        gd = torch.from_numpy(g).cuda()
        U.check(U.lib().ccu_adam_clipped(_ptr(p), _ptr(gd), _ptr(m), _ptr(v), n, lr, b1, b2, eps, step, 0.0,
                                         _ptr(state), ratio, None))
        norm = float(np.sqrt(np.sum(g.astype(np.float64) ** 2)))
        ema = ema if ema > 0 else norm
        kept = min(norm, ratio * ema)
        scale = kept / norm
        ema = 0.95 * ema + 0.05 * kept
        gs = g * scale
        rm = b1 * rm + (1 - b1) * gs
        rv = b2 * rv + (1 - b2) * gs * gs
        rp -= lr * (rm / (1 - b1 ** step)) / (np.sqrt(rv / (1 - b2 ** step)) + eps)
        torch.cuda.synchronize()
        assert float(state[2]) == pytest.approx(scale, rel=1e-9)
        assert float(state[1]) == pytest.approx(ema, rel=1e-9)
    assert float(state[2]) == pytest.approx(1.0)
    np.testing.assert_allclose(p.cpu().numpy(), rp, rtol=1e-5, atol=1e-6)
    np.testing.assert_allclose(m.cpu().numpy(), rm, rtol=1e-4, atol=1e-7)
    np.testing.assert_allclose(v.cpu().numpy(), rv, rtol=1e-4, atol=1e-9)
