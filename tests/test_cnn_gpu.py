"""BF16 tensor-core 3-D convolutions of the learned preconditioner against
torch's FP32 convolution of the same BF16-rounded operands.  FP32
accumulation in another order: rel-L2 1e-5 for outputs computed in FP32;
1e-2 where the result is stored as BF16."""
import pytest
import torch
import torch.nn.functional as F

from helpers import rel_l2

pytestmark = pytest.mark.gpu
DEFAULT_FORM = "tcgen05-tma"


@pytest.fixture(scope="module", autouse=True)
def _ready():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _torch_w(w):
    """[27][co][ci] -> torch [co][ci][3][3][3] (tap = kd*9 + kh*3 + kw)."""
    return w.float().reshape(3, 3, 3, 16, 16).permute(3, 4, 0, 1, 2).contiguous()


def _ncdhw(x):
    return x.float().permute(3, 0, 1, 2).unsqueeze(0)


@pytest.mark.parametrize("shape", [(5, 7, 37), (3, 4, 16), (6, 9, 50)])
@pytest.mark.parametrize("relu", [False, True])
def test_forward_matches_torch(shape, relu):
    from efwi.cnn import conv3d_raw
    g = torch.Generator(device="cuda").manual_seed(1)
    x = torch.randn(shape + (16,), device="cuda", generator=g).to(torch.bfloat16)
    w = (0.2 * torch.randn(27, 16, 16, device="cuda", generator=g)).to(torch.bfloat16)
    b = torch.randn(16, device="cuda", generator=g)
    ours = conv3d_raw(x, w, b, relu, out_f32=True)
    ref = F.conv3d(_ncdhw(x), _torch_w(w), b, padding=1)
    if relu:
        ref = torch.relu(ref)
    ref = ref[0].permute(1, 2, 3, 0)
    assert rel_l2(ours.cpu(), ref.cpu()) < 1e-5
    ours_b = conv3d_raw(x, w, b, relu)
    assert rel_l2(ours_b.float().cpu(), ref.cpu()) < 1e-2


@pytest.mark.parametrize("form_tc", ["tcgen05", "tcgen05-tma", "tcgen05-tma3", "tcgen05-ws",
                                     "tcgen05-ws3"])
@pytest.mark.parametrize("shape", [(1, 1, 1), (3, 17, 9), (4, 33, 70), (2, 16, 8)])
def test_tcgen05_form_matches_mma_form_and_torch(shape, form_tc):
    """The tcgen05 convolution (accumulator in tensor memory) against the
    mma.sync one and torch, on tiles cut at every edge (8 x 16 voxel tiles)."""
    from efwi.cnn import conv3d_raw, conv3d_status, set_conv_kernel
    g = torch.Generator(device="cuda").manual_seed(5)
    x = torch.randn(shape + (16,), device="cuda", generator=g).to(torch.bfloat16)
    w = (0.2 * torch.randn(27, 16, 16, device="cuda", generator=g)).to(torch.bfloat16)
    b = torch.randn(16, device="cuda", generator=g)
    ref = torch.relu(F.conv3d(_ncdhw(x), _torch_w(w), b, padding=1))[0].permute(1, 2, 3, 0)
    try:
        set_conv_kernel("mma")
        mma = conv3d_raw(x, w, b, True, out_f32=True)
        for form in (form_tc,):
            set_conv_kernel(form)
            tc = conv3d_raw(x, w, b, True, out_f32=True)
            tcb = conv3d_raw(x, w, b, True)
            torch.cuda.synchronize()
            assert not conv3d_status()
            assert rel_l2(tc.cpu(), ref.cpu()) < 1e-5, form
            assert rel_l2(tc.cpu(), mma.cpu()) < 1e-5, form
            assert rel_l2(tcb.float().cpu(), ref.cpu()) < 1e-2, form
    finally:
        set_conv_kernel(DEFAULT_FORM)


@pytest.mark.parametrize("shape", [(1, 1, 1), (3, 17, 9), (6, 7, 41), (5, 40, 24)])
def test_tcgen05_weight_gradient_matches_mma_and_torch(shape):
    """The tcgen05 weight gradient (eight taps per MMA) against the mma.sync
    one and torch's FP32 conv3d_weight of the same BF16 operands, on units
    (8 x 16 voxels) cut at every edge; 1e-5 rel-L2."""
    from efwi.cnn import conv3d_status, conv3d_wgrad, set_wgrad_kernel
    g = torch.Generator(device="cuda").manual_seed(9)
    x = torch.randn(shape + (16,), device="cuda", generator=g).to(torch.bfloat16)
    dy = torch.randn(shape + (16,), device="cuda", generator=g).to(torch.bfloat16)
    w = torch.zeros(27, 16, 16)
    ref = torch.nn.grad.conv3d_weight(_ncdhw(x), _torch_w(w).shape, _ncdhw(dy), padding=1)
    ref = ref.permute(2, 3, 4, 0, 1).reshape(27, 16, 16)
    try:
        set_wgrad_kernel("mma")
        mma = conv3d_wgrad(x, dy)
        set_wgrad_kernel("tcgen05")
        tc = conv3d_wgrad(x, dy)
        torch.cuda.synchronize()
        assert not conv3d_status()
    finally:
        set_wgrad_kernel("tcgen05")
    assert rel_l2(tc.cpu(), ref.cpu()) < 1e-5
    assert rel_l2(tc.cpu(), mma.cpu()) < 1e-5


def test_input_and_weight_gradients_match_torch():
    from efwi.cnn import conv3d_raw, conv3d_wgrad
    g = torch.Generator(device="cuda").manual_seed(2)
    shape = (6, 7, 41)
    x = torch.randn(shape + (16,), device="cuda", generator=g).to(torch.bfloat16)
    w = (0.2 * torch.randn(27, 16, 16, device="cuda", generator=g)).to(torch.bfloat16)
    dy = torch.randn(shape + (16,), device="cuda", generator=g).to(torch.bfloat16)
    wt = w.flip(0).transpose(1, 2).contiguous()
    dx = conv3d_raw(dy, wt, None, False, out_f32=True)
    ref_dx = torch.nn.grad.conv3d_input(_ncdhw(x).shape, _torch_w(w), _ncdhw(dy), padding=1)
    assert rel_l2(dx.cpu(), ref_dx[0].permute(1, 2, 3, 0).cpu()) < 1e-5
    dw = conv3d_wgrad(x, dy)
    ref_dw = torch.nn.grad.conv3d_weight(_ncdhw(x), _torch_w(w).shape, _ncdhw(dy), padding=1)
    ref_dw = ref_dw.permute(2, 3, 4, 0, 1).reshape(27, 16, 16)
    assert rel_l2(dw.cpu(), ref_dw.cpu()) < 1e-5


def test_network_trains():
    """A few Adam steps on one (features, target) pair lower the loss; the
    autograd path runs every kernel (forward, input gradient, weight
    gradient)."""
    from efwi.cnn import Preconditioner
    torch.manual_seed(0)
    net = Preconditioner(cin=3, seed=3).cuda()
    feats = torch.randn(3, 12, 14, 40, device="cuda")
    target = torch.tanh(feats[0] - 0.5 * feats[1])
    opt = torch.optim.Adam(net.parameters(), lr=3e-3)
    losses = []
    for _ in range(30):
        opt.zero_grad()
        loss = torch.mean((net(feats) - target) ** 2)
        loss.backward()
        opt.step()
        losses.append(loss.item())
    assert losses[-1] < 0.7 * losses[0]
