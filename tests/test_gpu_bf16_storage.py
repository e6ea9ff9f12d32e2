"""The storage kernels of BF16 runs too large for float32 step sizes and sinograms: strided float32 <-> BF16 row
conversion (round to nearest one way, exact widening the other, untouched columns past the rows), the step sizes
rounded toward zero (never above the float32 value), and the primal update reading them, bit for bit the float32
update given the widened steps."""
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _lib():
    from diffractom_b200 import _lib
    return _lib


def test_convert_rows_both_ways():
    lib = _lib()
    g = torch.Generator(device="cuda").manual_seed(4)
    rows, cols, ld32, ld16 = 37, 75, 80, 136
    f = torch.randn((rows, ld32), generator=g, device="cuda") * 100
    b = torch.full((rows, ld16), 9.0, dtype=torch.bfloat16, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    lib.call("dfx_convert_rows", 1, f.data_ptr(), ld32, b.data_ptr() + 2 * 16, ld16, rows, cols, s)
    torch.cuda.synchronize()
    assert torch.equal(b[:, 16:16 + cols], f[:, :cols].to(torch.bfloat16))
    assert torch.all(b[:, :16] == 9.0) and torch.all(b[:, 16 + cols:] == 9.0)
    back = torch.full((rows, ld32), -1.0, device="cuda")
    lib.call("dfx_convert_rows", 0, back.data_ptr(), ld32, b.data_ptr() + 2 * 16, ld16, rows, cols, s)
    torch.cuda.synchronize()
    assert torch.equal(back[:, :cols], b[:, 16:16 + cols].float())
    assert torch.all(back[:, cols:] == -1.0)
    lib.call("dfx_convert_rows", 1, f.data_ptr(), ld32, b.data_ptr(), ld16, 0, cols, s)      # nothing to do
    with pytest.raises(ValueError):
        lib.call("dfx_convert_rows", 1, f.data_ptr(), 10, b.data_ptr(), ld16, rows, cols, s)


def test_steps_toward_zero_and_the_bf16_primal_update():
    lib = _lib()
    g = torch.Generator(device="cuda").manual_seed(5)
    n = 100_003
    T = torch.rand(n, generator=g, device="cuda") * 1e3
    T[::7] = 0.0
    T16 = torch.empty(n, dtype=torch.bfloat16, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    lib.call("dfx_f32_to_bf16_rz", T.data_ptr(), T16.data_ptr(), n, s)
    torch.cuda.synchronize()
    trunc = (T.view(torch.int32) & -65536).view(torch.float32)       # the upper 16 bits: rounding toward zero
    assert torch.equal(T16.float(), trunc)
    assert torch.all(T16.float() <= T)
    x0 = torch.rand(n, generator=g, device="cuda")
    z0 = torch.randn(n, generator=g, device="cuda")
    dz = torch.randn(n, generator=g, device="cuda") * 1e-3
    x1, z1, x2, z2 = x0.clone(), z0.clone(), x0.clone(), z0.clone()
    Tw = T16.float()
    lib.call("dfx_spdhg_primal_update", x1.data_ptr(), z1.data_ptr(), Tw.data_ptr(), dz.data_ptr(), 3.0, 0.25, n, s)
    lib.call("dfx_spdhg_primal_update_t16", x2.data_ptr(), z2.data_ptr(), T16.data_ptr(), dz.data_ptr(), 3.0, 0.25,
             n, s)
    torch.cuda.synchronize()
    assert torch.equal(x1, x2) and torch.equal(z1, z2)
    assert torch.all(x2[::7] == 0.0)
