"""The tcgen05 BF16 pole-figure products against float32 GEMMs of the same BF16 operands: ragged sizes (K and CP not
multiples of the 64-wide slices or of the 128-row tiles, one and two translation tiles), subset angle lists, the
accumulate flag, untouched rows, and the device-side wait flags."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _lib():
    from diffractom_b200 import _lib
    return _lib


def tc_flags():
    f = ctypes.c_uint(0)
    _lib().check(_lib().lib().dfx_tc_status(ctypes.byref(f), 1))
    return f.value


def rand_bf16(shape, gen, density=1.0):
    x = torch.rand(shape, generator=gen, device="cuda") * 2 - 1
    if density < 1.0:
        x = x * (torch.rand(shape, generator=gen, device="cuda") < density)
    return x.to(torch.bfloat16)


def test_pf_tc_products_with_a_compact_pf():
    """A PF of the subset's angles only (n_sub, Ktot, CPpad; pf_compact = 1, as generated for one subset) gives the
    products of the full PF of all angles bit for bit, forward (into the subset's data rows) and adjoint."""
    lib = _lib()
    gen = torch.Generator(device="cuda").manual_seed(17)
    R, ktot, CP, cp_pad, my = 6, 264, 700, 704, 131
    pf = rand_bf16((R, ktot, cp_pad), gen, density=0.2)
    pf[:, :, CP:] = 0
    omegas = torch.tensor([5, 1, 3], dtype=torch.int32, device="cuda")
    n_sub = omegas.numel()
    pfc = pf[omegas.long()].contiguous()
    z = rand_bf16((n_sub, my, ktot), gen)
    d = rand_bf16((R, my, cp_pad), gen)
    s = torch.cuda.current_stream().cuda_stream
    tc_flags()
    out = []
    for src, compact in ((pf, 0), (pfc, 1)):
        data = torch.full((R, my, CP), 3.0, device="cuda")
        lib.call("dfx_pf_tc_forward", src.data_ptr(), ktot, 0, ktot, CP, cp_pad, R, z.data_ptr(), omegas.data_ptr(),
                 n_sub, my, data.data_ptr(), 1, compact, s)
        zo = torch.zeros((n_sub, my, ktot), dtype=torch.bfloat16, device="cuda")
        lib.call("dfx_pf_tc_adjoint", src.data_ptr(), ktot, 0, ktot, CP, cp_pad, R, d.data_ptr(), omegas.data_ptr(),
                 n_sub, my, 0.75, zo.data_ptr(), compact, s)
        torch.cuda.synchronize()
        out.append((data, zo))
    assert torch.equal(out[0][0], out[1][0]) and torch.equal(out[0][1], out[1][1])
    assert tc_flags() == 0


@pytest.mark.parametrize("my", [103, 263])
def test_pf_tc_products_match_fp32_gemm(my):
    lib = _lib()
    gen = torch.Generator(device="cuda").manual_seed(my)
    R, ktot, CP = 5, 392, 900
    cp_pad = 904
    pf = rand_bf16((R, ktot, cp_pad), gen, density=0.2)
    pf[:, :, CP:] = 0
    omegas = torch.tensor([3, 0, 4], dtype=torch.int32, device="cuda")
    n_sub = omegas.numel()
    z = rand_bf16((n_sub, my, ktot), gen)
    tc_flags()
    s = torch.cuda.current_stream().cuda_stream
    data = torch.full((R, my, CP), 7.0, device="cuda")
    lib.call("dfx_pf_tc_forward", pf.data_ptr(), ktot, 0, ktot, CP, cp_pad, R, z.data_ptr(), omegas.data_ptr(),
             n_sub, my, data.data_ptr(), 0, 0, s)
    ref = torch.stack([z[i].float() @ pf[int(r), :, :CP].float() for i, r in enumerate(omegas.tolist())])
    got = data[omegas.long()]
    assert float((got - ref).abs().max() / ref.abs().max()) < 1e-5
    assert torch.all(data[[1, 2]] == 7.0)
    lib.call("dfx_pf_tc_forward", pf.data_ptr(), ktot, 0, ktot, CP, cp_pad, R, z.data_ptr(), omegas.data_ptr(),
             n_sub, my, data.data_ptr(), 1, 0, s)
    assert float((data[omegas.long()] - 2 * ref).abs().max() / ref.abs().max()) < 1e-5
    # a range of orientations (one batch of a wider Z): rows k0 .. k0+kn-1 only, nothing read past them
    k0, kn = 104, 200
    lib.call("dfx_pf_tc_forward", pf.data_ptr(), ktot, k0, kn, CP, cp_pad, R, z.data_ptr(), omegas.data_ptr(),
             n_sub, my, data.data_ptr(), 0, 0, s)
    ref = torch.stack([z[i, :, k0:k0 + kn].float() @ pf[int(r), k0:k0 + kn, :CP].float()
                       for i, r in enumerate(omegas.tolist())])
    assert float((data[omegas.long()] - ref).abs().max() / ref.abs().max()) < 1e-5

    d = rand_bf16((R, my, cp_pad), gen)
    d[:, :, CP:] = 0
    zo = torch.zeros((n_sub, my, ktot), dtype=torch.bfloat16, device="cuda")
    alpha = 57.29
    lib.call("dfx_pf_tc_adjoint", pf.data_ptr(), ktot, 0, ktot, CP, cp_pad, R, d.data_ptr(), omegas.data_ptr(),
             n_sub, my, alpha, zo.data_ptr(), 0, s)
    ref = torch.stack([alpha * (d[int(r)].float() @ pf[int(r)].float().T) for r in omegas.tolist()])
    # the output is rounded to BF16 once: within half a BF16 ulp of the float32 value (2^-9 relative)
    err = (zo.float() - ref).abs()
    assert bool(torch.all(err <= ref.abs() * 2.0 ** -8 + 1e-6 * float(ref.abs().max())))
    zo.fill_(3.0)
    lib.call("dfx_pf_tc_adjoint", pf.data_ptr(), ktot, k0, kn, CP, cp_pad, R, d.data_ptr(), omegas.data_ptr(),
             n_sub, my, alpha, zo.data_ptr(), 0, s)
    err = (zo[:, :, k0:k0 + kn].float() - ref[:, :, k0:k0 + kn]).abs()
    assert bool(torch.all(err <= ref[:, :, k0:k0 + kn].abs() * 2.0 ** -8 + 1e-6 * float(ref.abs().max())))
    assert torch.all(zo[:, :, :k0] == 3.0) and torch.all(zo[:, :, k0 + kn:] == 3.0)
    torch.cuda.synchronize()
    assert tc_flags() == 0


def test_rows_to_bf16_and_dense_bf16_padding():
    lib = _lib()
    gen = torch.Generator(device="cuda").manual_seed(3)
    R, my, CP, cp_pad = 4, 7, 10, 16
    x = torch.rand((R, my, CP), generator=gen, device="cuda")
    out = torch.full((R, my, cp_pad), 5.0, dtype=torch.bfloat16, device="cuda")
    om = torch.tensor([2, 0], dtype=torch.int32, device="cuda")
    lib.call("dfx_rows_to_bf16", x.data_ptr(), out.data_ptr(), om.data_ptr(), 2, my, CP, cp_pad,
             torch.cuda.current_stream().cuda_stream)
    for r in (0, 2):
        assert torch.equal(out[r, :, :CP], x[r].to(torch.bfloat16))
        assert torch.all(out[r, :, CP:] == 0)
    assert torch.all(out[[1, 3]] == 5.0)


def test_tc_argument_errors():
    lib = _lib()
    pf = torch.zeros((2, 16, 16), dtype=torch.bfloat16, device="cuda")
    z = torch.zeros((2, 3, 16), dtype=torch.bfloat16, device="cuda")
    data = torch.zeros((2, 3, 16), device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    with pytest.raises(ValueError):      # Ktot not a multiple of 8
        lib.call("dfx_pf_tc_forward", pf.data_ptr(), 12, 0, 12, 16, 16, 2, z.data_ptr(), None, 2, 3, data.data_ptr(),
                 0, 0, s)
    with pytest.raises(ValueError):      # cp_pad < cp
        lib.call("dfx_pf_tc_forward", pf.data_ptr(), 16, 0, 16, 16, 8, 2, z.data_ptr(), None, 2, 3, data.data_ptr(),
                 0, 0, s)
    with pytest.raises(ValueError):      # orientation range start not a multiple of 8 / past Ktot
        lib.call("dfx_pf_tc_forward", pf.data_ptr(), 16, 4, 8, 16, 16, 2, z.data_ptr(), None, 2, 3, data.data_ptr(),
                 0, 0, s)
    with pytest.raises(ValueError):
        lib.call("dfx_pf_tc_forward", pf.data_ptr(), 16, 8, 16, 16, 16, 2, z.data_ptr(), None, 2, 3, data.data_ptr(),
                 0, 0, s)
    with pytest.raises(ValueError):      # misaligned operand
        lib.call("dfx_pf_tc_forward", pf.data_ptr() + 2, 16, 0, 16, 16, 16, 2, z.data_ptr(), None, 2, 3,
                 data.data_ptr(), 0, 0, s)
