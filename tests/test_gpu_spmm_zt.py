"""The blocked forward PF product through the lines-fastest Radon output (dfx_spmm_pf_forward_blocked_zt) against the
blocked product on the channel-fastest output (dfx_spmm_pf_forward_blocked), bit for bit, on synthetic eta-blocked
rows: rings below, at and above eight (ring groups), detector lines below and above 288 (several line blocks), one
and several line groups per warp, all angles and omega subsets, a transpose buffer of one angle (chunks of one
angle) and of all of them, data rows accumulated onto (+=) and bins whose rows are empty left untouched. The
operator-level products are checked against the CSR kernel in tests/test_gpu_operator.py (storage modes)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _blocked_rows(rng, R, P, C, kb, max_len=24):
    """Random eta-blocked rows of R angles: (fb_ptr, fb_k, fb_v (n, 4), mask) as the builder lays them out (k
    ascending per block row, value 0 where the bin's row has no entry, mask bit u set iff bin 4 cb + u has one)."""
    ncb = -(-C // 4)
    n = R * P * ncb
    ptr, ks, vs, mask = [0], [], [], np.zeros(n, np.uint8)
    for g in range(n):
        cb = (g % (P * ncb)) // P
        valid = [4 * cb + u < C for u in range(4)]
        cnt = int(rng.integers(0, max_len + 1)) if rng.random() > 0.1 else 0
        k = np.sort(rng.choice(kb, size=min(cnt, kb), replace=False))
        v = rng.standard_normal((len(k), 4)).astype(np.float32)
        live = np.array([valid[u] and rng.random() > 0.25 for u in range(4)])
        v[:, ~live] = 0.0
        v[rng.random(v.shape) < 0.3] = 0.0                 # a bin's row may lack some of the block's orientations
        m = 0
        for u in range(4):
            if live[u] and len(k) and np.any(v[:, u] != 0):
                m |= 1 << u
            else:
                v[:, u] = 0.0
        keep = np.any(v != 0, axis=1)
        k, v = k[keep], v[keep]
        mask[g] = m
        ks.append(k.astype(np.uint16))
        vs.append(v)
        ptr.append(ptr[-1] + len(k))
    fk = np.concatenate(ks) if ptr[-1] else np.zeros(1, np.uint16)
    fv = np.concatenate(vs) if ptr[-1] else np.zeros((1, 4), np.float32)
    return np.array(ptr, np.int32), fk, fv, mask


@pytest.mark.parametrize("P,C,my,kb,R,subset", [
    (8, 36, 263, 300, 5, None),
    (8, 18, 263, 1012, 3, [2, 0]),
    (3, 10, 40, 77, 4, [3, 0, 2]),
    (1, 7, 31, 33, 3, None),
    (12, 9, 70, 64, 2, [1]),
    (32, 5, 300, 50, 2, None),
])
@pytest.mark.parametrize("max_groups,one_angle", [(0, False), (1, True), (4, False)])
def test_lines_fastest_blocked_forward_equals_blocked(P, C, my, kb, R, subset, max_groups, one_angle):
    from diffractom_b200 import _lib
    rng = np.random.default_rng(P * 1000 + my + kb + max_groups)
    ptr, fk, fv, mask = _blocked_rows(rng, R, P, C, kb)
    kstride = kb + 5
    n_sub = R if subset is None else len(subset)
    dev = "cuda"
    sino = torch.as_tensor(rng.standard_normal((n_sub, my, kstride)).astype(np.float32), device=dev)
    data0 = torch.as_tensor(rng.standard_normal((R, my, C * P)).astype(np.float32), device=dev)
    t_ptr = torch.as_tensor(ptr, device=dev)
    t_k = torch.as_tensor(fk.view(np.int16), device=dev)
    t_v = torch.as_tensor(fv, device=dev).contiguous()
    t_m = torch.as_tensor(mask, device=dev)
    om = None if subset is None else torch.as_tensor(np.array(subset, np.int32), device=dev)
    om_ptr = None if om is None else om.data_ptr()
    s = torch.cuda.current_stream().cuda_stream
    a, b = data0.clone(), data0.clone()
    _lib.call("dfx_spmm_pf_forward_blocked", sino.data_ptr(), t_ptr.data_ptr(), t_k.data_ptr(), t_v.data_ptr(),
              t_m.data_ptr(), a.data_ptr(), om_ptr, n_sub, my, P, C, kstride, kb, s)
    per = int(_lib.lib().dfx_spmm_pf_forward_zt_floats(1, my, kb))
    assert per == kb * 32 * (-(-my // 32))
    zt = torch.full((per if one_angle else per * n_sub,), float("nan"), device=dev)
    _lib.call("dfx_spmm_pf_forward_blocked_zt", sino.data_ptr(), zt.data_ptr(), zt.numel(), t_ptr.data_ptr(),
              t_k.data_ptr(), t_v.data_ptr(), t_m.data_ptr(), b.data_ptr(), om_ptr, n_sub, my, P, C, kstride, kb,
              max_groups, s)
    torch.cuda.synchronize()
    assert torch.equal(a, b)
    assert not torch.equal(a, data0)
    # bins without entries keep their values bit for bit (no += 0 on them)
    rows = set(range(R)) if subset is None else set(subset)
    for r in set(range(R)) - rows:
        assert torch.equal(b[r], data0[r])


def test_lines_fastest_blocked_forward_rejects_bad_arguments():
    from diffractom_b200 import _lib
    lib = _lib.lib()
    dev = "cuda"
    x = torch.zeros(64, device=dev)
    i = torch.zeros(64, dtype=torch.int32, device=dev)
    s = torch.cuda.current_stream().cuda_stream
    per = int(lib.dfx_spmm_pf_forward_zt_floats(1, 40, 8))
    # buffer smaller than one angle, more than 32 rings, max_groups out of range
    for zt_n, P, mg in [(per - 1, 2, 0), (per, 33, 0), (per, 2, 10)]:
        rc = lib.dfx_spmm_pf_forward_blocked_zt(x.data_ptr(), x.data_ptr(), zt_n, i.data_ptr(), i.data_ptr(),
                                                x.data_ptr(), i.data_ptr(), x.data_ptr(), None, 1, 40, P, 4, 8, 8,
                                                mg, s)
        assert rc != 0
    assert lib.dfx_spmm_pf_forward_zt_floats(0, 40, 8) < 0


def _csr_rows(rng, n_rows, n_cols, max_len):
    """Random CSR rows (columns ascending, distinct): (row_ptr int32, cols uint16, vals float32)."""
    ptr, cols, vals = [0], [], []
    for _ in range(n_rows):
        cnt = int(rng.integers(0, max_len + 1)) if rng.random() > 0.1 else 0
        c = np.sort(rng.choice(n_cols, size=min(cnt, n_cols), replace=False)).astype(np.uint16)
        cols.append(c)
        vals.append(rng.standard_normal(len(c)).astype(np.float32))
        ptr.append(ptr[-1] + len(c))
    c = np.concatenate(cols) if ptr[-1] else np.zeros(1, np.uint16)
    v = np.concatenate(vals) if ptr[-1] else np.zeros(1, np.float32)
    return np.array(ptr, np.int32), c, v


def _csr_rows_fast(rng, n_rows, n_cols, max_len):
    """As _csr_rows, vectorised (many rows)."""
    L = np.minimum(rng.integers(0, max_len + 1, n_rows), n_cols)
    L[rng.random(n_rows) < 0.1] = 0
    order = np.argsort(rng.random((n_rows, n_cols)), axis=1)
    chosen = np.where(np.arange(n_cols)[None, :] < L[:, None], order, n_cols)
    chosen.sort(axis=1)
    cols = chosen[chosen < n_cols].astype(np.uint16)
    ptr = np.concatenate([[0], np.cumsum(L)]).astype(np.int32)
    vals = rng.standard_normal(len(cols)).astype(np.float32)
    return ptr, (cols if len(cols) else np.zeros(1, np.uint16)), (vals if len(vals) else np.zeros(1, np.float32))


@pytest.mark.parametrize("cp,my,kb,R,subset,compact", [
    (30, 40, 2000, 30, None, 0),          # many blocks: four orientation rows per warp
    (30, 40, 2000, 20, None, 1),          # two per warp
    (2880, 263, 300, 4, None, 0),
    (2880, 263, 1012, 3, [2, 0], 0),
    (30, 40, 77, 4, [3, 0, 2], 1),
    (7, 31, 33, 3, None, 0),
    (108, 300, 64, 2, [1], 1),
])
@pytest.mark.parametrize("max_groups,one_angle", [(0, False), (1, True), (4, False)])
def test_lines_fastest_adjoint_equals_adjoint(cp, my, kb, R, subset, compact, max_groups, one_angle):
    from diffractom_b200 import _lib
    rng = np.random.default_rng(cp + my + kb + max_groups + compact)
    n_sub = R if subset is None else len(subset)
    rows = (n_sub if compact else R) * kb
    ptr, col, val = (_csr_rows if rows < 5000 else _csr_rows_fast)(rng, rows, cp, 48)
    kstride = kb + 7
    dev = "cuda"
    data = torch.as_tensor(rng.standard_normal((R, my, cp)).astype(np.float32), device=dev)
    t_ptr = torch.as_tensor(ptr, device=dev)
    t_c = torch.as_tensor(col.view(np.int16), device=dev)
    t_v = torch.as_tensor(val, device=dev)
    om = None if subset is None else torch.as_tensor(np.array(subset, np.int32), device=dev)
    om_ptr = None if om is None else om.data_ptr()
    s = torch.cuda.current_stream().cuda_stream
    alpha = float(np.float32(0.37))
    a = torch.full((n_sub, my, kstride), -5.0, device=dev)
    b = torch.full((n_sub, my, kstride), -6.0, device=dev)
    _lib.call("dfx_spmm_pf_adjoint", data.data_ptr(), t_ptr.data_ptr(), t_c.data_ptr(), t_v.data_ptr(), a.data_ptr(),
              om_ptr, n_sub, my, kb, cp, kstride, alpha, compact, s)
    per = int(_lib.lib().dfx_spmm_pf_adjoint_zt_floats(1, my, cp))
    assert per == cp * 32 * (-(-my // 32))
    dt = torch.full((per if one_angle else per * n_sub,), float("nan"), device=dev)
    _lib.call("dfx_spmm_pf_adjoint_zt", data.data_ptr(), dt.data_ptr(), dt.numel(), t_ptr.data_ptr(), t_c.data_ptr(),
              t_v.data_ptr(), b.data_ptr(), om_ptr, n_sub, my, kb, cp, kstride, alpha, compact, max_groups, s)
    torch.cuda.synchronize()
    assert torch.equal(a, b)
    assert torch.all(b[:, :, kb:] == 0)
