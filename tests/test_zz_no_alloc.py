"""The allocation-free entry point gives the allocating entry point's results (GPU, through the C ABI).

pd_cluster_compute_static is for callers that cannot call cudaMalloc: a plugin whose host
program's memory pool (CUDA.jl's, PyTorch's caching allocator) has already claimed the device
memory, a host with a fixed device-memory budget, or a real-time loop kept out of the
allocator.  Its scratch is one static device array shared by every call.  The tests run calls
in a row (same system moved, then other sizes and boxes) so that a call that saw the previous
call's leftovers would show, compare each call with the allocating entry point and with the FP64
oracle, and check that a warmed call leaves the device's free memory unchanged.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RC = 9.0


def _system(pd, n=3000, seed=5, L=None):
    L = (n / 0.0375) ** (1 / 3) if L is None else L
    pos, q, box = pd.synthetic.ionic_melt(n, L, 2.2, seed=seed)
    pos = pos.astype(np.float32).astype(np.float64)
    alpha = pd.splits.alpha_from_tolerance(RC, 1e-5)
    cp = pd.splits.coulomb_polynomial(alpha, pd.synthetic.COULOMB_EV_A, RC)
    table = pd.splits.lj_type_table(2.8, 0.01, RC)
    eng = pd.ClusterPairEngine(n, box, rmax=RC, skin=1.0, prune_buffer=0.3, lj=dict(table=table), coulomb=cp,
                               selfc=pd.splits.self_coefficient(alpha))
    return eng, pos, q, box, alpha


def _arrays(pos, q):
    import torch
    d = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float32, device="cuda")
    n = len(q)
    x, y, z, qq = d(pos[:, 0]), d(pos[:, 1]), d(pos[:, 2]), d(q)
    typ = torch.ones(n, dtype=torch.int32, device="cuda")
    out = [torch.zeros(n, device="cuda") for _ in range(4)] + [torch.zeros((n, 6), device="cuda")]
    return (x, y, z, qq, typ), out


def _static(pd, params, box, ins, outs):
    import torch
    x, y, z, q, typ = ins
    fx, fy, fz, e, w = outs
    stream = torch.cuda.current_stream().cuda_stream
    pd._native.call("pd_cluster_compute_static", C.byref(params), pd._native.dbl3(box), x.data_ptr(),
                    y.data_ptr(), z.data_ptr(), q.data_ptr(), typ.data_ptr(), fx.data_ptr(), fy.data_ptr(),
                    fz.data_ptr(), e.data_ptr(), w.data_ptr(), 1, stream)
    torch.cuda.synchronize()


def _allocating(eng, ins, outs):
    import torch
    x, y, z, q, typ = ins
    fx, fy, fz, e, w = outs
    eng.compute(x, y, z, q, typ, fx, fy, fz, e, w, energy=True)
    torch.cuda.synchronize()


def _host(outs):
    import torch
    fx, fy, fz, e, w = outs
    return (torch.stack([fx, fy, fz], 1).double().cpu().numpy(), e.double().cpu().numpy(),
            w.double().cpu().numpy())


def _close(a, b, tol=1e-5):
    """Relative agreement of forces, total energy and total virial (the Coulomb pair tests' bound)."""
    Fa, Ea, Wa = a
    Fb, Eb, Wb = b
    return (np.linalg.norm(Fa - Fb) / np.linalg.norm(Fb) < tol and abs(Ea.sum() - Eb.sum()) < tol * abs(Eb.sum())
            and np.linalg.norm(Wa.sum(0) - Wb.sum(0)) < tol * np.linalg.norm(Wb.sum(0)))


def _oracle(pd, ora, pos, q, box, alpha):
    Cc = pd.synthetic.COULOMB_EV_A
    ref = ora.pairs_cells(pos, box, q=q, kind=1, sigma=2.8, eps=0.01, rc_lj=RC, C=Cc, alpha=alpha, rc_coul=RC)
    self_e = -Cc * alpha / np.sqrt(np.pi) * (q * q)
    return ref["F"], ref["E"] + self_e, ref["W"]


def _check_call(pd, ora, eng, pos, q, box, alpha):
    ins, out_a = _arrays(pos, q)
    _, out_s = _arrays(pos, q)
    _allocating(eng, ins, out_a)
    _static(pd, eng.params, box, ins, out_s)
    got = _host(out_s)
    assert _close(got, _host(out_a)), "static entry point differs from the allocating one"
    assert _close(got, _oracle(pd, ora, pos, q, box, alpha)), "static entry point differs from the FP64 oracle"
    return ins, out_s


def test_static_scratch_matches_allocating_entry(pd, ora, cuda):
    import torch
    eng, pos, q, box, alpha = _system(pd)
    rng = np.random.default_rng(1)
    for call in range(2):   # two calls in a row: the second must not see the first's leftovers
        if call == 1:
            pos = (pos + rng.uniform(-0.05, 0.05, size=pos.shape)).astype(np.float32).astype(np.float64)
        ins, outs = _check_call(pd, ora, eng, pos, q, box, alpha)
    # a warmed call allocates nothing: device free memory and torch's allocated bytes are unchanged
    torch.cuda.synchronize()
    free0, alloc0 = torch.cuda.mem_get_info()[0], torch.cuda.memory_allocated()
    _static(pd, eng.params, box, ins, outs)
    free1, alloc1 = torch.cuda.mem_get_info()[0], torch.cuda.memory_allocated()
    assert free1 == free0 and alloc1 == alloc0, (free0 - free1, alloc1 - alloc0)
    eng.close()


def test_static_scratch_other_sizes_and_boxes(pd, ora, cuda):
    # the carved buffers move when N and the box change; each call still matches both references
    for n, seed, L in ((4000, 11, None), (600, 12, 26.0), (2400, 13, 38.0), (600, 14, 26.0)):
        eng, pos, q, box, alpha = _system(pd, n=n, seed=seed, L=L)
        _check_call(pd, ora, eng, pos, q, box, alpha)
        eng.close()


def test_static_scratch_error_then_clean_call(pd, ora, cuda):
    # a non-finite coordinate latches PD_ENONFINITE in the arena's status word; the next call clears it
    eng, pos, q, box, alpha = _system(pd, n=1000, seed=3, L=30.0)
    bad = pos.copy()
    bad[17, 2] = np.nan
    ins, outs = _arrays(bad, q)
    with pytest.raises(pd._native.NativeError) as ei:
        _static(pd, eng.params, box, ins, outs)
    assert ei.value.code == pd._native.PD_ENONFINITE
    _check_call(pd, ora, eng, pos, q, box, alpha)
    eng.close()


def test_static_scratch_rejects_oversize(pd, cuda):
    eng, pos, q, box, _ = _system(pd)
    params = pd._native.ClusterParams.from_buffer_copy(eng.params)
    params.n = 4097   # one more than PD_STATIC_MAX_N
    ins, outs = _arrays(np.zeros((4, 3)), np.zeros(4))
    with pytest.raises(pd._native.NativeError) as ei:
        _static(pd, params, box, ins, outs)
    assert ei.value.code == pd._native.PD_EINVAL
    assert "static scratch serves" in str(ei.value)
    eng.close()
