"""The allocation-free entry point gives the allocating entry point's results (GPU, through the C ABI).

pd_cluster_compute_static is for callers that cannot call cudaMalloc (a fixed device
memory budget, code running while a graph region is built, a real-time loop kept out of the
allocator): its scratch is one static device array shared by every call.  Two calls in a
row check that a call does not see the previous call's leftovers.
"""
import ctypes as C
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _system(pd, n=3000, seed=5):
    L = (n / 0.0375) ** (1 / 3)
    pos, q, box = pd.synthetic.ionic_melt(n, L, 2.2, seed=seed)
    rc = 9.0
    alpha = pd.splits.alpha_from_tolerance(rc, 1e-5)
    cp = pd.splits.coulomb_polynomial(alpha, pd.synthetic.COULOMB_EV_A, rc)
    table = pd.splits.lj_type_table(2.8, 0.01, rc)
    eng = pd.ClusterPairEngine(n, box, rmax=rc, skin=1.0, prune_buffer=0.3, lj=dict(table=table), coulomb=cp,
                               selfc=pd.splits.self_coefficient(alpha))
    return eng, pos, q, box


def _arrays(pos, q):
    import torch
    d = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float32, device="cuda")
    n = len(q)
    x, y, z, qq = d(pos[:, 0]), d(pos[:, 1]), d(pos[:, 2]), d(q)
    typ = torch.ones(n, dtype=torch.int32, device="cuda")
    out = [torch.zeros(n, device="cuda") for _ in range(4)] + [torch.zeros((n, 6), device="cuda")]
    return (x, y, z, qq, typ), out


def _static(pd, eng, box, ins, outs):
    import torch
    x, y, z, q, typ = ins
    fx, fy, fz, e, w = outs
    stream = torch.cuda.current_stream().cuda_stream
    pd._native.call("pd_cluster_compute_static", C.byref(eng.params), pd._native.dbl3(box), x.data_ptr(),
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


def test_static_scratch_matches_allocating_entry(pd, cuda):
    eng, pos, q, box = _system(pd)
    rng = np.random.default_rng(1)
    for call in range(2):   # two calls in a row: the second must not see the first's leftovers
        if call == 1:
            pos = pos + rng.uniform(-0.05, 0.05, size=pos.shape)
        ins, out_a = _arrays(pos, q)
        _, out_s = _arrays(pos, q)
        _allocating(eng, ins, out_a)
        _static(pd, eng, box, ins, out_s)
        Fa, Ea, Wa = _host(out_a)
        Fs, Es, Ws = _host(out_s)
        # the parity bound the Coulomb pair tests use (relative RMS 1e-5)
        assert np.linalg.norm(Fs - Fa) / np.linalg.norm(Fa) < 1e-5, call
        assert abs(Es.sum() - Ea.sum()) < 1e-5 * abs(Ea.sum()), call
        assert np.linalg.norm(Ws.sum(0) - Wa.sum(0)) < 1e-5 * np.linalg.norm(Wa.sum(0)), call
    eng.close()


def test_static_scratch_rejects_oversize(pd, cuda):
    eng, pos, q, box = _system(pd)
    params = pd._native.ClusterParams.from_buffer_copy(eng.params)
    params.n = 4097   # one more than PD_STATIC_MAX_N
    ins, outs = _arrays(np.zeros((4, 3)), np.zeros(4))
    with pytest.raises(pd._native.NativeError) as ei:
        _static(pd, type("E", (), {"params": params})(), box, ins, outs)
    assert ei.value.code == pd._native.PD_EINVAL
    assert "static scratch serves" in str(ei.value)
    eng.close()
